// Internal interfaces between the C-ABI layer (swg_api.cu) and the kernel files.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace swg {

enum { kModeSwgMpi = 0, kModeSwgMs = 1, kModeNw = 2 };

// One plain-kernel launch: the pairs of one block.
struct PlainJob {
  const uint8_t* seq;      // device: concatenated residues
  const int64_t* off;      // device: offsets, count + 1 entries
  int rs, re, cs, ce;      // block (inclusive global indices)
  int tri;                 // 1: pairs (i, j) with cs <= j < i (diagonal SWG-MPI/NW block)
  long long npairs;
  int16_t* out;            // device output
  long long ld;
  int out_r0, out_c0;      // global index of out's element (0, 0)
  int mirror;              // also write (j, i)
  const int16_t* scores;   // device [128*128]
  const uint8_t* flags;    // device [128*128]
  int o, e;
  int mode;
  int protein;
  void* carry;             // device scratch, plain_carry_bytes(mode, threads, maxlen, dist_fn)
  const int2* list;        // optional explicit pairs (s1 index, s2 index); replaces the block
  const int* list_count;   // device count of list entries (at most npairs are read)
  // optional query set (serving; list mode only): s1 index = query slot, distance to qout[slot][j]
  const uint8_t* qseq;
  const int64_t* qoff;
  const int32_t* qlen;
  int16_t* const* qout;
  int dist_fn;             // SW_DIST_*: Kimura2 / JukesCantor count transitions on the path
  int* throws;             // set when SWG-MPI JukesCantor meets log(0) (the reference throws)
};

struct sw_pair_result_dev {
  int score, score_is_neg_inf;
  int end1, end2, start1, start2, identity, similarity, gaps, length;
  int diag, transitions, transversions;  // for Kimura2 / JukesCantor
};

struct PairJob {
  const uint8_t* s1;
  const uint8_t* s2;
  int m, n;
  const int16_t* scores;
  const uint8_t* flags;
  int o, e;
  void* carry;  // pair_carry_bytes(n)
  sw_pair_result_dev* out;
};

// Second step of the two-pass SW path: for each pair the first pass found the best cell
// (ie, je) and score S of, the counters of the reference's traceback path from a DP confined to
// a region around that path (box_scan_kernel + box_band_kernel, then box_kernel for the pairs
// whose region the first two cannot hold).
struct BoxJob {
  const uint8_t* seq;      // dense residue codes 0..A-1 (the engine's), same offsets as the residues
  const int64_t* off;
  const int4* list;        // (s1 index, s2 index, S | T_rest << 16, ie << 16 | je), ie and je 1-based
  const int* count;
  uint32_t* win;           // per list entry kRegWinWords threshold-code words (swg_box_reg.cuh)
  int* cls[2];             // band classes 0..3 (width <= 8, 16, 24, 32): list indices, classes 0 / 2
                           // from the front of cls[0] / cls[1], classes 1 / 3 from the back
  int* cls_count;          // [4]
  // query mode (serving): s1 = query slot q of qseq / qoff (raw residue bytes), the tables have a
  // row per residue byte (qsc: S; qscf: S << 8 | counted flag, kRegPadScore in the pad column),
  // distances go to qout[q][d]
  const uint8_t* qseq;
  const int64_t* qoff;
  int16_t* const* qout;
  const int* qsc;
  const int* qscf;
  int16_t* out;
  long long ld;
  int mirror;
  const int32_t* lettab;   // device [(A+1)^2] S(a, b) + o of the dense codes
  const uint32_t* flagtab; // device [(A+1)^2] counted-column flags
  int A;
  int o, e;
  int maxlen;
  long long budget;        // cells of the reverse scan and of the box before giving up
  int2* rerun;             // pairs given up on: the 32-bit full DP
  int* rerun_count;
  int rerun_cap;
  unsigned long long* stats;  // [1] pairs finished in 16-bit lanes, [3] pairs given up on,
                              // [4] pairs handed to the warp box kernel
  long long list_cap;      // entries `list` holds (the count is clipped to it)
  int max_score;           // box_kernel: pairs with a larger S cannot fit: straight to the 32-bit lanes
  int4* spill;             // box_scan_kernel: pairs for the warp box kernel
  int* spill_count;
  int spill_cap;
  int2* fb;                // pairs given up on, for the 16-bit counter kernel (nullptr: the 32-bit lanes)
  int* fb_count;
  long long fb_cap;
};

constexpr int kWarpBoxMaxCols = 256;  // box_kernel's largest box (columns and rows)

// One pair per thread, DP rows in registers (swg_box_reg.cuh): the reverse scan sorts the pairs
// into the band classes or hands them to J.spill; the band DP of class c writes distances and
// hands the rest to the 32-bit lanes.
cudaError_t launch_box_scan(const BoxJob& J, int sms, cudaStream_t st);
cudaError_t launch_box_band(const BoxJob& J, int c, int sms, cudaStream_t st);
// Warp per pair (reverse scan on 64-column shuffle windows, box DP as a 32-row wavefront).
cudaError_t launch_box(const BoxJob& J, int grid, int block, cudaStream_t st);

// Alignment strings of a list of pairs (swg_trace.cu): one thread per pair, a decision byte per
// DP cell in dirs (dir_stride bytes per pair), two int rows of row_stride / 2 ints in vrow.
struct TraceResult {
  int score, valid, end1, end2, start1, start2;
  int identity, similarity, gaps, length, diag, transitions, transversions;
};

struct TraceJob {
  const uint8_t* seq;      // residues (the context's), offsets as uploaded
  const int64_t* off;
  const int32_t* rows;     // s1 index of pair k
  const int32_t* cols;     // s2 index of pair k
  long long npairs;
  const int16_t* scores;   // [128 * 128]
  int o, e;
  uint8_t* dirs;
  long long dir_stride;
  int* vrow;
  long row_stride;
  char* aln1;              // aligned strings of pair k at aln1 + out_off[k] (and aln2)
  char* aln2;
  const int64_t* out_off;
  TraceResult* out;
};

size_t trace_scratch_bytes(int m, int n);
cudaError_t launch_traceback(const TraceJob& J, bool local, cudaStream_t st);

size_t plain_carry_bytes(int mode, long threads, int maxlen, int dist_fn = 0);
cudaError_t launch_plain_block(const PlainJob& J, int grid, int block, cudaStream_t st);
size_t pair_carry_bytes(int n);
cudaError_t launch_align_pair(const PairJob& J, cudaStream_t st);
cudaError_t measure_int_peak(double* max_ops, double* add_ops);

}  // namespace swg
