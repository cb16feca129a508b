// Whole-job engine: every pair of an all-pairs job, scheduled by persistent kernels.
//
// Work decomposition.  A work item is (query q, a chunk of the database ordered by length).
// The query is the DP's s1 (rows) and every chunk entry d that the job orients as (s1 = q,
// s2 = d) is aligned against it: SWG-MPI/NW reproduce the block driver's orientation for a
// given MPI world size (MPIComputeLowerTriangularBlocked.Compute, Salsa.SmithWatermanMPI/
// Program.cs:618-642: diagonal blocks align (s_i, s_j) for j < i, off-diagonal block (r, c) is
// aligned by rank r when r > c with r+c even or r < c with r+c odd), SWG-MS aligns every
// ordered pair (Salsa.SmithWatermanMS/Program.cs:341-375).  Items are binned by the query's
// rows-per-lane K and sorted longest first; one persistent kernel per bin pops items from a
// device counter.  The per-bin launches are captured in a CUDA graph and replayed.
//
// Kernel.  A CTA stages the query profile in shared memory; each warp aligns the query against
// two database sequences at once, one per 16-bit half of every score register (lane A = low
// half, lane B = high half).  Lane t of the warp owns K consecutive query rows; the DP sweeps
// the database columns as a wavefront, row-block t working on column s - t at step s and
// receiving the state of the row above it from lane t-1 by shuffle.  Queries longer than 32*K
// rows take several passes, the last row of a pass reaching the next through per-warp scratch.
//
// Score lanes hold value + bias in [0, 32767]: 32-bit integer adds never carry between the
// halves and the signed 16x2 max instructions see the true order.  A pair is given to these
// lanes only when max(score) * (min(m, n) + 1) + bias <= 32767 (static guard); a lane whose
// best score still reaches the trip threshold is rerun with 32-bit lanes.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../../include/swgb200.h"
#include "swg_box_reg.cuh"
#include "swg_device.cuh"
#include "swg_engine.h"
#include "swg_internal.h"

namespace swg {

// Warps per CTA and CTAs per SM for K rows per lane, from the registers a lane needs (65,536 per
// SM): up to 8 rows fit 128 registers (2 CTAs of 8 warps), 10-12 rows fit 168 (1 CTA of 12
// warps), 14-16 rows need up to 255 (1 CTA of 8 warps).  Measured on B200, 12 warps run the
// 10- and 12-row kernels 16% faster than 8.
// NW carries twice the counter words and spills a little at these register caps; measured on
// B200, the occupancy still pays more than the spills cost (8 warps with no spill: -9 %).
// The score-only first pass keeps 5 registers per row: up to 10 rows fit 128 registers (2 CTAs
// of 8 warps), 12-16 rows fit 168 (1 CTA of 12 warps).
constexpr int kMaxWarps = 12;
constexpr int kKindScoreShape = 2;  // the kind value of the score-only kernels (see kKindScore)
constexpr int kKindKimShape = 3;    // the kind value of the Kimura2 / JukesCantor kernels (kKindKim)
// The Kimura2 / JukesCantor kernels keep 15 registers per row (two counter words per state and
// lane): at most 8 rows per lane, one CTA of 8 warps per SM (two at 4 rows).
__host__ __device__ constexpr int warps_of(int K, int kind = 0) {
  return kind == kKindScoreShape ? (K <= 10 ? 8 : 12) : kind == kKindKimShape ? 8 : (K <= 8 ? 8 : K <= 12 ? 12 : 8);
}
__host__ __device__ constexpr int ctas_of(int K, int kind = 0) {
  return kind == kKindScoreShape ? (K <= 10 ? 2 : 1) : kind == kKindKimShape ? (K <= 4 ? 2 : 1) : (K <= 8 ? 2 : 1);
}
constexpr int kKimMaxK = 8;  // rows per lane of the Kimura2 / JukesCantor kernels
constexpr int kMaxChunk = 1024;
constexpr int kFbChunk = 64;     // third-pass partners per work item, at most
constexpr int kFbChunkMin = 2;   // ... and at least (one warp's two lanes A / B)
constexpr int kScrWords = 8;    // words of carried state per column in the pass scratch
constexpr int kScrWordsKim = 12;  // Kimura2 / JukesCantor: V, G and two counter words per state and lane

struct EngineJob {
  const uint8_t* code;      // dense residue codes (pad code = A), same offsets as the residues
  const int64_t* off;
  const int32_t* sorted;    // sequence indices by length
  const int4* items;        // (query, chunk begin, chunk end, passes)
  int nitems;
  int* counter;             // next item of this launch
  const int32_t* lettab;    // [(A+1)*(A+1)] S(a, b) + o; pad row/column -bias + o
  const uint32_t* flagtab;  // [(A+1)*(A+1)] counted-column flags
  int A, o, e, bias, thresh;
  int mode, ranks, nseq, rb_a, rb_b;
  int blk_mode, col_lo, col_hi;  // one block of the pair matrix: 1 diagonal, 2 off-diagonal (0: a job)
  int16_t* out;
  long long ld;
  int mirror;               // also write (d, q): symmetric jobs and diagonal blocks, never other blocks
  uint32_t* scratch;        // per (CTA, warp) slot: maxcol * kScrWords words
  int maxcol;               // longest database sequence
  int2* rerun;              // pairs to redo with 32-bit lanes
  int* rerun_count;
  int rerun_cap;
  int mpad;                 // profile rows staged (passes * 32 * K of the bin)
  long long scratch_words;  // pass scratch from `scratch` on, and rows' bounds from `rowbuf` on
  long long rowbuf_words;   // (the kernel checks its slots against them)
  int protein;              // NW distance rule: similarity over the full length
  int dist_fn;              // Kimura2 / JukesCantor kernels: SW_DIST_KIMURA2 or SW_DIST_JUKES_CANTOR
  int* throws;              // set by a SWG-MPI JukesCantor pair whose log argument is <= 0
  unsigned long long* stats; // [0] items taken, [1] pairs finished in 16-bit lanes, [2] tripped
  // third pass (fb_cnt != nullptr): the box step's give-ups bucketed by query, query k (k < fb_nq)
  // holding fb_cnt[k] partners at sorted[fb_start[k] ..] in chunks of fb_total[1] partners; item
  // it is chunk it - fb_cstart[k] of the query k with fb_cstart[k] <= it < fb_cstart[k + 1],
  // fb_total[0] items
  const int* fb_cnt;
  const int* fb_start;
  const int* fb_cstart;
  const int* fb_total;
  int fb_nq, fb_lo;
  int4* box;                // two-pass: pairs whose counters the box step finds
  uint32_t* boxwin;         // two-pass: per box record, the threshold codes of the 128 rows above ie
  int* box_count;
  int box_cap;
  uint32_t* rowbuf;         // two-pass: per (CTA, warp) slot, mpad words: each row's best V (lanes A | B)
  // Query mode (serving): s1 is query slot q of a separate set, s2 every database entry of the
  // chunk, the distance goes to qout[q][d].  Raw residue bytes index qtab/qflag (row 127 = pad).
  int qmode;
  const uint8_t* qseq;
  const int64_t* qoff;
  const int32_t* qlen;
  int16_t* const* qout;
  const int32_t* qtab;      // [128 * (A+1)] S(x, letter c) + o; pad row/column -bias + o
  const uint32_t* qflag;    // [128 * (A+1)]
};

// Rank owning a global row index under RangePartitioner (Program.cs:791-802).
__device__ __forceinline__ int block_of(int x, int a, int b) {
  return x < b * (a + 1) ? x / (a + 1) : b + (x - b * (a + 1)) / a;
}

__device__ __forceinline__ bool oriented(const EngineJob& J, int q, int d) {
  if (J.qmode) return true;
  if (J.blk_mode)  // the block's columns; a diagonal block of SWG-MPI / NW only below its diagonal
    return d >= J.col_lo && d <= J.col_hi && (J.blk_mode == 2 || J.mode == kModeSwgMs || d < q);
  if (J.mode == kModeSwgMs) return true;
  if (q == d) return false;
  const int bq = block_of(q, J.rb_a, J.rb_b), bd = block_of(d, J.rb_a, J.rb_b);
  if (bq == bd) return q > d;
  const bool odd = ((bq + bd) & 1) != 0;
  return (bq > bd && !odd) || (bq < bd && odd);
}

// Per-halfword signed max of a and b, with hi/lo = (a >= b) for the high/low halves, i.e. "the
// max of that half is a's".  The result register is early-clobbered: it must never share a
// register with a, or the comparison below would see the max in place of a and report "a won"
// for every half -- which happens exactly when the result overwrites a (BEST = max(BEST, V)).
__device__ __forceinline__ uint32_t vmax2(uint32_t a, uint32_t b, bool& hi, bool& lo) {
  uint32_t r, ph, pl;
  asm("{\n\t"
      ".reg .pred p0, p1;\n\t"
      ".reg .s16 m0, m1, a0, a1;\n\t"
      "max.s16x2 %0, %3, %4;\n\t"
      "mov.b32 {m0, m1}, %0;\n\t"
      "mov.b32 {a0, a1}, %3;\n\t"
      "setp.eq.s16 p0, m0, a0;\n\t"
      "setp.eq.s16 p1, m1, a1;\n\t"
      "selp.u32 %2, 1, 0, p0;\n\t"
      "selp.u32 %1, 1, 0, p1;\n\t"
      "}"
      : "=&r"(r), "=r"(ph), "=r"(pl)
      : "r"(a), "r"(b));
  hi = ph != 0u;
  lo = pl != 0u;
  return r;
}

// x * 65536 + y as one multiply-add (the FMA pipe has room; the ALU pipe is the bound).
__device__ __forceinline__ uint32_t mad_hi16(uint32_t x, uint32_t y) {
  uint32_t r;
  asm("mad.lo.u32 %0, %1, 65536, %2;" : "=r"(r) : "r"(x), "r"(y));
  return r;
}

// One warp, query rows in registers, two database sequences (lanes A/B) in lockstep.
// prof: shared-memory profile planes, plane(c, kind) at ((c*NP+kind) * mpad) words, rows stored
// per pass in lane-interleaved groups of 4 so each lane's 128-bit load hits distinct banks.
// NP = 3: score + o, (score + o) << 16, counted flag; NP = 2 (large alphabets, where three
// planes would not fit shared memory): score + o and flag, lane B's word shifted by a multiply-add.
// ca/cb: shared-memory code buffers with 32 pad entries before column 0.
template <int K, int NP>
__device__ __forceinline__ void align_two(const uint32_t* __restrict__ prof, int mpad, int passes,
                                          const uint8_t* __restrict__ ca,
                                          const uint8_t* __restrict__ cb, int ncols,
                                          const EngineJob& J, uint32_t* __restrict__ scr,
                                          int lane, int& bestA, int& rowA, uint32_t& cntA,
                                          int& bestB, int& rowB, uint32_t& cntB) {
  const uint32_t bias2 = (uint32_t)J.bias * 0x10001u;
  const uint32_t O2 = (uint32_t)J.o * 0x10001u, E2 = (uint32_t)J.e * 0x10001u;
  const uint32_t sent2 = (uint32_t)(J.bias - J.o - J.e) * 0x10001u;  // -infinity + bias
  const uint32_t best0 = (uint32_t)(J.bias - 1) * 0x10001u;          // below any V
  const uint32_t vo_top = (uint32_t)(J.bias - J.o) * 0x10001u;        // V(0,j) - o + bias
  const int plane = NP * mpad;
  bestA = bestB = -1;
  rowA = rowB = 0;
  cntA = cntB = 0u;
  for (int p = 0; p < passes; p++) {
    uint32_t VOL[K], H[K], BEST[K], clA[K], clB[K], chA[K], chB[K], bcA[K], bcB[K];
#pragma unroll
    for (int r = 0; r < K; r++) {
      VOL[r] = vo_top; H[r] = sent2; BEST[r] = best0;
      clA[r] = clB[r] = chA[r] = chB[r] = bcA[r] = bcB[r] = 0u;
    }
    // state received from the row block above (lane - 1), and its previous column
    uint32_t uVO = vo_top, uG = sent2, ucvA = 0, ucvB = 0, ucgA = 0, ucgB = 0;
    uint32_t dVO = vo_top, dcA = 0, dcB = 0;
    const int pbase = p * 32 * K;
    const uint32_t* pl = prof + pbase + lane * 4;
    const int nsteps = ncols + 31;
    // 14-16 rows per lane: the next column's residue codes are loaded one step ahead (the
    // 168-register kernels at 10-12 rows lose more to the extra registers than they gain)
    constexpr bool kPrefetch = K >= 14;
    int nxa = kPrefetch ? ca[32 - lane] : 0, nxb = kPrefetch ? cb[32 - lane] : 0;
    for (int s = 0; s < nsteps; s++) {
      // bottom row of this lane after the previous step, sent down one lane
      const uint32_t bVO = __shfl_up_sync(0xffffffffu, uVO, 1);
      const uint32_t bG = __shfl_up_sync(0xffffffffu, uG, 1);
      const uint32_t bcvA = __shfl_up_sync(0xffffffffu, ucvA, 1);
      const uint32_t bcvB = __shfl_up_sync(0xffffffffu, ucvB, 1);
      const uint32_t bcgA = __shfl_up_sync(0xffffffffu, ucgA, 1);
      const uint32_t bcgB = __shfl_up_sync(0xffffffffu, ucgB, 1);
      uint32_t VOU, GU, cvuA, cvuB, cguA, cguB;
      if (lane == 0) {
        if (p == 0 || s >= ncols) {
          VOU = vo_top; GU = sent2; cvuA = cvuB = cguA = cguB = 0u;
        } else {
          const uint4 x = *reinterpret_cast<const uint4*>(scr + (long)s * kScrWords);
          const uint2 y = *reinterpret_cast<const uint2*>(scr + (long)s * kScrWords + 4);
          VOU = x.x; GU = x.y; cvuA = x.z; cvuB = x.w; cguA = y.x; cguB = y.y;
        }
      } else {
        VOU = bVO; GU = bG; cvuA = bcvA; cvuB = bcvB; cguA = bcgA; cguB = bcgB;
      }
      // diagonal of the first row: the row above at the previous column
      uint32_t VOD = dVO, cdA = dcA, cdB = dcB;
      dVO = VOU; dcA = cvuA; dcB = cvuB;
      const int col = 32 + s - lane;  // index into the code buffers (pad before column 0)
      int xa, xb;
      if (kPrefetch) {
        xa = nxa; xb = nxb;
        nxa = ca[col + 1]; nxb = cb[col + 1];  // col + 1 <= ncols + 63: inside the pad
      } else {
        xa = ca[col]; xb = cb[col];
      }
      const uint32_t* pla = pl + xa * plane;
      const uint32_t* phb = pl + xb * plane + (NP == 3 ? mpad : 0);
      const uint32_t* pma = pl + xa * plane + (NP - 1) * mpad;
      const uint32_t* pmb = pl + xb * plane + (NP - 1) * mpad;
      // one row of the lane's block: the cell (row r, column col) of both pairs
      auto cell = [&](const int r, const uint32_t pl_r, const uint32_t ph_r, const uint32_t ma_r,
                      const uint32_t mb_r) {
        const uint32_t F = (NP == 3) ? VOD + pl_r + ph_r : mad_hi16(ph_r, VOD + pl_r);
        const uint32_t cfA = cdA + ma_r + 0x10000u;
        const uint32_t cfB = cdB + mb_r + 0x10000u;
        bool hiB, loA;
        // vertical gap: reopen from V above unless extending is strictly better
        const uint32_t G = vmax2(VOU, GU - E2, hiB, loA);
        const uint32_t cgA = (loA ? cvuA : cguA) + 0x10000u;
        const uint32_t cgB = (hiB ? cvuB : cguB) + 0x10000u;
        // horizontal gap
        H[r] = vmax2(VOL[r], H[r] - E2, hiB, loA);
        chA[r] = (loA ? clA[r] : chA[r]) + 0x10000u;
        chB[r] = (hiB ? clB[r] : chB[r]) + 0x10000u;
        // V = max(F, G, H, 0) with STOP > DIAGONAL > UP > LEFT on ties
        const uint32_t GHv = vmax2(G, H[r], hiB, loA);
        const uint32_t cghA = loA ? cgA : chA[r];
        const uint32_t cghB = hiB ? cgB : chB[r];
        const uint32_t FGH = vmax2(F, GHv, hiB, loA);
        const uint32_t cfgA = loA ? cfA : cghA;
        const uint32_t cfgB = hiB ? cfB : cghB;
        const uint32_t V = vmax2(bias2, FGH, hiB, loA);
        const uint32_t cvA = loA ? 0u : cfgA;
        const uint32_t cvB = hiB ? 0u : cfgB;
        // first strictly greater V of this row (columns ascend within a lane)
        BEST[r] = vmax2(BEST[r], V, hiB, loA);
        bcA[r] = loA ? bcA[r] : cvA;
        bcB[r] = hiB ? bcB[r] : cvB;
        const uint32_t VO = V - O2;
        VOD = VOL[r]; cdA = clA[r]; cdB = clB[r];
        VOL[r] = VO; clA[r] = cvA; clB[r] = cvB;
        VOU = VO; GU = G; cvuA = cvA; cvuB = cvB; cguA = cgA; cguB = cgB;
      };
#pragma unroll
      for (int g = 0; g < K / 4; g++) {
        const uint4 PL = *reinterpret_cast<const uint4*>(pla + g * 128);
        const uint4 PH = *reinterpret_cast<const uint4*>(phb + g * 128);
        const uint4 MA = *reinterpret_cast<const uint4*>(pma + g * 128);
        const uint4 MB = *reinterpret_cast<const uint4*>(pmb + g * 128);
        cell(g * 4 + 0, PL.x, PH.x, MA.x, MB.x);
        cell(g * 4 + 1, PL.y, PH.y, MA.y, MB.y);
        cell(g * 4 + 2, PL.z, PH.z, MA.z, MB.z);
        cell(g * 4 + 3, PL.w, PH.w, MA.w, MB.w);
      }
      if (K % 4 == 2) {
        // the last two rows of each lane sit after the groups of four, two words per lane
        const int t2 = (K / 4) * 128 - lane * 2;
        const uint2 PL = *reinterpret_cast<const uint2*>(pla + t2);
        const uint2 PH = *reinterpret_cast<const uint2*>(phb + t2);
        const uint2 MA = *reinterpret_cast<const uint2*>(pma + t2);
        const uint2 MB = *reinterpret_cast<const uint2*>(pmb + t2);
        cell(K - 2, PL.x, PH.x, MA.x, MB.x);
        cell(K - 1, PL.y, PH.y, MA.y, MB.y);
      }
      uVO = VOU; uG = GU; ucvA = cvuA; ucvB = cvuB; ucgA = cguA; ucgB = cguB;
      if (lane == 31 && p + 1 < passes) {
        const int j = s - 31;
        if (j >= 0 && j < ncols) {
          *reinterpret_cast<uint4*>(scr + (long)j * kScrWords) = make_uint4(uVO, uG, ucvA, ucvB);
          *reinterpret_cast<uint2*>(scr + (long)j * kScrWords + 4) = make_uint2(ucgA, ucgB);
        }
      }
    }
    __syncwarp();
    // rows ascend within a lane and across passes: keep the first strictly greater
#pragma unroll
    for (int r = 0; r < K; r++) {
      const int row = pbase + lane * K + r;
      const int sA = (int)(int16_t)(BEST[r] & 0xFFFFu) - J.bias;
      const int sB = (int)(int16_t)(BEST[r] >> 16) - J.bias;
      if (sA > bestA) { bestA = sA; rowA = row; cntA = bcA[r]; }
      if (sB > bestB) { bestB = sB; rowB = row; cntB = bcB[r]; }
    }
  }
}

// Kimura2 / JukesCantor counterpart of align_two (nucleic jobs whose letters fit three profile
// planes): each state and lane carries the two KimCnt words of Alignment.cs:254-348 -- aligned
// columns << 16 | A-flagged columns, non-gap columns << 16 | B-flagged columns -- and the flag
// plane holds the residue pair's A | B << 16 (transition / transversion, or identical / none).
// Gap steps add an aligned column; a diagonal step adds an aligned and a non-gap column and the
// pair's flags; STOP clears both words.  The best cell is tracked as in align_two.
template <int K>
__device__ __forceinline__ void align_two_kim(const uint32_t* __restrict__ prof, int mpad, int passes,
                                              const uint8_t* __restrict__ ca,
                                              const uint8_t* __restrict__ cb, int ncols,
                                              const EngineJob& J, uint32_t* __restrict__ scr,
                                              int lane, int& bestA, int& rowA, uint2& cntA,
                                              int& bestB, int& rowB, uint2& cntB) {
  const uint32_t bias2 = (uint32_t)J.bias * 0x10001u;
  const uint32_t O2 = (uint32_t)J.o * 0x10001u, E2 = (uint32_t)J.e * 0x10001u;
  const uint32_t sent2 = (uint32_t)(J.bias - J.o - J.e) * 0x10001u;  // -infinity + bias
  const uint32_t best0 = (uint32_t)(J.bias - 1) * 0x10001u;          // below any V
  const uint32_t vo_top = (uint32_t)(J.bias - J.o) * 0x10001u;        // V(0,j) - o + bias
  const int plane = 3 * mpad;
  bestA = bestB = -1;
  rowA = rowB = 0;
  cntA = cntB = make_uint2(0u, 0u);
  for (int p = 0; p < passes; p++) {
    uint32_t VOL[K], H[K], BEST[K];
    uint32_t clA0[K], clA1[K], clB0[K], clB1[K], chA0[K], chA1[K], chB0[K], chB1[K];
    uint32_t bcA0[K], bcA1[K], bcB0[K], bcB1[K];
#pragma unroll
    for (int r = 0; r < K; r++) {
      VOL[r] = vo_top; H[r] = sent2; BEST[r] = best0;
      clA0[r] = clA1[r] = clB0[r] = clB1[r] = 0u;
      chA0[r] = chA1[r] = chB0[r] = chB1[r] = 0u;
      bcA0[r] = bcA1[r] = bcB0[r] = bcB1[r] = 0u;
    }
    uint32_t uVO = vo_top, uG = sent2;
    uint32_t ucvA0 = 0, ucvA1 = 0, ucvB0 = 0, ucvB1 = 0, ucgA0 = 0, ucgA1 = 0, ucgB0 = 0, ucgB1 = 0;
    uint32_t dVO = vo_top, dcA0 = 0, dcA1 = 0, dcB0 = 0, dcB1 = 0;
    const int pbase = p * 32 * K;
    const uint32_t* pl = prof + pbase + lane * 4;
    const int nsteps = ncols + 31;
    for (int s = 0; s < nsteps; s++) {
      const uint32_t bVO = __shfl_up_sync(0xffffffffu, uVO, 1);
      const uint32_t bG = __shfl_up_sync(0xffffffffu, uG, 1);
      const uint32_t bcvA0 = __shfl_up_sync(0xffffffffu, ucvA0, 1);
      const uint32_t bcvA1 = __shfl_up_sync(0xffffffffu, ucvA1, 1);
      const uint32_t bcvB0 = __shfl_up_sync(0xffffffffu, ucvB0, 1);
      const uint32_t bcvB1 = __shfl_up_sync(0xffffffffu, ucvB1, 1);
      const uint32_t bcgA0 = __shfl_up_sync(0xffffffffu, ucgA0, 1);
      const uint32_t bcgA1 = __shfl_up_sync(0xffffffffu, ucgA1, 1);
      const uint32_t bcgB0 = __shfl_up_sync(0xffffffffu, ucgB0, 1);
      const uint32_t bcgB1 = __shfl_up_sync(0xffffffffu, ucgB1, 1);
      uint32_t VOU, GU, cvuA0, cvuA1, cvuB0, cvuB1, cguA0, cguA1, cguB0, cguB1;
      if (lane == 0) {
        if (p == 0 || s >= ncols) {
          VOU = vo_top; GU = sent2;
          cvuA0 = cvuA1 = cvuB0 = cvuB1 = cguA0 = cguA1 = cguB0 = cguB1 = 0u;
        } else {
          const uint4 x = *reinterpret_cast<const uint4*>(scr + (long)s * kScrWordsKim);
          const uint4 y = *reinterpret_cast<const uint4*>(scr + (long)s * kScrWordsKim + 4);
          const uint2 z = *reinterpret_cast<const uint2*>(scr + (long)s * kScrWordsKim + 8);
          VOU = x.x; GU = x.y; cvuA0 = x.z; cvuA1 = x.w;
          cvuB0 = y.x; cvuB1 = y.y; cguA0 = y.z; cguA1 = y.w;
          cguB0 = z.x; cguB1 = z.y;
        }
      } else {
        VOU = bVO; GU = bG; cvuA0 = bcvA0; cvuA1 = bcvA1; cvuB0 = bcvB0; cvuB1 = bcvB1;
        cguA0 = bcgA0; cguA1 = bcgA1; cguB0 = bcgB0; cguB1 = bcgB1;
      }
      uint32_t VOD = dVO, cdA0 = dcA0, cdA1 = dcA1, cdB0 = dcB0, cdB1 = dcB1;
      dVO = VOU; dcA0 = cvuA0; dcA1 = cvuA1; dcB0 = cvuB0; dcB1 = cvuB1;
      const int col = 32 + s - lane;
      const int xa = ca[col], xb = cb[col];
      const uint32_t* pla = pl + xa * plane;
      const uint32_t* phb = pl + xb * plane + mpad;
      const uint32_t* pma = pl + xa * plane + 2 * mpad;
      const uint32_t* pmb = pl + xb * plane + 2 * mpad;
      auto cell = [&](const int r, const uint32_t pl_r, const uint32_t ph_r, const uint32_t ma_r,
                      const uint32_t mb_r) {
        const uint32_t F = VOD + pl_r + ph_r;
        const uint32_t cfA0 = cdA0 + (ma_r & 0xFFFFu) + 0x10000u, cfA1 = cdA1 + (ma_r >> 16) + 0x10000u;
        const uint32_t cfB0 = cdB0 + (mb_r & 0xFFFFu) + 0x10000u, cfB1 = cdB1 + (mb_r >> 16) + 0x10000u;
        bool hiB, loA;
        // vertical gap: reopen from V above unless extending is strictly better
        const uint32_t G = vmax2(VOU, GU - E2, hiB, loA);
        const uint32_t cgA0 = (loA ? cvuA0 : cguA0) + 0x10000u, cgA1 = loA ? cvuA1 : cguA1;
        const uint32_t cgB0 = (hiB ? cvuB0 : cguB0) + 0x10000u, cgB1 = hiB ? cvuB1 : cguB1;
        // horizontal gap
        H[r] = vmax2(VOL[r], H[r] - E2, hiB, loA);
        chA0[r] = (loA ? clA0[r] : chA0[r]) + 0x10000u;
        chA1[r] = loA ? clA1[r] : chA1[r];
        chB0[r] = (hiB ? clB0[r] : chB0[r]) + 0x10000u;
        chB1[r] = hiB ? clB1[r] : chB1[r];
        // V = max(F, G, H, 0) with STOP > DIAGONAL > UP > LEFT on ties
        const uint32_t GHv = vmax2(G, H[r], hiB, loA);
        const uint32_t cghA0 = loA ? cgA0 : chA0[r], cghA1 = loA ? cgA1 : chA1[r];
        const uint32_t cghB0 = hiB ? cgB0 : chB0[r], cghB1 = hiB ? cgB1 : chB1[r];
        const uint32_t FGH = vmax2(F, GHv, hiB, loA);
        const uint32_t cfgA0 = loA ? cfA0 : cghA0, cfgA1 = loA ? cfA1 : cghA1;
        const uint32_t cfgB0 = hiB ? cfB0 : cghB0, cfgB1 = hiB ? cfB1 : cghB1;
        const uint32_t V = vmax2(bias2, FGH, hiB, loA);
        const uint32_t cvA0 = loA ? 0u : cfgA0, cvA1 = loA ? 0u : cfgA1;
        const uint32_t cvB0 = hiB ? 0u : cfgB0, cvB1 = hiB ? 0u : cfgB1;
        // first strictly greater V of this row (columns ascend within a lane)
        BEST[r] = vmax2(BEST[r], V, hiB, loA);
        bcA0[r] = loA ? bcA0[r] : cvA0;
        bcA1[r] = loA ? bcA1[r] : cvA1;
        bcB0[r] = hiB ? bcB0[r] : cvB0;
        bcB1[r] = hiB ? bcB1[r] : cvB1;
        const uint32_t VO = V - O2;
        VOD = VOL[r]; cdA0 = clA0[r]; cdA1 = clA1[r]; cdB0 = clB0[r]; cdB1 = clB1[r];
        VOL[r] = VO; clA0[r] = cvA0; clA1[r] = cvA1; clB0[r] = cvB0; clB1[r] = cvB1;
        VOU = VO; GU = G;
        cvuA0 = cvA0; cvuA1 = cvA1; cvuB0 = cvB0; cvuB1 = cvB1;
        cguA0 = cgA0; cguA1 = cgA1; cguB0 = cgB0; cguB1 = cgB1;
      };
#pragma unroll
      for (int g = 0; g < K / 4; g++) {
        const uint4 PL = *reinterpret_cast<const uint4*>(pla + g * 128);
        const uint4 PH = *reinterpret_cast<const uint4*>(phb + g * 128);
        const uint4 MA = *reinterpret_cast<const uint4*>(pma + g * 128);
        const uint4 MB = *reinterpret_cast<const uint4*>(pmb + g * 128);
        cell(g * 4 + 0, PL.x, PH.x, MA.x, MB.x);
        cell(g * 4 + 1, PL.y, PH.y, MA.y, MB.y);
        cell(g * 4 + 2, PL.z, PH.z, MA.z, MB.z);
        cell(g * 4 + 3, PL.w, PH.w, MA.w, MB.w);
      }
      if (K % 4 == 2) {
        const int t2 = (K / 4) * 128 - lane * 2;
        const uint2 PL = *reinterpret_cast<const uint2*>(pla + t2);
        const uint2 PH = *reinterpret_cast<const uint2*>(phb + t2);
        const uint2 MA = *reinterpret_cast<const uint2*>(pma + t2);
        const uint2 MB = *reinterpret_cast<const uint2*>(pmb + t2);
        cell(K - 2, PL.x, PH.x, MA.x, MB.x);
        cell(K - 1, PL.y, PH.y, MA.y, MB.y);
      }
      uVO = VOU; uG = GU;
      ucvA0 = cvuA0; ucvA1 = cvuA1; ucvB0 = cvuB0; ucvB1 = cvuB1;
      ucgA0 = cguA0; ucgA1 = cguA1; ucgB0 = cguB0; ucgB1 = cguB1;
      if (lane == 31 && p + 1 < passes) {
        const int j = s - 31;
        if (j >= 0 && j < ncols) {
          *reinterpret_cast<uint4*>(scr + (long)j * kScrWordsKim) = make_uint4(uVO, uG, ucvA0, ucvA1);
          *reinterpret_cast<uint4*>(scr + (long)j * kScrWordsKim + 4) = make_uint4(ucvB0, ucvB1, ucgA0, ucgA1);
          *reinterpret_cast<uint2*>(scr + (long)j * kScrWordsKim + 8) = make_uint2(ucgB0, ucgB1);
        }
      }
    }
    __syncwarp();
    // rows ascend within a lane and across passes: keep the first strictly greater
#pragma unroll
    for (int r = 0; r < K; r++) {
      const int row = pbase + lane * K + r;
      const int sA = (int)(int16_t)(BEST[r] & 0xFFFFu) - J.bias;
      const int sB = (int)(int16_t)(BEST[r] >> 16) - J.bias;
      if (sA > bestA) { bestA = sA; rowA = row; cntA = make_uint2(bcA0[r], bcA1[r]); }
      if (sB > bestB) { bestB = sB; rowB = row; cntB = make_uint2(bcB0[r], bcB1[r]); }
    }
  }
}

// Score-only counterpart of align_two (first pass of the two-pass SW path): the same DP without
// counters, keeping per query row the best V and the column where it was first reached.  Returns
// per lane half the best score and its cell (row and column, 0-based) in the reference's order
// (first strictly greater in row-major order), and stores each row's best V (value + bias, lanes
// A | B) at rowbuf[row]: the box step's bound of that row (padding columns can only raise it).
template <int K, int NP>
__device__ __forceinline__ void score_two(const uint32_t* __restrict__ prof, int mpad, int passes,
                                          const uint8_t* __restrict__ ca,
                                          const uint8_t* __restrict__ cb, int ncols,
                                          const EngineJob& J, uint32_t* __restrict__ scr,
                                          uint32_t* __restrict__ rowbuf,
                                          int lane, int& bestA, int& rowA, uint32_t& colA,
                                          int& bestB, int& rowB, uint32_t& colB) {
  const uint32_t bias2 = (uint32_t)J.bias * 0x10001u;
  const uint32_t O2 = (uint32_t)J.o * 0x10001u, E2 = (uint32_t)J.e * 0x10001u;
  const uint32_t sent2 = (uint32_t)(J.bias - J.o - J.e) * 0x10001u;  // -infinity + bias
  const uint32_t best0 = (uint32_t)(J.bias - 1) * 0x10001u;          // below any V
  const uint32_t vo_top = (uint32_t)(J.bias - J.o) * 0x10001u;        // V(0,j) - o + bias
  const int plane = NP * mpad;
  bestA = bestB = -1;
  rowA = rowB = 0;
  colA = colB = 0u;
  for (int p = 0; p < passes; p++) {
    uint32_t VOL[K], H[K], BEST[K], bcA[K], bcB[K];
#pragma unroll
    for (int r = 0; r < K; r++) {
      VOL[r] = vo_top; H[r] = sent2; BEST[r] = best0;
      bcA[r] = bcB[r] = 0u;
    }
    uint32_t uVO = vo_top, uG = sent2, dVO = vo_top;
    const int pbase = p * 32 * K;
    const uint32_t* pl = prof + pbase + lane * 4;
    const int nsteps = ncols + 31;
    for (int s = 0; s < nsteps; s++) {
      const uint32_t bVO = __shfl_up_sync(0xffffffffu, uVO, 1);
      const uint32_t bG = __shfl_up_sync(0xffffffffu, uG, 1);
      uint32_t VOU, GU;
      if (lane == 0) {
        if (p == 0 || s >= ncols) {
          VOU = vo_top; GU = sent2;
        } else {
          const uint2 x = *reinterpret_cast<const uint2*>(scr + (long)s * 2);
          VOU = x.x; GU = x.y;
        }
      } else {
        VOU = bVO; GU = bG;
      }
      uint32_t VOD = dVO;
      dVO = VOU;
      const int col = 32 + s - lane;
      const uint32_t colv = (uint32_t)(s - lane);  // this lane's column at this step
      const int xa = ca[col], xb = cb[col];
      const uint32_t* pla = pl + xa * plane;
      const uint32_t* phb = pl + xb * plane + (NP == 3 ? mpad : 0);
      auto cell = [&](const int r, const uint32_t pl_r, const uint32_t ph_r) {
        const uint32_t F = (NP == 3) ? VOD + pl_r + ph_r : mad_hi16(ph_r, VOD + pl_r);
        // G and H floored at 0 (bias), so that V = max(F, G, H) needs no floor of its own (one
        // max fewer per cell pair).  By induction a floored G' is max(G, 0) of the unfloored G:
        // max(VO, max(G, 0) - e, 0) = max(VO, G - e, -e, 0) = max(G_next, 0), and likewise H'; so
        // max(F, G', H') = max(F, G, H, 0) and every V -- hence every row's best and its first
        // column -- is unchanged.  This pass keeps no pointers: G and H are not needed otherwise.
        const uint32_t G = __vimax3_s16x2(VOU, GU - E2, bias2);
        H[r] = __vimax3_s16x2(VOL[r], H[r] - E2, bias2);
        const uint32_t V = __vimax3_s16x2(F, G, H[r]);
        bool hiB, loA;
        BEST[r] = vmax2(BEST[r], V, hiB, loA);  // kept unless V is strictly greater
        bcA[r] = loA ? bcA[r] : colv;
        bcB[r] = hiB ? bcB[r] : colv;
        const uint32_t VO = V - O2;
        VOD = VOL[r];
        VOL[r] = VO;
        VOU = VO;
        GU = G;
      };
#pragma unroll
      for (int g = 0; g < K / 4; g++) {
        const uint4 PL = *reinterpret_cast<const uint4*>(pla + g * 128);
        const uint4 PH = *reinterpret_cast<const uint4*>(phb + g * 128);
        cell(g * 4 + 0, PL.x, PH.x);
        cell(g * 4 + 1, PL.y, PH.y);
        cell(g * 4 + 2, PL.z, PH.z);
        cell(g * 4 + 3, PL.w, PH.w);
      }
      if (K % 4 == 2) {
        const int t2 = (K / 4) * 128 - lane * 2;
        const uint2 PL = *reinterpret_cast<const uint2*>(pla + t2);
        const uint2 PH = *reinterpret_cast<const uint2*>(phb + t2);
        cell(K - 2, PL.x, PH.x);
        cell(K - 1, PL.y, PH.y);
      }
      uVO = VOU;
      uG = GU;
      if (lane == 31 && p + 1 < passes) {
        const int j = s - 31;
        if (j >= 0 && j < ncols) *reinterpret_cast<uint2*>(scr + (long)j * 2) = make_uint2(uVO, uG);
      }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < K; r += 2)
      *reinterpret_cast<uint2*>(rowbuf + pbase + lane * K + r) = make_uint2(BEST[r], BEST[r + 1]);
#pragma unroll
    for (int r = 0; r < K; r++) {
      const int row = pbase + lane * K + r;
      const int sA = (int)(int16_t)(BEST[r] & 0xFFFFu) - J.bias;
      const int sB = (int)(int16_t)(BEST[r] >> 16) - J.bias;
      if (sA > bestA) { bestA = sA; rowA = row; colA = bcA[r]; }
      if (sB > bestB) { bestB = sB; rowB = row; colB = bcB[r]; }
    }
  }
}

// NW (global) counterpart of align_two: V = max(F, G, H) without the 0 floor, boundaries
// V(i,0) = -o-(i-1)e and V(0,j) = -o-(j-1)e reached through the gap chains, the result taken at
// (m, n) of each pair.  Lanes hold value + bias with a bias that covers the all-gap lower bound of
// every cell a pass touches (padding rows and columns score 0, so they stay inside the same
// bounds); lanes start at their own column 0, so steps before it change nothing.
//
// One counter word per state and lane: columns << 16 | counted columns.  The trimmed identity of
// nucleic jobs (Salsa.NeedlemanWunschTPL/Program.cs:547-571) divides by the columns between the
// first and the last column with no gap in either string: the alignment less its leading gap run
// and its trailing gap run.  A global path from (0, 0) to (m, n) leaves column 0 (or row 0) for
// good at its first non-UP (non-LEFT) step, so its leading run is exactly its steps on column 0
// or row 0; once on column n (row m) it can only go UP (LEFT), so its trailing run is exactly its
// UP steps within column n or LEFT steps within row m.  Nucleic jobs therefore count no column on
// the boundary (V(i, 0), V(0, j) carry 0), and the UP / LEFT steps into a cell of column n / row m
// add no column (ginc / hinc 0 there); every other step adds one.  Protein jobs divide by the
// whole alignment: every step counts and the boundaries carry i / j columns.
template <int K, int NP>
__device__ __forceinline__ void align_two_nw(const uint32_t* __restrict__ prof, int mpad, int passes,
                                             int m, const uint8_t* __restrict__ ca,
                                             const uint8_t* __restrict__ cb, int ncols, int nA, int nB,
                                             const EngineJob& J, uint32_t* __restrict__ scr, int lane,
                                             uint32_t& capA, uint32_t& capB) {
  const int B = J.bias, o = J.o, e = J.e;
  const uint32_t O2 = (uint32_t)o * 0x10001u, E2 = (uint32_t)e * 0x10001u;
  const uint32_t sent2 = (uint32_t)e * 0x10001u;  // -infinity: loses to any opening, minus e is 0
  const bool trim = !J.protein;
  const uint32_t bmul = trim ? 0u : 0x10000u;     // boundary columns counted (protein) or not
  const int plane = NP * mpad;
  // the cell (m, n) of each pair: its pass, lane, row in the lane, and the step that reaches it
  const int pm = (m - 1) / (32 * K), tm = ((m - 1) % (32 * K)) / K, rm = (m - 1) % K;
  const int sA = nA - 1 + tm, sB = nB - 1 + tm;
  // the step at which this lane is at column n of pair A / B (-1: never counts as trailing)
  const int gsA = trim ? nA - 1 + lane : -1, gsB = trim ? nB - 1 + lane : -1;
  capA = capB = 0u;
  for (int p = 0; p < passes; p++) {
    const int pbase = p * 32 * K;
    // the steps at which this lane holds (m, n) of pair A / B in this pass (-1: none)
    const bool holder = p == pm && lane == tm;
    const int cA = holder ? sA : -1, cB = holder ? sB : -1;
    uint32_t VOL[K], H[K], clA[K], clB[K], chA[K], chB[K], hinc[K];
#pragma unroll
    for (int r = 0; r < K; r++) {
      const int i = pbase + lane * K + r + 1;  // V(i, 0) = -o - (i-1)e after i UP steps
      VOL[r] = (uint32_t)(B - 2 * o - (i - 1) * e) * 0x10001u;
      H[r] = sent2;
      clA[r] = clB[r] = (uint32_t)i * bmul;
      chA[r] = chB[r] = 0u;
      hinc[r] = (trim && i == m) ? 0u : 0x10000u;  // LEFT steps within row m: the trailing run
    }
    // the row above the lane's first row, at column 0 (the first step's diagonal)
    const int i0 = pbase + lane * K;
    uint32_t dVO = (uint32_t)(i0 == 0 ? B - o : B - 2 * o - (i0 - 1) * e) * 0x10001u;
    uint32_t dcA = (uint32_t)i0 * bmul, dcB = dcA;
    uint32_t uVO = 0, uG = 0, ucvA = 0, ucvB = 0, ucgA = 0, ucgB = 0;
    const uint32_t* pl = prof + pbase + lane * 4;
    const int nsteps = ncols + 31;
    for (int s = 0; s < nsteps; s++) {
      const uint32_t bVO = __shfl_up_sync(0xffffffffu, uVO, 1);
      const uint32_t bG = __shfl_up_sync(0xffffffffu, uG, 1);
      const uint32_t bcvA = __shfl_up_sync(0xffffffffu, ucvA, 1);
      const uint32_t bcvB = __shfl_up_sync(0xffffffffu, ucvB, 1);
      const uint32_t bcgA = __shfl_up_sync(0xffffffffu, ucgA, 1);
      const uint32_t bcgB = __shfl_up_sync(0xffffffffu, ucgB, 1);
      if (s >= lane) {  // the lane's columns start at step `lane`
        uint32_t VOU, GU, cvuA, cvuB, cguA, cguB;
        if (lane == 0) {
          if (p == 0) {
            // row 0: V(0, j) = -o - (j-1)e for column j = s + 1 (past the end: clamped)
            const int j = min(s, ncols - 1) + 1;
            VOU = (uint32_t)(B - 2 * o - (j - 1) * e) * 0x10001u;
            GU = sent2;
            cvuA = cvuB = (uint32_t)j * bmul;
            cguA = cguB = 0u;
          } else {
            const int js = min(s, ncols - 1);
            const uint4 x = *reinterpret_cast<const uint4*>(scr + (long)js * kScrWords);
            const uint2 y = *reinterpret_cast<const uint2*>(scr + (long)js * kScrWords + 4);
            VOU = x.x; GU = x.y; cvuA = x.z; cvuB = x.w; cguA = y.x; cguB = y.y;
          }
        } else {
          VOU = bVO; GU = bG; cvuA = bcvA; cvuB = bcvB; cguA = bcgA; cguB = bcgB;
        }
        uint32_t VOD = dVO, cdA = dcA, cdB = dcB;
        dVO = VOU; dcA = cvuA; dcB = cvuB;
        const int jc = s - lane;  // this step's column (0-based)
        // UP steps within column n: the trailing run
        const uint32_t gincA = s == gsA ? 0u : 0x10000u;
        const uint32_t gincB = s == gsB ? 0u : 0x10000u;
        const int col = 32 + jc;
        const int xa = ca[col], xb = cb[col];
        const uint32_t* pla = pl + xa * plane;
        const uint32_t* phb = pl + xb * plane + (NP == 3 ? mpad : 0);
        const uint32_t* pma = pl + xa * plane + (NP - 1) * mpad;
        const uint32_t* pmb = pl + xb * plane + (NP - 1) * mpad;
        auto cell = [&](const int r, const uint32_t pl_r, const uint32_t ph_r, const uint32_t ma_r,
                        const uint32_t mb_r) {
          const uint32_t F = (NP == 3) ? VOD + pl_r + ph_r : mad_hi16(ph_r, VOD + pl_r);
          const uint32_t cfA = cdA + ma_r + 0x10000u;
          const uint32_t cfB = cdB + mb_r + 0x10000u;
          bool hiB, loA;
          // vertical gap: opening wins ties (extend only if strictly better)
          const uint32_t G = vmax2(VOU, GU - E2, hiB, loA);
          const uint32_t cgA = (loA ? cvuA : cguA) + gincA;
          const uint32_t cgB = (hiB ? cvuB : cguB) + gincB;
          // horizontal gap
          H[r] = vmax2(VOL[r], H[r] - E2, hiB, loA);
          chA[r] = (loA ? clA[r] : chA[r]) + hinc[r];
          chB[r] = (hiB ? clB[r] : chB[r]) + hinc[r];
          // V = max(F, G, H) with DIAGONAL > UP > LEFT on ties
          const uint32_t GHv = vmax2(G, H[r], hiB, loA);
          const uint32_t cghA = loA ? cgA : chA[r];
          const uint32_t cghB = hiB ? cgB : chB[r];
          const uint32_t V = vmax2(F, GHv, hiB, loA);
          const uint32_t cvA = loA ? cfA : cghA;
          const uint32_t cvB = hiB ? cfB : cghB;
          const uint32_t VO = V - O2;
          VOD = VOL[r]; cdA = clA[r]; cdB = clB[r];
          VOL[r] = VO; clA[r] = cvA; clB[r] = cvB;
          VOU = VO; GU = G; cvuA = cvA; cvuB = cvB; cguA = cgA; cguB = cgB;
        };
#pragma unroll
        for (int g = 0; g < K / 4; g++) {
          const uint4 PL = *reinterpret_cast<const uint4*>(pla + g * 128);
          const uint4 PH = *reinterpret_cast<const uint4*>(phb + g * 128);
          const uint4 MA = *reinterpret_cast<const uint4*>(pma + g * 128);
          const uint4 MB = *reinterpret_cast<const uint4*>(pmb + g * 128);
          cell(g * 4 + 0, PL.x, PH.x, MA.x, MB.x);
          cell(g * 4 + 1, PL.y, PH.y, MA.y, MB.y);
          cell(g * 4 + 2, PL.z, PH.z, MA.z, MB.z);
          cell(g * 4 + 3, PL.w, PH.w, MA.w, MB.w);
        }
        if (K % 4 == 2) {
          const int t2 = (K / 4) * 128 - lane * 2;
          const uint2 PL = *reinterpret_cast<const uint2*>(pla + t2);
          const uint2 PH = *reinterpret_cast<const uint2*>(phb + t2);
          const uint2 MA = *reinterpret_cast<const uint2*>(pma + t2);
          const uint2 MB = *reinterpret_cast<const uint2*>(pmb + t2);
          cell(K - 2, PL.x, PH.x, MA.x, MB.x);
          cell(K - 1, PL.y, PH.y, MA.y, MB.y);
        }
        uVO = VOU; uG = GU; ucvA = cvuA; ucvB = cvuB; ucgA = cguA; ucgB = cguB;
        // the (m, n) cells: lane tm of pass pm holds them after steps sA / sB
        if (s == cA || s == cB) {
#pragma unroll
          for (int r = 0; r < K; r++)
            if (r == rm) {
              if (s == cA) capA = clA[r];
              if (s == cB) capB = clB[r];
            }
        }
        if (lane == 31 && p + 1 < passes) {
          const int j = s - 31;
          if (j >= 0 && j < ncols) {
            *reinterpret_cast<uint4*>(scr + (long)j * kScrWords) = make_uint4(uVO, uG, ucvA, ucvB);
            *reinterpret_cast<uint2*>(scr + (long)j * kScrWords + 4) = make_uint2(ucgA, ucgB);
          }
        }
      }
    }
    __syncwarp();
  }
  // the holder of (m, n) is lane tm: everyone gets its counters
  capA = __shfl_sync(0xffffffffu, capA, tm);
  capB = __shfl_sync(0xffffffffu, capB, tm);
}

// NW distance (Salsa.NeedlemanWunschTPL/Program.cs:547-571, :583-604) from the counter word of
// (m, n): counted columns over the trimmed (nucleic) or whole (protein) alignment.
__device__ __forceinline__ int16_t engine_nw_distance(uint32_t w) {
  return fraction_distance((int)(w & 0xFFFFu), (int)(w >> 16));
}

// Counter word of a pair with an empty side: all of it one gap run along the boundary (nucleic:
// all of it trimmed away).
__device__ __forceinline__ uint32_t nw_boundary(int m, int n, int protein) {
  return protein ? (uint32_t)(m + n) << 16 : 0u;
}

// Lexicographic (max score, min row) over the warp; lane 0 ends with the winner.
__device__ __forceinline__ void warp_best(int& best, int& row, uint32_t& cnt) {
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) {
    const int ob = __shfl_down_sync(0xffffffffu, best, d);
    const int orow = __shfl_down_sync(0xffffffffu, row, d);
    const uint32_t oc = __shfl_down_sync(0xffffffffu, cnt, d);
    if (ob > best || (ob == best && orow < row)) { best = ob; row = orow; cnt = oc; }
  }
}

// warp_best with the two KimCnt words.
__device__ __forceinline__ void warp_best2(int& best, int& row, uint2& cnt) {
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) {
    const int ob = __shfl_down_sync(0xffffffffu, best, d);
    const int orow = __shfl_down_sync(0xffffffffu, row, d);
    const uint32_t ox = __shfl_down_sync(0xffffffffu, cnt.x, d);
    const uint32_t oy = __shfl_down_sync(0xffffffffu, cnt.y, d);
    if (ob > best || (ob == best && orow < row)) { best = ob; row = orow; cnt = make_uint2(ox, oy); }
  }
}

__device__ __forceinline__ void emit(const EngineJob& J, int q, int d, int16_t dist) {
  if (J.qmode) {
    J.qout[q][d] = dist;
    return;
  }
  J.out[(long long)q * J.ld + d] = dist;
  if (J.mirror) J.out[(long long)d * J.ld + q] = dist;
}

// The first self-check violation of a launch: stats[7] = site << 48 | index (0: none).
__device__ __forceinline__ void record_error(const EngineJob& J, int site, int index) {
  atomicCAS(J.stats + 7, 0ull, ((unsigned long long)site << 48) | (unsigned long long)(unsigned)index);
}

// What a kernel instantiation computes per pair.
enum { kKindSw = 0, kKindNw = 1, kKindScore = 2, kKindKim = 3 };

template <int K, int NP, int KIND>
__global__ void __launch_bounds__(warps_of(K, KIND) * 32, ctas_of(K, KIND)) engine_kernel(EngineJob J) {
  static_assert(kKindScore == kKindScoreShape && kKindKim == kKindKimShape, "kernel kinds");
  constexpr bool NW = KIND == kKindNw;
  constexpr int kEngWarps = warps_of(K, KIND);
  constexpr int kScr = KIND == kKindKim ? kScrWordsKim : kScrWords;
  extern __shared__ __align__(16) uint8_t smem[];
  uint32_t* prof = reinterpret_cast<uint32_t*>(smem);
  const int A1 = J.A + 1;
  int* list = reinterpret_cast<int*>(smem + (size_t)A1 * NP * J.mpad * 4);
  uint8_t* codes = reinterpret_cast<uint8_t*>(list + kMaxChunk);
  const int cbuf = 64 + ((J.maxcol + 31) / 32) * 32;
  __shared__ int s_item, s_count, s_next, s_q;
  __shared__ int s_wc[kMaxWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* ca = codes + (size_t)warp * 2 * cbuf;
  uint8_t* cb = ca + cbuf;
  uint32_t* scr = J.scratch + ((long)blockIdx.x * kEngWarps + warp) * (long)J.maxcol * kScr;
  uint32_t* rowb = J.rowbuf ? J.rowbuf + ((long)blockIdx.x * kEngWarps + warp) * (long)J.mpad : nullptr;
  if (threadIdx.x == 0) s_q = -1;
  const int nitems = J.fb_cnt ? *J.fb_total : J.nitems;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(J.counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= nitems) break;
    int q, c0, c1, passes;
    if (J.fb_cnt) {  // third pass: a chunk of a query's pairs the box step gave up on
      int lo = 0, hi = J.fb_nq;  // fb_cstart[lo] <= it < fb_cstart[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (J.fb_cstart[mid] <= it) lo = mid;
        else hi = mid;
      }
      q = J.fb_lo + lo;
      const int chunk = J.fb_total[1];
      c0 = J.fb_start[lo] + (it - J.fb_cstart[lo]) * chunk;
      c1 = min(J.fb_start[lo] + J.fb_cnt[lo], c0 + chunk);
      if (c1 == c0) {
        __syncthreads();  // every thread has read s_item
        continue;
      }
      const int mq = J.qmode ? J.qlen[q] : (int)(J.off[q + 1] - J.off[q]);
      passes = max(1, (mq + 32 * K - 1) / (32 * K));
    } else {
      const int4 item = J.items[it];
      q = item.x; c0 = item.y; c1 = item.z; passes = item.w;
    }
    if (threadIdx.x == 0 && !J.fb_cnt) atomicAdd(J.stats, 1ull);  // planned items only
    const int mrows = passes * 32 * K;
    // self-checks (CTA-uniform): a work item outside the plan's bounds is recorded and skipped
    if ((!J.qmode && (q < 0 || q >= J.nseq)) || c1 < c0 || mrows > J.mpad ||
        (passes > 1 && ((long long)blockIdx.x + 1) * kEngWarps * J.maxcol * kScr > J.scratch_words) ||
        (rowb && ((long long)blockIdx.x + 1) * kEngWarps * J.mpad > J.rowbuf_words)) {
      if (threadIdx.x == 0) record_error(J, 1, it);
      continue;  // every thread has read s_item
    }
    const int m = J.qmode ? J.qlen[q] : (int)(J.off[q + 1] - J.off[q]);
    // query profile (rows beyond m and the pad column score -bias, count nothing)
    const bool rebuild = (q != s_q);
    __syncthreads();
    if (rebuild) {
      const uint8_t* qc = J.qmode ? J.qseq + J.qoff[q] : J.code + J.off[q];
      const int32_t* ptab = J.qmode ? J.qtab : J.lettab;
      const uint32_t* ftab = J.qmode ? J.qflag : J.flagtab;
      const int pad = J.qmode ? kPadCode : J.A;
      for (int idx = threadIdx.x; idx < A1 * mrows; idx += blockDim.x) {
        const int c = idx / mrows, i = idx - c * mrows;
        const int pp = i / (32 * K), rem = i - pp * 32 * K, t = rem / K, rr = rem - t * K;
        // rows in groups of four per lane (lane-interleaved), then a group of two when K % 4 == 2
        const int pos = pp * 32 * K + (rr < (K & ~3) ? ((rr >> 2) * 32 + t) * 4 + (rr & 3)
                                                     : (K & ~3) * 32 + t * 2 + (rr & 1));
        const int a = (i < m) ? (int)qc[i] : pad;
        const int v = ptab[a * A1 + c];
        uint32_t* pc = prof + (size_t)c * NP * J.mpad;
        pc[pos] = (uint32_t)v;
        if (NP == 3) pc[J.mpad + pos] = (uint32_t)v << 16;
        pc[(NP - 1) * J.mpad + pos] = ftab[a * A1 + c];
      }
    }
    if (threadIdx.x == 0) s_q = q;
    // segments of at most kMaxChunk entries (a chunk is one; a third-pass query may have more)
    for (int seg0 = c0; seg0 < c1; seg0 += kMaxChunk) {
    const int seg1 = min(c1, seg0 + kMaxChunk);
    if (threadIdx.x == 0) { s_count = 0; s_next = 0; }
    __syncthreads();
    // compact the chunk entries this query aligns, keeping the chunk's ascending-length order
    for (int base = seg0; base < seg1; base += blockDim.x) {
      const int k = base + threadIdx.x;
      const int d = (k < seg1) ? J.sorted[k] : -1;
      const bool ok = d >= 0 && (J.fb_cnt != nullptr || oriented(J, q, d));
      const unsigned bal = __ballot_sync(0xffffffffu, ok);
      if (lane == 0) s_wc[warp] = __popc(bal);
      __syncthreads();
      int before = s_count;
      for (int w = 0; w < warp; w++) before += s_wc[w];
      if (ok) list[before + __popc(bal & ((1u << lane) - 1u))] = d;
      __syncthreads();
      if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < kEngWarps; w++) tot += s_wc[w];
        s_count += tot;
      }
      __syncthreads();
    }
    const int cnt = s_count;
    for (;;) {
      int pi = 0;
      if (lane == 0) pi = atomicAdd(&s_next, 2);
      pi = __shfl_sync(0xffffffffu, pi, 0);
      if (pi >= cnt) break;
      const int dA = list[pi];
      const int dB = (pi + 1 < cnt) ? list[pi + 1] : -1;
      if (dA < 0 || dA >= J.nseq || dB >= J.nseq) {  // self-check (warp-uniform)
        if (lane == 0) record_error(J, 2, dA);
        continue;
      }
      const int nA = (int)(J.off[dA + 1] - J.off[dA]);
      const int nB = dB >= 0 ? (int)(J.off[dB + 1] - J.off[dB]) : 0;
      const int ncols = max(nA, nB);
      if (ncols > J.maxcol) {
        if (lane == 0) record_error(J, 3, dA);
        continue;
      }
      const uint8_t* sa = J.code + J.off[dA];
      const uint8_t* sb = dB >= 0 ? J.code + J.off[dB] : sa;
      for (int k = lane; k < 32 + ncols; k += 32) {
        const int j = k - 32;
        ca[k] = (j >= 0 && j < nA) ? sa[j] : (uint8_t)J.A;
        cb[k] = (j >= 0 && j < nB) ? sb[j] : (uint8_t)J.A;
      }
      for (int k = 32 + ncols + lane; k < 64 + ncols; k += 32) { ca[k] = (uint8_t)J.A; cb[k] = (uint8_t)J.A; }
      __syncwarp();
      if constexpr (KIND == kKindScore) {
        // first pass of the two-pass path: best score, its cell and the rows' bounds; the box step
        // finds the counters
        int bA = 0, rA = 0, bB = 0, rB = 0;
        uint32_t cA = 0, cB = 0;
        if (m > 0 && ncols > 0)
          score_two<K, NP>(prof, J.mpad, passes, ca, cb, ncols, J, scr, rowb, lane, bA, rA, cA, bB, rB, cB);
        warp_best(bA, rA, cA);
        warp_best(bB, rB, cB);
        bA = __shfl_sync(0xffffffffu, bA, 0);
        rA = __shfl_sync(0xffffffffu, rA, 0);
        cA = __shfl_sync(0xffffffffu, cA, 0);
        bB = __shfl_sync(0xffffffffu, bB, 0);
        rB = __shfl_sync(0xffffffffu, rB, 0);
        cB = __shfl_sync(0xffffffffu, cB, 0);
        const bool goA = m > 0 && nA > 0 && bA > 0 && bA <= J.thresh;
        const bool goB = dB >= 0 && m > 0 && nB > 0 && bB > 0 && bB <= J.thresh;
        int wA = 0, wB = 0;
        if (lane == 0) {
          unsigned long long done16 = 0;
          auto other = [&](int d, int n, int best) {  // pairs that skip the box step
            if (m == 0 || n == 0 || best <= 0) {  // empty alignment: 0/0
              emit(J, q, d, fraction_distance(0, 0));
              done16++;
            } else {  // the 16-bit lanes may have saturated: 32-bit DP
              const int w = atomicAdd(J.rerun_count, 1);
              if (w < J.rerun_cap) J.rerun[w] = make_int2(q, d);
              atomicAdd(J.stats + 2, 1ull);
            }
          };
          if (!goA) other(dA, nA, bA);
          if (dB >= 0 && !goB) other(dB, nB, bB);
          const int ng = (int)goA + (int)goB;
          if (ng) {
            wA = atomicAdd(J.box_count, ng);
            wB = wA + (int)goA;
          }
          atomicAdd(J.stats + 1, done16 + (unsigned long long)ng);
        }
        wA = __shfl_sync(0xffffffffu, wA, 0);
        wB = __shfl_sync(0xffffffffu, wB, 0);
        __syncwarp();  // the rows' bounds in rowb are visible to every lane
        // each half-warp writes one pair's box record and the threshold codes of its 128 rows
        // above ie (rows further up share one threshold, in the record)
        const int hl = lane & 15;
        const bool hB = lane >= 16;
        const bool go = hB ? goB : goA;
        const int S = hB ? bB : bA, ie = (hB ? rB : rA) + 1, w = hB ? wB : wA;
        uint32_t word = 0u;
        int umax = 0;
        if (go) {
          auto bound = [&](int i) {  // position row i >= 1: the best V of query row i - 1
            const uint32_t v = rowb[i - 1];
            return (int)(int16_t)(hB ? (v >> 16) : (v & 0xFFFFu)) - J.bias;
          };
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const int i = ie - 1 - (hl * 8 + u);
            const int ub = i >= 1 ? bound(i) : 0;
            word |= (uint32_t)reg_code_of(S - min(ub, S)) << (4 * u);
          }
          for (int i = 1 + hl; i <= ie - 1 - kRegWinRows; i += 16) umax = max(umax, bound(i));
        }
#pragma unroll
        for (int x = 8; x >= 1; x >>= 1) umax = max(umax, __shfl_xor_sync(0xffffffffu, umax, x));
        if (go && w < J.box_cap) {
          J.boxwin[(long long)w * kRegWinWords + hl] = word;
          if (hl == 0)
            J.box[w] = make_int4(q, hB ? dB : dA, S | ((S - min(umax, S)) << 16),
                                 (int)(((uint32_t)ie << 16) | ((hB ? cB : cA) + 1)));
        }
        __syncwarp();
        continue;
      }
      if constexpr (KIND == kKindKim) {
        int bA, rA, bB, rB;
        uint2 cA, cB;
        if (m > 0 && ncols > 0) {
          align_two_kim<K>(prof, J.mpad, passes, ca, cb, ncols, J, scr, lane, bA, rA, cA, bB, rB, cB);
        } else {
          bA = bB = 0; rA = rB = 0; cA = cB = make_uint2(0u, 0u);
        }
        warp_best2(bA, rA, cA);
        warp_best2(bB, rB, cB);
        if (lane == 0) {
          const bool tA = bA > J.thresh && m > 0 && nA > 0, tB = dB >= 0 && bB > J.thresh && m > 0 && nB > 0;
          atomicAdd(J.stats + 1, (unsigned long long)(1 + (dB >= 0)) - (unsigned long long)(tA + tB));
          if (tA + tB) atomicAdd(J.stats + 2, (unsigned long long)(tA + tB));
          // Int16 distance from the counters (SWG-MS caps Kimura2 and maps Log(Zero) to 10)
          const bool ms = J.mode == kModeSwgMs;
          if (tA) {
            const int w = atomicAdd(J.rerun_count, 1);
            if (w < J.rerun_cap) J.rerun[w] = make_int2(q, dA);
          } else {
            const uint2 c = (m > 0 && nA > 0) ? cA : make_uint2(0u, 0u);
            emit(J, q, dA, kim_distance(KimCnt::T{c.x, c.y}, J.dist_fn, ms, J.throws));
          }
          if (dB >= 0) {
            if (tB) {
              const int w = atomicAdd(J.rerun_count, 1);
              if (w < J.rerun_cap) J.rerun[w] = make_int2(q, dB);
            } else {
              const uint2 c = (m > 0 && nB > 0) ? cB : make_uint2(0u, 0u);
              emit(J, q, dB, kim_distance(KimCnt::T{c.x, c.y}, J.dist_fn, ms, J.throws));
            }
          }
        }
        __syncwarp();
        continue;
      }
      if constexpr (NW) {
        uint32_t wa = 0, wb = 0;
        if (m > 0 && ncols > 0)
          align_two_nw<K, NP>(prof, J.mpad, passes, m, ca, cb, ncols, nA, nB, J, scr, lane, wa, wb);
        if (lane == 0) {
          if (m == 0 || nA == 0) wa = nw_boundary(m, nA, J.protein);
          emit(J, q, dA, engine_nw_distance(wa));
          if (dB >= 0) {
            if (m == 0 || nB == 0) wb = nw_boundary(m, nB, J.protein);
            emit(J, q, dB, engine_nw_distance(wb));
          }
          atomicAdd(J.stats + 1, (unsigned long long)(1 + (dB >= 0)));
        }
        __syncwarp();
        continue;
      }
      int bA, rA, bB, rB;
      uint32_t cA, cB;
      if (m > 0 && ncols > 0) {
        align_two<K, NP>(prof, J.mpad, passes, ca, cb, ncols, J, scr, lane, bA, rA, cA, bB, rB, cB);
      } else {
        bA = bB = 0; rA = rB = 0; cA = cB = 0u;
      }
      warp_best(bA, rA, cA);
      warp_best(bB, rB, cB);
      if (lane == 0) {
        const unsigned long long tripped = (bA > J.thresh && m > 0 && nA > 0) + (dB >= 0 && bB > J.thresh && m > 0 && nB > 0);
        atomicAdd(J.stats + 1, (unsigned long long)(1 + (dB >= 0)) - tripped);
        if (tripped) atomicAdd(J.stats + 2, tripped);
        // a lane whose best reached the trip level is redone with 32-bit lanes
        if (bA > J.thresh && m > 0 && nA > 0) {
          const int w = atomicAdd(J.rerun_count, 1);
          if (w < J.rerun_cap) J.rerun[w] = make_int2(q, dA);
        } else {
          const uint32_t c = (m > 0 && nA > 0) ? cA : 0u;
          emit(J, q, dA, fraction_distance((int)(c & 0xFFFFu), (int)(c >> 16)));
        }
        if (dB >= 0) {
          if (bB > J.thresh && m > 0 && nB > 0) {
            const int w = atomicAdd(J.rerun_count, 1);
            if (w < J.rerun_cap) J.rerun[w] = make_int2(q, dB);
          } else {
            const uint32_t c = (m > 0 && nB > 0) ? cB : 0u;
            emit(J, q, dB, fraction_distance((int)(c & 0xFFFFu), (int)(c >> 16)));
          }
        }
      }
      __syncwarp();
    }
    __syncthreads();
    }  // segments
  }
}

// ---- third pass: the box step's give-ups bucketed by query (count, offsets, scatter) -----------
__global__ void fb_count_kernel(const int2* fb, const int* n, long long cap, int lo, int* cnt) {
  const long long np = min((long long)*n, cap);
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x)
    atomicAdd(cnt + (fb[p].x - lo), 1);
}

// Inclusive scan of v over the 1024 threads of the CTA (buf: 1024 ints of shared memory); all =
// the sum over the CTA.  buf is free again when it returns.
__device__ __forceinline__ int cta_scan_1024(int* buf, int v, int& all) {
  const int t = threadIdx.x;
  buf[t] = v;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const int x = t >= d ? buf[t - d] : 0;
    __syncthreads();
    buf[t] += x;
    __syncthreads();
  }
  const int r = buf[t];
  all = buf[1023];
  __syncthreads();
  return r;
}

// Exclusive prefix sums over the nq queries (one CTA of 1024 threads): start[] of the partner
// counts and cstart[] of their chunks (cstart[nq] = total[0] = all chunks); fill reset to 0.
// The chunk size (total[1], even, kFbChunkMin..kFbChunk partners) spreads the give-ups over
// about `target` work items (the launch's CTAs): a few hundred give-ups of long pairs -- a
// serving wave's -- then run on many SMs at once instead of a few CTAs working through 64
// partners each, which left the rest of the GPU idle for the whole launch.
__global__ void __launch_bounds__(1024) fb_scan_kernel(const int* cnt, int* start, int* fill, int* cstart,
                                                       int* total, int nq, int target) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const int per = (nq + 1023) / 1024, lo = min(nq, t * per), hi = min(nq, lo + per);
  int sum = 0;
  for (int k = lo; k < hi; k++) sum += cnt[k];
  int all, call;
  const int incl = cta_scan_1024(part, sum, all);
  const int want = (all + max(target, 1) - 1) / max(target, 1);
  const int chunk = min(kFbChunk, max(kFbChunkMin, (want + 1) & ~1));
  int csum = 0;
  for (int k = lo; k < hi; k++) csum += (cnt[k] + chunk - 1) / chunk;
  const int cincl = cta_scan_1024(part, csum, call);
  int run = incl - sum, crun = cincl - csum;
  for (int k = lo; k < hi; k++) {
    start[k] = run;
    cstart[k] = crun;
    run += cnt[k];
    crun += (cnt[k] + chunk - 1) / chunk;
    fill[k] = 0;
  }
  if (t == 0) {
    cstart[nq] = call;
    total[0] = call;
    total[1] = chunk;
  }
}

__global__ void fb_scatter_kernel(const int2* fb, const int* n, long long cap, int lo, const int* start, int* fill,
                                  int* sorted) {
  const long long np = min((long long)*n, cap);
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    const int2 pr = fb[p];
    const int q = pr.x - lo;
    sorted[start[q] + atomicAdd(fill + q, 1)] = pr.y;
  }
}

__global__ void zero_diagonal_kernel(int16_t* out, long long ld, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[(long long)i * ld + i] = 0;
}

// ------------------------------------------------------------------------------------------------
namespace {

constexpr int kNumK = 7;
constexpr int kKs[kNumK] = {4, 6, 8, 10, 12, 14, 16};
// Engine work counters: items taken, pairs finished in 16-bit lanes, tripped 16-bit lanes, pairs
// the box step gave up on, pairs handed to the warp box kernel.
constexpr int kNumStats = 8;
constexpr int kFbK = 16;  // rows per lane of the third pass (any query length, in passes of 512 rows)

// Largest alphabet of the 16-bit lanes (two-plane profiles beyond 8 letters).
constexpr int kMaxAlpha16 = 32;
int planes_of(int A) { return A > 8 ? 2 : 3; }

size_t engine_smem(int A, int mpad, int maxcol, int K, int kind = 0) {
  const int cbuf = 64 + ((maxcol + 31) / 32) * 32;
  return (size_t)(A + 1) * planes_of(A) * mpad * 4 + kMaxChunk * 4 + (size_t)warps_of(K, kind) * 2 * cbuf;
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

struct CodeLut {
  uint8_t v[128];
};

// Dense codes of residue bytes (refresh_codes).
__global__ void recode_kernel(const uint8_t* __restrict__ seq, uint8_t* __restrict__ code, int64_t n, CodeLut lut) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    code[k] = lut.v[seq[k] & 127];
}

// Calls fn(std::integral_constant<int, K>) for the engine instantiation of K rows per lane.
template <class Fn>
auto with_k(int K, Fn fn) {
  switch (K) {
    case 4: return fn(std::integral_constant<int, 4>());
    case 6: return fn(std::integral_constant<int, 6>());
    case 8: return fn(std::integral_constant<int, 8>());
    case 10: return fn(std::integral_constant<int, 10>());
    case 12: return fn(std::integral_constant<int, 12>());
    case 14: return fn(std::integral_constant<int, 14>());
    default: return fn(std::integral_constant<int, 16>());
  }
}

// The kernel instantiation for K rows per lane, the planes of alphabet A and the DP kind.
template <class Fn>
auto with_kp(int K, int A, int kind, Fn fn) {
  return with_k(K, [&](auto k) {
    constexpr int kk = decltype(k)::value;
    const int threads = warps_of(kk, kind) * 32;
    const bool p3 = planes_of(A) == 3;
    if (kind == kKindNw) return p3 ? fn(engine_kernel<kk, 3, kKindNw>, threads) : fn(engine_kernel<kk, 2, kKindNw>, threads);
    if (kind == kKindScore) return p3 ? fn(engine_kernel<kk, 3, kKindScore>, threads) : fn(engine_kernel<kk, 2, kKindScore>, threads);
    if (kind == kKindKim) {  // three planes and at most kKimMaxK rows per lane (the planner's rule)
      constexpr int kq = kk > kKimMaxK ? kKimMaxK : kk;
      return fn(engine_kernel<kq, 3, kKindKim>, warps_of(kq, kKindKim) * 32);
    }
    return p3 ? fn(engine_kernel<kk, 3, kKindSw>, threads) : fn(engine_kernel<kk, 2, kKindSw>, threads);
  });
}

// Raises an instantiation's dynamic shared-memory allowance to at least smem.  The attribute is
// per function and process-wide (every context and thread launches the same kernels), so it only
// ever grows: lowering it would fail launches of plans built earlier with a larger profile.
cudaError_t allow_smem_k(int K, int A, int kind, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int>, size_t> granted;  // (device, K, planes, kind)
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  size_t& g = granted[std::make_tuple(dev, K, planes_of(A), kind)];
  if (smem <= g) return cudaSuccess;
  const cudaError_t e = with_kp(K, A, kind, [&](auto kern, int) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  if (e == cudaSuccess) g = smem;
  return e;
}

cudaError_t launch_engine_k(int K, int kind, const EngineJob& J, int grid, size_t smem, cudaStream_t st) {
  return with_kp(K, J.A, kind, [&](auto kern, int threads) {
    kern<<<grid, threads, smem, st>>>(J);
    return cudaGetLastError();
  });
}

int occupancy_k(int K, int A, int kind, size_t smem) {
  return with_kp(K, A, kind, [&](auto kern, int threads) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem);
    return n;
  });
}

// Relative cost of one computed row at K rows per lane (100 = the cheapest), from B200 row-padded
// cell rates with K forced for every query: SW on the uneven 3,000-sequence DNA job, NW on the
// 3,000-sequence uniform 300-500 DNA job.
long k_weight_nw(int k) {
  switch (k) {
    case 4: return 160;
    case 6: return 127;
    case 8: return 106;
    case 10: return 107;
    case 12: return 100;
    case 14: return 105;
    default: return 100;
  }
}

long k_weight(int k) {
  switch (k) {
    case 4: return 188;
    case 6: return 157;
    case 8: return 132;
    case 10: return 106;
    case 12: return 101;
    case 14: return 111;
    default: return 100;
  }
}

// Rows per lane and passes for a query of m rows: fewest padded rows, then fewest passes.
// kmax: the largest rows per lane the kernel kind has (Kimura2 / JukesCantor: kKimMaxK).
void choose_k(int m, int kov, int* K, int* passes, bool nw = false, const int* tuned = nullptr, int kmax = 16) {
  if (kov) {
    kov = std::min(kov, kmax);
    *K = kov;
    *passes = std::max(1, (m + 32 * kov - 1) / (32 * kov));
    return;
  }
  long best = -1;
  for (int k : kKs) {
    if (k > kmax) continue;
    const int p = std::max(1, (m + 32 * k - 1) / (32 * k));
    // rows computed (padding included) times the per-row cost of that K (few rows per lane do
    // not amortise the per-step shuffles, loads and column bookkeeping); ties go to fewer passes
    // (each pass adds a wavefront fill and a scratch round trip)
    const int ki = (int)(std::find(std::begin(kKs), std::end(kKs), k) - std::begin(kKs));
    const long weight = (tuned && tuned[ki] > 0) ? tuned[ki] : nw ? k_weight_nw(k) : k_weight(k);
    const long cost = (long)p * 32 * k * weight * 16 + p;
    if (best < 0 || cost < best) { best = cost; *K = k; *passes = p; }
  }
}

struct Bin {
  int K;
  int mpad;
  int max_passes = 0;
  std::vector<int4> items;
  std::vector<double> cost;
  double total_cost = 0;
  int item_offset = 0;
  size_t smem = 0;
  int grid = 0;
  size_t scratch_off = 0;  // words into the pass scratch (bins run concurrently)
  size_t rowbuf_off = 0;   // two-pass: words into the rows' bounds buffer
  double padded = 0;       // cells computed, padding rows included
};

template <class T>
int upload_vec(T** dst, const std::vector<T>& v, std::string* msg, const char* what) {
  cudaFree(*dst);
  *dst = nullptr;
  if (cudaMalloc(dst, std::max<size_t>(v.size(), 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *msg = std::string("cudaMalloc ") + what;
    return SW_E_OOM;
  }
  if (!v.empty() && cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
    *msg = std::string("upload ") + what;
    return SW_E_CUDA;
  }
  return SW_OK;
}

// State of one sequence set shared by every plan: residue codes, length order, tables.
struct Base {
  int alpha = 0, bias = 1, max_s = 0, maxcol = 1;
  bool nw16 = false;  // NW fits the 16-bit lanes
  std::vector<int> len, sorted_h, letters;
  uint8_t* d_code = nullptr;
  int32_t* d_sorted = nullptr;
  int32_t* d_lettab = nullptr;
  uint32_t* d_flagtab = nullptr;
  uint32_t* d_kimtab = nullptr;  // Kimura2 / JukesCantor: A-flag | B-flag << 16 per letter pair
  uint32_t* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  void* d_carry = nullptr;
  long carry_threads = 0;
  CodeLut lut;  // residue byte -> dense code of d_code
  // two-pass SW: the first pass's box records (pair, best score, best cell) with the threshold
  // codes of the rows above each best cell, the box step's band classes and the pairs it hands to
  // the warp box kernel, and the score kernels' per-warp row bounds
  int4* d_box = nullptr;
  uint32_t* d_boxwin = nullptr;
  int* d_cls[2] = {nullptr, nullptr};
  int* d_counts = nullptr;     // [0] box records, [1] spilled pairs, [2..5] band classes
  long long box_cap = 0;
  int4* d_spill = nullptr;
  long long spill_cap = 0;
  uint32_t* d_rowbuf = nullptr;
  size_t rowbuf_bytes = 0;
  // third pass: the give-ups (pair list, bucketed partners) and per-query counts / offsets / fill
  int2* d_fb = nullptr;
  int* d_fbsorted = nullptr;
  int* d_fbq = nullptr;         // [4 * nseq + 3]: counts, offsets, fill, chunk offsets (+1), chunks, chunk size
  void free_box() {
    cudaFree(d_box); cudaFree(d_boxwin); cudaFree(d_cls[0]); cudaFree(d_cls[1]); cudaFree(d_spill);
    cudaFree(d_fb); cudaFree(d_fbsorted);
    d_box = nullptr; d_boxwin = nullptr; d_cls[0] = d_cls[1] = nullptr; d_spill = nullptr;
    d_fb = nullptr; d_fbsorted = nullptr;
    box_cap = spill_cap = 0;
  }
  ~Base() {
    cudaFree(d_code); cudaFree(d_sorted); cudaFree(d_lettab); cudaFree(d_flagtab); cudaFree(d_kimtab);
    cudaFree(d_scratch); cudaFree(d_carry);
    free_box();
    cudaFree(d_counts); cudaFree(d_rowbuf); cudaFree(d_fbq);
  }
};

// Residue codes of the sequence set, its length order and the dense score/flag tables of the
// 16-bit lanes (alphabets of up to 8 letters), plus the 32-bit lanes' scratch.
int build_base(Base& B, const EngineParams& P, std::string* msg) {
  const int N = P.nseq;
  const int64_t total = P.h_off[N];
  int code_of[128];
  std::fill(code_of, code_of + 128, -1);
  // (the dense code of every byte, for refresh_codes: bytes of no letter map to the pad code)
  std::vector<int> letters;
  for (int64_t k = 0; k < total; k++) {
    const int b = P.h_seq[k];
    if (code_of[b] < 0) { code_of[b] = (int)letters.size(); letters.push_back(b); }
  }
  B.alpha = (int)letters.size();
  B.letters = letters;
  B.len.resize(N);
  for (int i = 0; i < N; i++) B.len[i] = (int)(P.h_off[i + 1] - P.h_off[i]);
  B.maxcol = std::max(P.maxlen, 1);
  B.sorted_h.resize(N);
  std::iota(B.sorted_h.begin(), B.sorted_h.end(), 0);
  std::stable_sort(B.sorted_h.begin(), B.sorted_h.end(), [&](int a, int b) { return B.len[a] < B.len[b]; });
  int rc;
  // the 32-bit lanes (reruns, NW, large alphabets) need the plain kernel's scratch
  B.carry_threads = (long)P.sms * 8 * 128;
  if (cudaMalloc(&B.d_carry, plain_carry_bytes(P.mode == kModeNw ? kModeNw : kModeSwgMpi, B.carry_threads, B.maxcol, P.protein ? 0 : P.dist_fn)) != cudaSuccess) {
    cudaGetLastError(); B.d_carry = nullptr; *msg = "cudaMalloc 32-bit lane scratch"; return SW_E_OOM;
  }
  if (B.alpha > kMaxAlpha16 || P.lanes == SW_LANES_32) return SW_OK;
  const int A = B.alpha, A1 = A + 1;
  int maxS = 0, minS = 0;
  for (int a : letters)
    for (int b : letters) {
      const int s = P.h_scores[a * 128 + b];
      maxS = std::max(maxS, s);
      minS = std::min(minS, s);
    }
  const bool nw = P.mode == kModeNw;
  if (nw) {
    // Global alignment has no floor: the bias covers the all-gap lower bound of every cell a
    // pass touches (rows padded by up to 32 x 16 - 1, columns by up to 63), minus the most
    // negative score and a gap open + extend of intermediate values.  The lanes hold the
    // scores only if the highest possible V still fits: otherwise 32-bit lanes.
    const long span = (long)B.maxcol + 512 + (long)B.maxcol + 64;
    const long bias = 3L * P.o + 2L * P.e + span * P.e - minS;
    if (bias + (long)maxS * (B.maxcol + 1) > 32767) return SW_OK;
    B.bias = (int)bias;
    B.nw16 = true;
  } else {
    B.bias = std::max(std::max(P.o + 2 * P.e, -minS), 1);
  }
  B.max_s = maxS;
  std::vector<int32_t> lettab((size_t)A1 * A1);
  std::vector<uint32_t> flagtab((size_t)A1 * A1, 0u), kimtab((size_t)A1 * A1, 0u);
  for (int a = 0; a < A1; a++)
    for (int c = 0; c < A1; c++) {
      int s;
      uint32_t f = 0, fk = 0;
      if (a == A || c == A) s = nw ? 0 : -B.bias;  // padding: NW keeps its values bounded
      else {
        s = P.h_scores[letters[a] * 128 + letters[c]];
        const uint32_t fl = P.h_flags[letters[a] * 128 + letters[c]];
        f = fl & kFlagCount;
        fk = ((fl & kFlagCntA) ? 1u : 0u) | ((fl & kFlagCntB) ? 0x10000u : 0u);
      }
      lettab[(size_t)a * A1 + c] = s + P.o;
      flagtab[(size_t)a * A1 + c] = f;
      kimtab[(size_t)a * A1 + c] = fk;
    }
  for (int x = 0; x < 128; x++) B.lut.v[x] = (uint8_t)(code_of[x] < 0 ? A : code_of[x]);
  std::vector<uint8_t> code((size_t)total + 64, (uint8_t)A);
  for (int64_t k = 0; k < total; k++) code[(size_t)k] = (uint8_t)code_of[P.h_seq[k]];
  if ((rc = upload_vec(&B.d_code, code, msg, "codes"))) return rc;
  if ((rc = upload_vec(&B.d_sorted, B.sorted_h, msg, "order"))) return rc;
  if ((rc = upload_vec(&B.d_lettab, lettab, msg, "score table"))) return rc;
  if ((rc = upload_vec(&B.d_flagtab, flagtab, msg, "flag table"))) return rc;
  if (P.dist_fn != 0 && !P.protein && (rc = upload_vec(&B.d_kimtab, kimtab, msg, "Kimura flag table")))
    return rc;
  return SW_OK;
}

// One job (mode, world size, query range): its work items, 32-bit pair list and CUDA graph.
struct Plan {
  bool plain_only = false;
  int kind = kKindSw;       // the bins' kernel: SW with counters, NW, or the two-pass first pass
  bool fb = false;          // two-pass: the box step's give-ups run on 16-bit lanes (third pass)
  int fb_mpad = 0, fb_grid = 0;
  size_t fb_smem = 0;
  bool zeroes_diagonal = false;
  int thresh = 0;
  std::vector<Bin> bins;
  std::vector<int> order;  // non-empty bins in launch order
  int big_count = 0, rerun_cap = 0;
  int64_t npairs = 0, ncells = 0;
  int4* d_items = nullptr;
  int* d_counters = nullptr;
  int2* d_rerun = nullptr;
  int* d_rerun_count = nullptr;
  unsigned long long* d_stats = nullptr;
  cudaGraphExec_t graph = nullptr;
  int16_t* graph_out = nullptr;
  long long graph_ld = 0;
  cudaStream_t graph_stream = nullptr;
  ~Plan() {
    if (graph) cudaGraphExecDestroy(graph);
    cudaFree(d_items); cudaFree(d_counters); cudaFree(d_rerun); cudaFree(d_rerun_count); cudaFree(d_stats);
  }
};

// A job's pairs: the queries row_lo..row_hi with the orientation of a `ranks`-rank run (block 0),
// or one block of the pair matrix, rows row_lo..row_hi by columns col_lo..col_hi (block 1: a
// diagonal block, block 2: off-diagonal).
struct PlanKey {
  int mode, ranks, row_lo, row_hi, block, col_lo, col_hi;
  bool operator<(const PlanKey& o) const {
    return std::tie(mode, ranks, row_lo, row_hi, block, col_lo, col_hi) <
           std::tie(o.mode, o.ranks, o.row_lo, o.row_hi, o.block, o.col_lo, o.col_hi);
  }
};

bool oriented_host(int mode, const std::vector<int>& blk, int q, int d) {
  if (mode == kModeSwgMs) return true;
  if (q == d) return false;
  if (blk[q] == blk[d]) return q > d;
  const bool odd = ((blk[q] + blk[d]) & 1) != 0;
  return (blk[q] > blk[d] && !odd) || (blk[q] < blk[d] && odd);
}

class EngineImpl : public Engine {
 public:
  ~EngineImpl() override { invalidate(); release_streams(); }
  int refresh_codes(const uint8_t* d_seq, int64_t total, cudaStream_t st, std::string* msg) override {
    if (!base_ || !base_->d_code || total <= 0) return SW_OK;
    recode_kernel<<<(int)std::min<int64_t>((total + 255) / 256, 4096), 256, 0, st>>>(d_seq, base_->d_code, total, base_->lut);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { *msg = std::string("recode: ") + cudaGetErrorString(e); return SW_E_CUDA; }
    return SW_OK;
  }
  void invalidate() override {
    plans_.clear();
    base_.reset();
    last_ = nullptr;
  }
  EngineOptions& options() override {
    plans_.clear();  // options shape the plans; sequence state stays
    last_ = nullptr;
    return opt_;
  }
  const EngineOptions& current_options() const override { return opt_; }
  void set_plan_only(int v) override { opt_.plan_only = v; }

  int64_t stat(const char* key) const override {
    const std::string k(key);
    if (!last_) return 0;
    if (k == "launches") {
      int64_t n = 2;  // the 32-bit lane kernel and the rerun-count reset
      for (auto& bn : last_->bins) n += bn.items.empty() ? 0 : 1;
      if (!last_->plain_only && last_->kind == kKindScore)  // the box step: scan, 4 band classes, warp kernel
        n += (opt_.box_reg ? 6 : 1) + (last_->fb ? 4 : 0);  // third pass: count, scan, scatter, kernel
      return n + (last_->zeroes_diagonal ? 1 : 0);
    }
    if (k == "bins") {
      int64_t n = 0;
      for (auto& bn : last_->bins) n += bn.items.empty() ? 0 : 1;
      return n;
    }
    if (k == "alphabet") return base_ ? base_->alpha : 0;
    if (k == "items" || k == "lane16_pairs" || k == "tripped" || k == "box_fallbacks" || k == "box_spilled" ||
        k == "box_third_pass" || k == "kernel_error") {
      if (!last_->d_stats) return 0;
      unsigned long long h[kNumStats] = {};
      cudaDeviceSynchronize();
      cudaMemcpy(h, last_->d_stats, sizeof(h), cudaMemcpyDeviceToHost);
      return (int64_t)(k == "items" ? h[0] : k == "lane16_pairs" ? h[1] : k == "tripped" ? h[2]
                       : k == "box_fallbacks" ? h[3] : k == "box_spilled" ? h[4]
                       : k == "box_third_pass" ? h[5] : h[7]);
    }
    if (k == "planned_items") {
      int64_t n = 0;
      for (auto& bn : last_->bins) n += (int64_t)bn.items.size();
      return n;
    }
    return -1;
  }

  int autotune(const EngineParams& P0, int weights[7], std::string* msg) override {
    int rc;
    for (int x = 0; x < kNumK; x++) weights[x] = 0;
    if (!base_) {
      base_.reset(new Base());
      if ((rc = build_base(*base_, P0, msg))) { base_.reset(); return rc; }
    }
    Base& B = *base_;
    const bool nw = P0.mode == kModeNw;
    const bool kim = P0.dist_fn != 0 && !P0.protein;
    // 32-bit lanes only: nothing to choose; Kimura2 / JukesCantor (at most 8 rows per lane, two
    // counter words) keep the built-in costs
    if (B.alpha > kMaxAlpha16 || (nw && !B.nw16) || kim || P0.lanes == SW_LANES_32 || P0.nseq < 2)
      return SW_OK;
    if ((rc = ensure_streams(msg))) return rc;
    // sample: the last R queries of the set (each aligned against every earlier sequence); each
    // K is timed on the sampled queries it serves in one pass with under 64 rows of padding
    // (lengths in (32(K-2), 32K]), the regime where it competes with its neighbours
    const int N = P0.nseq;
    double mean = 0;
    for (int l : B.len) mean += l;
    mean = std::max(1.0, mean / N);
    const int R = (int)std::max(64.0, std::min((double)N, 2e12 / ((double)N * mean * mean)));
    EngineParams P = P0;
    P.ranks = 1;
    P.row_lo = N - R;
    P.row_hi = N - 1;
    const PlanKey key{P.mode, 1, P.row_lo, P.row_hi, 0, 0, -1};
    const int saved = opt_.k_override;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    double rate[kNumK] = {0};
    for (int x = 0; x < kNumK; x++) {
      opt_.k_override = kKs[x];
      opt_.m_lo = 32 * (kKs[x] - 2);
      opt_.m_hi = 32 * kKs[x];
      Plan pl;
      rc = build_plan(P, key, pl, msg);
      opt_.m_lo = opt_.m_hi = 0;
      if (rc) break;
      double padded = 0;
      for (auto& bn : pl.bins) padded += bn.padded;
      if (padded < 1e9) continue;  // too few sampled queries of these lengths: built-in cost
      float ms = 0;
      cudaError_t e = enqueue(P, key, pl, t0, t1);
      if (e == cudaSuccess) e = cudaStreamSynchronize(P.stream);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
      if (e != cudaSuccess) { *msg = std::string("autotune: ") + cudaGetErrorString(e); rc = SW_E_CUDA; break; }
      if (ms > 0 && padded > 0) rate[x] = padded / ms;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    opt_.k_override = saved;
    if (rc) return rc;
    double best = 0;
    for (double r : rate) best = std::max(best, r);
    if (best <= 0) return SW_OK;
    int tuned[kNumK];
    for (int x = 0; x < kNumK; x++) tuned[x] = rate[x] > 0 ? (int)std::lround(100.0 * best / rate[x]) : 0;
    // keep the measured costs only if they plan the whole sample faster than the current ones
    double t_cur = 0, t_new = 0;
    const int saved_w[kNumK] = {opt_.k_weights[0], opt_.k_weights[1], opt_.k_weights[2], opt_.k_weights[3],
                                opt_.k_weights[4], opt_.k_weights[5], opt_.k_weights[6]};
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    for (int variant = 0; variant < 2 && rc == SW_OK; variant++) {
      for (int x = 0; x < kNumK; x++) opt_.k_weights[x] = variant ? tuned[x] : saved_w[x];
      Plan pl;
      if ((rc = build_plan(P, key, pl, msg))) break;
      float ms = 0;
      cudaError_t e = enqueue(P, key, pl, t0, t1);
      if (e == cudaSuccess) e = cudaStreamSynchronize(P.stream);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
      if (e != cudaSuccess) { *msg = std::string("autotune: ") + cudaGetErrorString(e); rc = SW_E_CUDA; break; }
      (variant ? t_new : t_cur) = ms;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    const bool take = rc == SW_OK && t_new > 0 && t_new < t_cur;
    for (int x = 0; x < kNumK; x++) {
      opt_.k_weights[x] = take ? tuned[x] : saved_w[x];
      weights[x] = take ? tuned[x] : 0;  // 0: the built-in table stays
    }
    plans_.clear();  // later plans use the chosen costs
    last_ = nullptr;
    return rc;
  }

  int rerun_count(cudaStream_t st, int64_t* count, std::string* msg) override {
    *count = 0;
    if (!last_ || last_->plain_only || !last_->d_rerun_count) return SW_OK;
    int hc = 0;
    cudaError_t e = cudaMemcpyAsync(&hc, last_->d_rerun_count, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { *msg = std::string("rerun count: ") + cudaGetErrorString(e); return SW_E_CUDA; }
    if (hc > last_->rerun_cap) { *msg = "rerun list overflow"; return SW_E_OOM; }
    *count = hc;
    return SW_OK;
  }

  int run(const EngineParams& P, int64_t* pairs, int64_t* cells, int64_t* reruns,
          std::string* msg) override {
    int rc;
    if (!base_) {
      base_.reset(new Base());
      if ((rc = build_base(*base_, P, msg))) { base_.reset(); return rc; }
    }
    const int N = P.nseq;
    PlanKey key{P.mode, P.ranks, std::max(0, P.row_lo), P.row_hi < 0 ? N - 1 : std::min(N - 1, P.row_hi),
                P.block, P.block ? P.col_lo : 0, P.block ? P.col_hi : -1};
    auto it = plans_.find(key);
    if (it == plans_.end()) {
      std::unique_ptr<Plan> pl(new Plan());
      if ((rc = build_plan(P, key, *pl, msg))) return rc;
      it = plans_.emplace(key, std::move(pl)).first;
    }
    Plan& pl = *it->second;
    last_ = &pl;
    if ((rc = ensure_streams(msg))) return rc;
    cudaError_t e;
    if (opt_.use_graph) {
      if (!pl.graph || P.out != pl.graph_out || P.ld != pl.graph_ld || P.stream != pl.graph_stream) {
        if (pl.graph) cudaGraphExecDestroy(pl.graph);
        pl.graph = nullptr;
        cudaStreamBeginCapture(P.stream, cudaStreamCaptureModeThreadLocal);
        e = enqueue(P, key, pl);
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(P.stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
          if (g) cudaGraphDestroy(g);
          cudaGetLastError();
          *msg = std::string("graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2);
          return SW_E_CUDA;
        }
        e = cudaGraphInstantiate(&pl.graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { pl.graph = nullptr; *msg = "graph instantiate"; return SW_E_CUDA; }
        pl.graph_out = P.out; pl.graph_ld = P.ld; pl.graph_stream = P.stream;
      }
      e = opt_.plan_only ? cudaSuccess : cudaGraphLaunch(pl.graph, P.stream);
    } else {
      e = opt_.plan_only ? cudaSuccess : enqueue(P, key, pl);
    }
    if (e != cudaSuccess) { *msg = std::string("engine launch: ") + cudaGetErrorString(e); return SW_E_CUDA; }
    *reruns = -1;  // known once the stream is done (rerun_count)
    *pairs = pl.npairs;
    *cells = pl.ncells;
    return SW_OK;
  }

 private:
  int build_plan(const EngineParams& P, const PlanKey& key, Plan& pl, std::string* msg) {
    Base& B = *base_;
    const int N = P.nseq;
    std::vector<int> starts(P.ranks), ends(P.ranks), blk(N);
    sw_partition_ranges(0, N, P.ranks, starts.data(), ends.data());
    for (int r = 0; r < P.ranks; r++)
      for (int x = starts[r]; x <= ends[r]; x++) blk[x] = r;
    int rc;
    // the pairs (s1 = q, s2 = d) of the job or block, and the columns d ranges over
    auto allowed = [&](int q, int d) {
      if (key.block) return d >= key.col_lo && d <= key.col_hi && (key.block == 2 || P.mode == kModeSwgMs || d < q);
      return oriented_host(P.mode, blk, q, d);
    };
    const int dlo = key.block ? key.col_lo : 0, dhi = key.block ? key.col_hi : N - 1;
    const bool nw = P.mode == kModeNw;
    // Kimura2 / JukesCantor of SWG-MPI / SWG-MS on nucleic letters that fit three profile planes:
    // the 16-bit kernels with two counter words; NW's and the MinMaxNormScore rule: 32-bit lanes
    const bool kim = P.dist_fn != 0 && !P.protein;
    const bool kim16 = kim && (P.dist_fn == 1 || P.dist_fn == 2) && !nw && planes_of(B.alpha) == 3;
    pl.plain_only = B.alpha > kMaxAlpha16 || (nw && !B.nw16) || (kim && !kim16) || P.lanes == SW_LANES_32;
    // Two passes pay off only where the box step finishes nearly every pair: a pair it gives up
    // on costs the int32 full DP, about nine times a score-pass cell, so a few per cent of them
    // eat the gain.  The box step needs short local alignments and short gap chains (they decay by
    // min(o, e) per column).  Measured on the CPU with the box step's own source over uneven DNA
    // families (EDNAFULL) and BLOSUM62 protein families: with o >= 3 max S and e >= 3 it finished
    // 93-100 % of the pairs; with cheaper opening (EDNAFULL o <= 12, any BLOSUM62 setting) unrelated
    // sequences align over most of their length and it finished 0-70 % (EDNAFULL 10/3: 3 %); with
    // e <= 2 the gap chains outrun its window (BLOSUM62 10/1: 2 %).  two_pass = 1 applies that
    // rule, 2 uses two passes whenever min(o, e) >= 2, 0 never.
    const bool two_pass_ok = std::min(P.o, P.e) >= 2 &&
                             (opt_.two_pass == 2 || (opt_.two_pass == 1 && P.o >= 3 * B.max_s && P.e >= 3));
    pl.kind = nw ? kKindNw : kim16 ? kKindKim : two_pass_ok ? kKindScore : kKindSw;
    std::vector<int2> big;
    if (pl.plain_only) {
      for (int q = key.row_lo; q <= key.row_hi; q++)
        for (int d = dlo; d <= dhi; d++) {
          if (!allowed(q, d)) continue;
          big.push_back(make_int2(q, d));
          pl.ncells += (int64_t)B.len[q] * B.len[d];
        }
      pl.npairs = (int64_t)big.size();
      pl.big_count = (int)big.size();
      pl.rerun_cap = std::max(pl.big_count, 1);
      if ((rc = upload_vec(&pl.d_rerun, big, msg, "pair list"))) return rc;
      std::vector<int> cnt(1, pl.big_count);
      return upload_vec(&pl.d_rerun_count, cnt, msg, "pair count");
    }
    const int A = B.alpha;
    pl.thresh = (opt_.int16_threshold >= 0) ? (int)opt_.int16_threshold : 32767 - B.bias - B.max_s;
    // large jobs: fewer, longer items (1 % faster on the 20,000-sequence job); small ones keep
    // enough items to fill the GPU (the 1,000-sequence job is 5 % slower with 1,024)
    const int chunk = opt_.chunk ? std::min(std::max(opt_.chunk, 32), kMaxChunk) : (N >= 8192 ? 1024 : 512);
    const int nchunks = (N + chunk - 1) / chunk;
    std::vector<std::vector<int>> cidx(nchunks);
    std::vector<std::vector<double>> csum(nchunks);
    std::vector<int> cmaxlen(nchunks, 0);
    for (int c = 0; c < nchunks; c++) {
      for (int k = c * chunk; k < std::min(N, (c + 1) * chunk); k++) {
        cidx[c].push_back(B.sorted_h[k]);
        cmaxlen[c] = std::max(cmaxlen[c], B.len[B.sorted_h[k]]);
      }
      std::sort(cidx[c].begin(), cidx[c].end());
      csum[c].assign(cidx[c].size() + 1, 0.0);
      for (size_t k = 0; k < cidx[c].size(); k++) csum[c][k + 1] = csum[c][k] + B.len[cidx[c][k]];
    }
    pl.bins.clear();
    for (int k : kKs) { Bin b; b.K = k; b.mpad = 0; pl.bins.push_back(b); }
    for (int q = key.row_lo; q <= key.row_hi; q++) {
      const int m = B.len[q];
      if (opt_.m_hi > 0 && (m <= opt_.m_lo || m > opt_.m_hi)) continue;  // autotuner sample
      int K, passes;
      choose_k(m, opt_.k_override, &K, &passes, nw, opt_.k_weights, pl.kind == kKindKim ? kKimMaxK : 16);
      // a profile beyond shared memory (long queries, large alphabets): 32-bit lanes
      const bool fits = engine_smem(A, passes * 32 * K, B.maxcol, K, pl.kind) <= 227 * 1024;
      const int bi = (int)(std::find(std::begin(kKs), std::end(kKs), K) - std::begin(kKs));
      const int bq = blk[q];
      for (int c = 0; c < nchunks; c++) {
        const auto& ix = cidx[c];
        long cnt = 0;
        double lsum = 0;
        auto range_count = [&](int lo, int hi) {  // entries with lo <= index < hi
          const auto a = std::lower_bound(ix.begin(), ix.end(), lo) - ix.begin();
          const auto b = std::lower_bound(ix.begin(), ix.end(), hi) - ix.begin();
          cnt += (long)(b - a);
          lsum += csum[c][b] - csum[c][a];
        };
        if (key.block) {
          const bool below = key.block == 1 && P.mode != kModeSwgMs;
          range_count(key.col_lo, below ? std::min(q, key.col_hi + 1) : key.col_hi + 1);
        } else if (P.mode == kModeSwgMs) {
          range_count(0, N);
        } else {
          for (int r = 0; r < P.ranks; r++) {
            if (starts[r] > ends[r]) continue;
            if (r == bq) range_count(starts[r], q);
            else {
              const bool odd = ((bq + r) & 1) != 0;
              if ((bq > r && !odd) || (bq < r && odd)) range_count(starts[r], ends[r] + 1);
            }
          }
        }
        if (cnt == 0) continue;
        pl.npairs += cnt;
        pl.ncells += (int64_t)((double)m * lsum);
        const int mn = std::min(m, cmaxlen[c]);
        if (!fits || (long)B.max_s * (mn + 1) + B.bias > 32767) {
          // 16-bit lanes cannot hold this item's scores: its pairs go to 32-bit lanes
          for (int k = c * chunk; k < std::min(N, (c + 1) * chunk); k++) {
            const int d = B.sorted_h[k];
            if (allowed(q, d)) big.push_back(make_int2(q, d));
          }
          continue;
        }
        Bin& bn = pl.bins[bi];
        bn.mpad = std::max(bn.mpad, passes * 32 * K);
        bn.max_passes = std::max(bn.max_passes, passes);
        bn.items.push_back(make_int4(q, c * chunk, std::min(N, (c + 1) * chunk), passes));
        bn.cost.push_back((double)passes * 32 * K * (lsum + 31.0 * cnt) * k_weight(K));
        bn.padded += (double)passes * 32 * K * lsum;
        bn.total_cost += bn.cost.back();
      }
    }
    std::vector<int4> all;
    for (auto& bn : pl.bins) {
      std::vector<size_t> ord(bn.items.size());
      std::iota(ord.begin(), ord.end(), 0);
      std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return bn.cost[a] > bn.cost[b]; });
      bn.item_offset = (int)all.size();
      for (size_t k : ord) all.push_back(bn.items[k]);
    }
    if ((rc = upload_vec(&pl.d_items, all, msg, "items"))) return rc;
    std::vector<unsigned long long> st0(kNumStats, 0ull);
    if ((rc = upload_vec(&pl.d_stats, st0, msg, "stats"))) return rc;
    std::vector<int> zeros(pl.bins.size() + 1, 0);
    if ((rc = upload_vec(&pl.d_counters, zeros, msg, "counters"))) return rc;
    // the bins run concurrently: each multi-pass bin gets its own scratch slots (and each
    // score bin its own rows' bounds)
    size_t scr_words = 0, row_words = 0;
    for (auto& bn : pl.bins) {
      if (bn.items.empty()) continue;
      bn.smem = engine_smem(A, bn.mpad, B.maxcol, bn.K, pl.kind);
      if (bn.smem > 227 * 1024) { *msg = "query profile exceeds shared memory"; return SW_E_UNSUPPORTED; }
      if (allow_smem_k(bn.K, A, pl.kind, bn.smem) != cudaSuccess) { cudaGetLastError(); *msg = "shared memory opt-in"; return SW_E_CUDA; }
      const int occ = std::max(1, occupancy_k(bn.K, A, pl.kind, bn.smem));
      bn.grid = (int)std::min<long>((long)P.sms * occ, (long)bn.items.size());
      bn.scratch_off = scr_words;
      if (bn.max_passes > 1)
        scr_words += (size_t)bn.grid * warps_of(bn.K, pl.kind) * B.maxcol * (pl.kind == kKindKim ? kScrWordsKim : kScrWords);
      bn.rowbuf_off = row_words;
      if (pl.kind == kKindScore) row_words += (size_t)bn.grid * warps_of(bn.K, pl.kind) * bn.mpad;
    }
    pl.order.clear();
    for (size_t b = 0; b < pl.bins.size(); b++)
      if (!pl.bins[b].items.empty()) pl.order.push_back((int)b);
    // most work first: its CTAs take the SMs, the lighter bins fill in as its queue drains
    std::stable_sort(pl.order.begin(), pl.order.end(),
                     [&](int a, int b) { return pl.bins[a].total_cost > pl.bins[b].total_cost; });
    pl.big_count = (int)big.size();
    // the two-pass box kernel may give any pair to the 32-bit lanes: room for all of them
    const int64_t spare = pl.kind == kKindScore ? pl.npairs : std::max<int64_t>(1 << 16, pl.npairs / 16);
    pl.rerun_cap = (int)std::min<int64_t>(pl.npairs + 1, (int64_t)big.size() + spare);
    if (pl.kind == kKindScore) {
      // one set of box-step buffers for every plan (plans run one after another); every plan's
      // graph holds their pointers, so growing them retires the graphs
      auto retire = [&]() {
        for (auto& kv : plans_) if (kv.second->graph) { cudaGraphExecDestroy(kv.second->graph); kv.second->graph = nullptr; }
      };
      if (pl.npairs > B.box_cap) {
        retire();
        B.free_box();
        const size_t n = (size_t)std::max<int64_t>(pl.npairs, 1);
        const size_t nspill = std::max<size_t>(n / 16, 1 << 16);
        if (cudaMalloc(&B.d_box, sizeof(int4) * n) != cudaSuccess ||
            cudaMalloc(&B.d_fb, sizeof(int2) * n) != cudaSuccess ||
            cudaMalloc(&B.d_fbsorted, sizeof(int) * n) != cudaSuccess ||
            cudaMalloc(&B.d_boxwin, sizeof(uint32_t) * kRegWinWords * n) != cudaSuccess ||
            cudaMalloc(&B.d_cls[0], sizeof(int) * n) != cudaSuccess ||
            cudaMalloc(&B.d_cls[1], sizeof(int) * n) != cudaSuccess ||
            cudaMalloc(&B.d_spill, sizeof(int4) * nspill) != cudaSuccess) {
          cudaGetLastError();
          B.free_box();
          *msg = "cudaMalloc two-pass pair lists";
          return SW_E_OOM;
        }
        B.box_cap = (long long)n;
        B.spill_cap = (long long)nspill;
      }
      if (!B.d_counts && cudaMalloc(&B.d_counts, sizeof(int) * 8) != cudaSuccess) {
        cudaGetLastError(); B.d_counts = nullptr; *msg = "cudaMalloc two-pass counts"; return SW_E_OOM;
      }
      if (!B.d_fbq && cudaMalloc(&B.d_fbq, sizeof(int) * (4 * (size_t)std::max(N, 1) + 3)) != cudaSuccess) {
        cudaGetLastError(); B.d_fbq = nullptr; *msg = "cudaMalloc third-pass counts"; return SW_E_OOM;
      }
      // the third pass (16 rows per lane, every query's profile in shared memory) where it fits;
      // its scratch carries multi-pass rows like the bins'
      pl.fb_mpad = ((B.maxcol + 32 * kFbK - 1) / (32 * kFbK)) * 32 * kFbK;
      pl.fb_smem = engine_smem(A, pl.fb_mpad, B.maxcol, kFbK, kKindSw);
      pl.fb = opt_.third_pass && pl.fb_smem <= 227 * 1024 &&
              allow_smem_k(kFbK, A, kKindSw, pl.fb_smem) == cudaSuccess;
      cudaGetLastError();
      if (pl.fb) {
        pl.fb_grid = P.sms * std::max(1, occupancy_k(kFbK, A, kKindSw, pl.fb_smem));
        scr_words = std::max(scr_words, (size_t)pl.fb_grid * warps_of(kFbK) * B.maxcol * kScrWords);
      }
      const size_t rb = std::max<size_t>(row_words * 4, 16);
      if (rb > B.rowbuf_bytes) {
        retire();
        cudaFree(B.d_rowbuf);
        B.d_rowbuf = nullptr;
        B.rowbuf_bytes = 0;
        if (cudaMalloc(&B.d_rowbuf, rb) != cudaSuccess) { cudaGetLastError(); *msg = "cudaMalloc row bounds"; return SW_E_OOM; }
        B.rowbuf_bytes = rb;
      }
    }
    const size_t scr = std::max<size_t>(scr_words * 4, 16);
    if (scr > B.scratch_bytes) {
      cudaFree(B.d_scratch);
      B.d_scratch = nullptr;
      B.scratch_bytes = 0;
      // every plan's graph holds the scratch pointer: growing it retires them
      for (auto& kv : plans_) if (kv.second->graph) { cudaGraphExecDestroy(kv.second->graph); kv.second->graph = nullptr; }
      if (cudaMalloc(&B.d_scratch, scr) != cudaSuccess) { cudaGetLastError(); *msg = "cudaMalloc pass scratch"; return SW_E_OOM; }
      B.scratch_bytes = scr;
    }
    std::vector<int2> rl(big);
    rl.resize((size_t)pl.rerun_cap);
    if ((rc = upload_vec(&pl.d_rerun, rl, msg, "rerun list"))) return rc;
    std::vector<int> cnt(1, 0);
    return upload_vec(&pl.d_rerun_count, cnt, msg, "rerun count");
  }

  // bins_t0 / bins_t1 (optional): events recorded around the bins' kernels (the autotuner's
  // timing: rows per lane changes them and nothing else).
  cudaError_t enqueue(const EngineParams& P, const PlanKey& key, Plan& pl, cudaEvent_t bins_t0 = nullptr,
                      cudaEvent_t bins_t1 = nullptr) {
    Base& B = *base_;
    cudaError_t e;
    pl.zeroes_diagonal = !key.block && P.mode != kModeSwgMs && P.nseq > 0 && key.row_lo == 0 && key.row_hi == P.nseq - 1;
    // the mirrored entry (s2, s1) of each pair: a symmetric job's, or a diagonal block's (inside the
    // block); an off-diagonal block's mirror lies outside the block and is the caller's to fill
    const int mirror = key.block ? (key.block == 1 ? 1 : 0) : (P.mode != kModeSwgMs ? 1 : 0);
    if (pl.zeroes_diagonal)
      zero_diagonal_kernel<<<(P.nseq + 255) / 256, 256, 0, P.stream>>>(P.out, P.ld, P.nseq);
    set_int_kernel<<<1, 1, 0, P.stream>>>(pl.d_rerun_count, pl.big_count);
    const bool two = !pl.plain_only && pl.kind == kKindScore;
    EngineJob J3;  // the bins' job, the third pass's template
    std::memset(&J3, 0, sizeof(J3));
    if (two && (e = cudaMemsetAsync(B.d_counts, 0, sizeof(int) * 8, P.stream)) != cudaSuccess) return e;
    if (!pl.plain_only) {
      if ((e = cudaMemsetAsync(pl.d_counters, 0, sizeof(int) * (pl.bins.size() + 1), P.stream)) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(pl.d_stats, 0, sizeof(unsigned long long) * kNumStats, P.stream)) != cudaSuccess) return e;
      EngineJob J;
      std::memset(&J, 0, sizeof(J));
      J.code = B.d_code; J.off = P.off; J.sorted = B.d_sorted;
      J.lettab = B.d_lettab; J.flagtab = pl.kind == kKindKim ? B.d_kimtab : B.d_flagtab;
      J.A = B.alpha; J.o = P.o; J.e = P.e; J.bias = B.bias; J.thresh = pl.thresh;
      J.mode = P.mode; J.ranks = P.ranks; J.nseq = P.nseq; J.protein = P.protein;
      J.dist_fn = P.dist_fn; J.throws = P.throws;
      J.rb_a = P.nseq / P.ranks; J.rb_b = P.nseq % P.ranks;
      J.blk_mode = key.block; J.col_lo = key.col_lo; J.col_hi = key.col_hi;
      J.out = P.out; J.ld = P.ld; J.mirror = mirror;
      J.scratch = B.d_scratch; J.maxcol = B.maxcol;
      J.rerun = pl.d_rerun; J.rerun_count = pl.d_rerun_count; J.rerun_cap = pl.rerun_cap;
      J.stats = pl.d_stats;
      J.box = B.d_box; J.boxwin = B.d_boxwin; J.box_count = B.d_counts;
      J.box_cap = (int)std::min<long long>(B.box_cap, 0x7fffffff);
      // fork: each bin on its own stream, all after the resets above; join before the rerun
      if (bins_t0 && (e = cudaEventRecord(bins_t0, P.stream)) != cudaSuccess) return e;
      const bool fork = pl.order.size() > 1;
      if (fork && (e = cudaEventRecord(fork_, P.stream)) != cudaSuccess) return e;
      for (size_t x = 0; x < pl.order.size(); x++) {
        const int b = pl.order[x];
        const Bin& bn = pl.bins[b];
        cudaStream_t st = fork ? side_[x] : P.stream;
        if (fork && (e = cudaStreamWaitEvent(st, fork_, 0)) != cudaSuccess) return e;
        J.items = pl.d_items + bn.item_offset;
        J.nitems = (int)bn.items.size();
        J.counter = pl.d_counters + b;
        J.mpad = bn.mpad;
        J.scratch = B.d_scratch + bn.scratch_off;
        J.scratch_words = (long long)(B.scratch_bytes / 4) - (long long)bn.scratch_off;
        J.rowbuf = two ? B.d_rowbuf + bn.rowbuf_off : nullptr;
        J.rowbuf_words = two ? (long long)(B.rowbuf_bytes / 4) - (long long)bn.rowbuf_off : 0;
        if ((e = launch_engine_k(bn.K, pl.kind, J, bn.grid, bn.smem, st)) != cudaSuccess) return e;
        if (fork) {
          if ((e = cudaEventRecord(join_[x], st)) != cudaSuccess) return e;
          if ((e = cudaStreamWaitEvent(P.stream, join_[x], 0)) != cudaSuccess) return e;
        }
      }
      if (bins_t1 && (e = cudaEventRecord(bins_t1, P.stream)) != cudaSuccess) return e;
      J3 = J;
    }
    if (two) {
      // counters of the first pass's best cells from regions around their traceback paths: the
      // register scan and band DPs (swg_box_reg.cuh), then the warp box kernel for the pairs whose
      // region is wider than theirs
      BoxJob X;
      std::memset(&X, 0, sizeof(X));
      X.seq = B.d_code; X.off = P.off;
      X.list = B.d_box; X.count = B.d_counts; X.win = B.d_boxwin;
      X.cls[0] = B.d_cls[0]; X.cls[1] = B.d_cls[1]; X.cls_count = B.d_counts + 2;
      X.out = P.out; X.ld = P.ld; X.mirror = mirror;
      X.lettab = B.d_lettab; X.flagtab = B.d_flagtab; X.A = B.alpha; X.o = P.o; X.e = P.e;
      X.maxlen = B.maxcol;
      X.rerun = pl.d_rerun; X.rerun_count = pl.d_rerun_count; X.rerun_cap = pl.rerun_cap;
      X.stats = pl.d_stats;
      X.list_cap = B.box_cap;
      X.spill = B.d_spill; X.spill_count = B.d_counts + 1;
      X.spill_cap = (int)std::min<long long>(B.spill_cap, 0x7fffffff);
      if (pl.fb) { X.fb = B.d_fb; X.fb_count = B.d_counts + 6; X.fb_cap = B.box_cap; }
      BoxJob Y = X;
      if (opt_.box_reg) {
        if ((e = launch_box_scan(X, P.sms, P.stream)) != cudaSuccess) return e;
        for (int c = 0; c < 4; c++)
          if ((e = launch_box_band(X, c, P.sms, P.stream)) != cudaSuccess) return e;
        Y.list = B.d_spill; Y.count = B.d_counts + 1; Y.list_cap = B.spill_cap;
      }
      // the warp kernel's box has at most kWarpBoxMaxCols columns: a larger S / max S cannot fit
      Y.max_score = kWarpBoxMaxCols * std::max(B.max_s, 0);
      Y.budget = 1 << 16;
      if ((e = launch_box(Y, (int)(B.carry_threads / 128), 128, P.stream)) != cudaSuccess) return e;
      if (pl.fb) {
        // third pass: the give-ups bucketed by query, then the one-pass counter kernel on them
        const int nq = key.row_hi - key.row_lo + 1;
        int* cnt = B.d_fbq;
        int* start = cnt + P.nseq;
        int* fill = start + P.nseq;
        int* cstart = fill + P.nseq;
        int* total = cstart + P.nseq + 1;
        if ((e = cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)nq, P.stream)) != cudaSuccess) return e;
        const int g = std::max(1, P.sms * 4);
        fb_count_kernel<<<g, 256, 0, P.stream>>>(B.d_fb, B.d_counts + 6, B.box_cap, key.row_lo, cnt);
        fb_scan_kernel<<<1, 1024, 0, P.stream>>>(cnt, start, fill, cstart, total, nq, pl.fb_grid);
        fb_scatter_kernel<<<g, 256, 0, P.stream>>>(B.d_fb, B.d_counts + 6, B.box_cap, key.row_lo, start, fill,
                                                   B.d_fbsorted);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        EngineJob F = J3;
        F.fb_cnt = cnt; F.fb_start = start; F.fb_cstart = cstart; F.fb_total = total;
        F.fb_nq = nq; F.fb_lo = key.row_lo;
        F.sorted = B.d_fbsorted;
        F.items = nullptr; F.nitems = 0;
        F.counter = B.d_counts + 7;
        F.mpad = pl.fb_mpad;
        F.scratch = B.d_scratch;
        F.scratch_words = (long long)(B.scratch_bytes / 4);
        F.rowbuf_words = 0;
        F.rowbuf = nullptr;
        F.box = nullptr; F.boxwin = nullptr;
        if ((e = launch_engine_k(kFbK, kKindSw, F, pl.fb_grid, pl.fb_smem, P.stream)) != cudaSuccess) return e;
      }
    }
    // 32-bit lanes: pairs the static guard routed here, those whose 16-bit lanes tripped, or all
    PlainJob R;
    std::memset(&R, 0, sizeof(R));
    R.seq = P.seq; R.off = P.off;
    R.list = pl.d_rerun; R.list_count = pl.d_rerun_count;
    R.npairs = pl.rerun_cap;
    R.out = P.out; R.ld = P.ld; R.out_r0 = 0; R.out_c0 = 0;
    R.mirror = mirror;
    R.scores = P.scores; R.flags = P.flags;
    R.o = P.o; R.e = P.e; R.mode = P.mode; R.protein = P.protein;
    R.dist_fn = P.dist_fn; R.throws = P.throws;
    R.carry = B.d_carry;
    const int grid = (pl.big_count > 0 || two) ? (int)(B.carry_threads / 128) : P.sms;
    return launch_plain_block(R, grid, 128, P.stream);
  }

  // Streams and events of the bins' fork/join, made once on the engine's device.
  int ensure_streams(std::string* msg) {
    if (streams_ok_) return SW_OK;
    if (cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError(); *msg = "event create"; return SW_E_CUDA;
    }
    for (int x = 0; x < kNumK; x++)
      if (cudaStreamCreateWithFlags(&side_[x], cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&join_[x], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError(); *msg = "stream create"; return SW_E_CUDA;
      }
    streams_ok_ = true;
    return SW_OK;
  }
  void release_streams() {
    if (!streams_ok_) return;
    cudaEventDestroy(fork_);
    for (int x = 0; x < kNumK; x++) { cudaStreamDestroy(side_[x]); cudaEventDestroy(join_[x]); }
    streams_ok_ = false;
  }

  EngineOptions opt_;
  bool streams_ok_ = false;
  cudaEvent_t fork_ = nullptr;
  cudaStream_t side_[kNumK] = {};
  cudaEvent_t join_[kNumK] = {};
  std::unique_ptr<Base> base_;
  std::map<PlanKey, std::unique_ptr<Plan>> plans_;
  Plan* last_ = nullptr;
};

// ---- query mode ---------------------------------------------------------------------------------
// Nominal rates of the cost model (GPU seconds of an item): row-padded cells per second of the
// 16-bit lanes at 16 rows per lane, and cells per second of the 32-bit lanes, on B200.
constexpr double kRate16 = 1.45e12;
constexpr double kRate32 = 1.4e11;
constexpr int kQueryChunk = 256;

class QueryRunnerImpl : public QueryRunner {
 public:
  ~QueryRunnerImpl() override {
    cudaFree(d_qtab_); cudaFree(d_qflag_); cudaFree(d_qbsc_); cudaFree(d_qbscf_);
    for (auto& w : wb_) {
      cudaFree(w.d_box); cudaFree(w.d_win); cudaFree(w.d_cls[0]); cudaFree(w.d_cls[1]); cudaFree(w.d_counts);
      cudaFree(w.d_fb); cudaFree(w.d_fbsorted); cudaFree(w.d_fbq); cudaFree(w.d_spill);
      cudaFree(w.d_rowbuf);
      cudaFree(w.d_items); cudaFree(w.d_counters); cudaFree(w.d_stats); cudaFree(w.d_rerun);
      cudaFree(w.d_rerun_count); cudaFreeHost(w.h_items); cudaFreeHost(w.h_rerun); cudaFree(w.d_scratch);
      if (w.fork) cudaEventDestroy(w.fork);
      if (w.plain_done) cudaEventDestroy(w.plain_done);
      for (int x = 0; x < kNumK; x++) {
        if (w.side[x]) cudaStreamDestroy(w.side[x]);
        if (w.join[x]) cudaEventDestroy(w.join[x]);
      }
    }
  }

  int init(const EngineParams& P, std::string* msg) {
    P_ = P;
    int rc = build_base(B_, P, msg);
    if (rc) return rc;
    N_ = P.nseq;
    nw_ = P.mode == kModeNw;
    third_ = P.third_pass != 0;
    // Kimura2 / JukesCantor of SWG-MPI / SWG-MS on letters that fit three profile planes: the
    // 16-bit kernels with two counter words (the batch planner's rule); otherwise 32-bit lanes
    const bool kim = P.dist_fn != 0 && !P.protein;
    kim_ = kim && (P.dist_fn == 1 || P.dist_fn == 2) && !nw_ && B_.alpha > 0 && planes_of(B_.alpha) == 3;
    lanes16_ = !(B_.alpha > kMaxAlpha16 || P.lanes == SW_LANES_32 || B_.alpha == 0 || (kim && !kim_));
    // database chunks in length order
    for (int c0 = 0; c0 < N_; c0 += kQueryChunk) {
      const int c1 = std::min(N_, c0 + kQueryChunk);
      int64_t sum = 0;
      int mx = 0;
      for (int k = c0; k < c1; k++) { sum += B_.len[B_.sorted_h[k]]; mx = std::max(mx, B_.len[B_.sorted_h[k]]); }
      chunk_lo_.push_back(c0); chunk_hi_.push_back(c1); chunk_sum_.push_back(sum); chunk_max_.push_back(mx);
      total_len_ += sum;
    }
    for (auto& w : wb_) {
      if (cudaEventCreateWithFlags(&w.fork, cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&w.plain_done, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError(); *msg = "event create"; return SW_E_CUDA;
      }
      for (int x = 0; x < kNumK; x++)
        if (cudaStreamCreateWithFlags(&w.side[x], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&w.join[x], cudaEventDisableTiming) != cudaSuccess) {
          cudaGetLastError(); *msg = "stream create"; return SW_E_CUDA;
        }
    }
    if (!lanes16_) return SW_OK;
    // query-side tables: any residue byte (rows) against the database letters (columns)
    const int A = B_.alpha, A1 = A + 1;
    int maxS = 0, minS = 0;
    for (int x = 0; x < 127; x++)
      for (int b : B_.letters) {
        const int v = P.h_scores[x * 128 + b];
        maxS = std::max(maxS, v);
        minS = std::min(minS, v);
      }
    if (nw_) {
      // NW lanes hold value + bias with the bias above the all-gap bound of every cell a pass
      // touches: query rows padded by up to 32 x 16 - 1, database columns by up to 63.  The
      // largest bias that still holds the highest score of any pair leaves the most room for long
      // queries; a query beyond that length (nw_qmax_) goes to 32-bit lanes.
      const long bias = 32767L - (long)maxS * (B_.maxcol + 1);
      const long fixed = 3L * P.o + 2L * P.e + (512L + B_.maxcol + 64) * P.e - minS;
      nw_qmax_ = bias > fixed && P.e > 0 ? (int)std::min<long>((bias - fixed) / P.e, 32767) : 0;
      if (nw_qmax_ < 1) { lanes16_ = false; return SW_OK; }
      bias_ = (int)bias;
    } else {
      bias_ = std::max(std::max(P.o + 2 * P.e, -minS), 1);
    }
    max_s_ = maxS;
    thresh_ = 32767 - bias_ - max_s_;
    std::vector<int32_t> qtab((size_t)128 * A1);
    std::vector<uint32_t> qflag((size_t)128 * A1, 0u);
    for (int x = 0; x < 128; x++)
      for (int c = 0; c < A1; c++) {
        int v = nw_ ? 0 : -bias_;  // padding (NW: 0 keeps its values inside the bias's bound)
        uint32_t f = 0;
        if (x != kPadCode && c != A) {
          v = P.h_scores[x * 128 + B_.letters[c]];
          const uint32_t fl = P.h_flags[x * 128 + B_.letters[c]];
          f = kim_ ? ((fl & kFlagCntA) ? 1u : 0u) | ((fl & kFlagCntB) ? 0x10000u : 0u) : fl & kFlagCount;
        }
        qtab[(size_t)x * A1 + c] = v + P.o;
        qflag[(size_t)x * A1 + c] = f;
      }
    if ((rc = upload_vec(&d_qtab_, qtab, msg, "query score table"))) return rc;
    if ((rc = upload_vec(&d_qflag_, qflag, msg, "query flag table"))) return rc;
    // two passes where the engine uses them (the same rule): the score-only kernels, then the box
    // step with a table row per query residue byte
    two_ = !nw_ && !kim_ && std::min(P.o, P.e) >= 2 &&
           (P.two_pass == 2 || (P.two_pass == 1 && P.o >= 3 * max_s_ && P.e >= 3));
    if (two_) {
      std::vector<int32_t> qsc((size_t)128 * A1), qscf((size_t)128 * A1);
      for (int x = 0; x < 128; x++)
        for (int c = 0; c < A1; c++) {
          const bool pad = x == kPadCode || c == A;
          const int v = pad ? kRegPadScore : P.h_scores[x * 128 + B_.letters[c]];
          const uint32_t f = pad ? 0u : (P.h_flags[x * 128 + B_.letters[c]] & kFlagCount);
          qsc[(size_t)x * A1 + c] = v;
          qscf[(size_t)x * A1 + c] = (int32_t)(((uint32_t)v << 8) | f);
        }
      if ((rc = upload_vec(&d_qbsc_, qsc, msg, "query box table"))) return rc;
      if ((rc = upload_vec(&d_qbscf_, qscf, msg, "query band table"))) return rc;
    }
    return SW_OK;
  }

  // The 16-bit kernel kind of this runner's waves.
  int kind() const { return nw_ ? kKindNw : kim_ ? kKindKim : two_ ? kKindScore : kKindSw; }

  int db_count() const override { return N_; }

  int64_t query_cells(int m) const override { return (int64_t)m * total_len_; }

  void plan_query(int slot, int m, std::vector<QueryItem>* items) const override {
    int K = 0, passes = 0;
    bool fits = lanes16_ && (!nw_ || m <= nw_qmax_);
    if (fits) {
      choose_k(m, 0, &K, &passes, false, nullptr, kim_ ? kKimMaxK : 16);
      // a profile beyond shared memory (queries of several thousand residues): 32-bit lanes
      fits = engine_smem(B_.alpha, passes * 32 * K, B_.maxcol, K, kind()) <= 227 * 1024;
    }
    for (size_t c = 0; c < chunk_lo_.size(); c++) {
      QueryItem it;
      it.slot = slot;
      it.c0 = chunk_lo_[c];
      it.c1 = chunk_hi_[c];
      const int cnt = it.c1 - it.c0;
      const int mn = std::min(m, chunk_max_[c]);
      if (fits && (long)max_s_ * (mn + 1) + bias_ <= 32767) {
        it.K = K;
        it.passes = passes;
        it.cost = (double)passes * 32 * K * ((double)chunk_sum_[c] + 31.0 * cnt) * k_weight(K) / 100.0 / kRate16;
      } else {
        // 16-bit lanes cannot hold these scores (or are not available): 32-bit lanes
        it.K = 0;
        it.passes = 0;
        it.cost = (double)std::max(m, 1) * ((double)chunk_sum_[c] + cnt) / kRate32;
      }
      items->push_back(it);
    }
  }

  int enqueue(int buf, const std::vector<QueryItem>& items, const QueryTables& T, cudaStream_t st,
              std::string* msg) override {
    WaveBuf& W = wb_[buf & 1];
    // bins by rows per lane, longest first inside each; 32-bit items become explicit pairs
    std::vector<std::vector<const QueryItem*>> bins(kNumK);
    std::vector<double> bin_cost(kNumK, 0.0);
    size_t n16 = 0, nbig = 0;
    long long pairs16 = 0;
    for (const QueryItem& it : items) {
      if (it.K == 0) { nbig += (size_t)(it.c1 - it.c0); continue; }
      const int b = (int)(std::find(std::begin(kKs), std::end(kKs), it.K) - std::begin(kKs));
      bins[b].push_back(&it);
      bin_cost[b] += it.cost;
      n16++;
      pairs16 += it.c1 - it.c0;
    }
    const size_t rerun_cap = std::max<size_t>(nbig + (size_t)pairs16, 1);
    int rc;
    if ((rc = grow(W, std::max<size_t>(n16, 1), rerun_cap, msg))) return rc;
    size_t big = 0;
    for (const QueryItem& it : items)
      if (it.K == 0)
        for (int k = it.c0; k < it.c1; k++) W.h_rerun[big++] = make_int2(it.slot, B_.sorted_h[k]);
    struct Launch { int K, b, offset, count, mpad, max_passes; };
    std::vector<Launch> ls;
    size_t pos = 0;
    for (int b = 0; b < kNumK; b++) {
      if (bins[b].empty()) continue;
      std::stable_sort(bins[b].begin(), bins[b].end(), [](const QueryItem* x, const QueryItem* y) { return x->cost > y->cost; });
      Launch L{kKs[b], b, (int)pos, (int)bins[b].size(), 0, 0};
      for (const QueryItem* it : bins[b]) {
        W.h_items[pos++] = make_int4(it->slot, it->c0, it->c1, it->passes);
        L.mpad = std::max(L.mpad, it->passes * 32 * L.K);
        L.max_passes = std::max(L.max_passes, it->passes);
      }
      ls.push_back(L);
    }
    std::stable_sort(ls.begin(), ls.end(), [&](const Launch& x, const Launch& y) { return bin_cost[x.b] > bin_cost[y.b]; });
    // per-bin launch shape and scratch (bins run concurrently, each multi-pass bin has its own;
    // two passes: each bin its own rows' bounds too)
    const int A = B_.alpha;
    const int kind = this->kind();
    std::vector<size_t> smem(ls.size()), scr_off(ls.size()), row_off(ls.size());
    std::vector<int> grid(ls.size());
    size_t scr_words = 0, row_words = 0;
    for (size_t x = 0; x < ls.size(); x++) {
      smem[x] = engine_smem(A, ls[x].mpad, B_.maxcol, ls[x].K, kind);
      if (smem[x] > 227 * 1024) { *msg = "query profile exceeds shared memory"; return SW_E_UNSUPPORTED; }
      if (allow_smem_k(ls[x].K, A, kind, smem[x]) != cudaSuccess) { cudaGetLastError(); *msg = "shared memory opt-in"; return SW_E_CUDA; }
      const int occ = std::max(1, occupancy_k(ls[x].K, A, kind, smem[x]));
      grid[x] = std::min(P_.sms * occ, ls[x].count);
      scr_off[x] = scr_words;
      if (ls[x].max_passes > 1)
        scr_words += (size_t)grid[x] * warps_of(ls[x].K, kind) * B_.maxcol * (kim_ ? kScrWordsKim : kScrWords);
      row_off[x] = row_words;
      if (two_) row_words += (size_t)grid[x] * warps_of(ls[x].K, kind) * ls[x].mpad;
    }
    // third pass (two passes): the box step's give-ups on the one-pass 16-bit counter kernel, the
    // wave's longest query in passes of 512 rows, where its profile fits shared memory
    int fb_nq = 0, fb_mpad = 0, fb_grid = 0;
    size_t fb_smem = 0;
    bool fb = false;
    if (two_ && !ls.empty() && third_) {
      int mrows = 0;
      for (const QueryItem& it : items)
        if (it.K) { fb_nq = std::max(fb_nq, it.slot + 1); mrows = std::max(mrows, it.passes * 32 * it.K); }
      fb_mpad = ((mrows + 32 * kFbK - 1) / (32 * kFbK)) * 32 * kFbK;
      fb_smem = engine_smem(A, fb_mpad, B_.maxcol, kFbK, kKindSw);
      fb = fb_nq > 0 && fb_smem <= 227 * 1024 && allow_smem_k(kFbK, A, kKindSw, fb_smem) == cudaSuccess;
      cudaGetLastError();
      if (fb) {
        fb_grid = P_.sms * std::max(1, occupancy_k(kFbK, A, kKindSw, fb_smem));
        scr_words = std::max(scr_words, (size_t)fb_grid * warps_of(kFbK) * B_.maxcol * kScrWords);
      }
    }
    if (two_ && (rc = grow_box(W, std::max<size_t>((size_t)pairs16, 1), std::max<size_t>(row_words * 4, 16), msg))) return rc;
    if (fb && (rc = grow_fbq(W, (size_t)fb_nq, msg))) return rc;
    if (scr_words * 4 > W.scratch_bytes) {
      // the earlier wave of this buffer is done; the other buffer's wave may run (own scratch)
      cudaFree(W.d_scratch);
      W.d_scratch = nullptr;
      W.scratch_bytes = 0;
      if (cudaMalloc(&W.d_scratch, scr_words * 4) != cudaSuccess) { cudaGetLastError(); *msg = "cudaMalloc pass scratch"; return SW_E_OOM; }
      W.scratch_bytes = scr_words * 4;
    }
    cudaError_t e;
    if (n16 && (e = cudaMemcpyAsync(W.d_items, W.h_items, n16 * sizeof(int4), cudaMemcpyHostToDevice, st)) != cudaSuccess) return cuda_err(e, msg);
    if (big && (e = cudaMemcpyAsync(W.d_rerun, W.h_rerun, big * sizeof(int2), cudaMemcpyHostToDevice, st)) != cudaSuccess) return cuda_err(e, msg);
    if ((e = cudaMemsetAsync(W.d_counters, 0, sizeof(int) * kNumK, st)) != cudaSuccess) return cuda_err(e, msg);
    if ((e = cudaMemsetAsync(W.d_stats, 0, sizeof(unsigned long long) * kNumStats, st)) != cudaSuccess) return cuda_err(e, msg);
    if (two_ && (e = cudaMemsetAsync(W.d_counts, 0, sizeof(int) * 8, st)) != cudaSuccess) return cuda_err(e, msg);
    set_int_kernel<<<1, 1, 0, st>>>(W.d_rerun_count, (int)big);
    EngineJob J;
    std::memset(&J, 0, sizeof(J));
    if (!ls.empty()) {
      J.code = B_.d_code; J.off = P_.off; J.sorted = B_.d_sorted;
      J.A = A; J.o = P_.o; J.e = P_.e; J.bias = bias_; J.thresh = thresh_;
      J.mode = P_.mode; J.ranks = 1; J.nseq = N_; J.protein = P_.protein;
      J.dist_fn = P_.dist_fn; J.throws = P_.throws;
      J.maxcol = B_.maxcol;
      J.rerun = W.d_rerun; J.rerun_count = W.d_rerun_count; J.rerun_cap = (int)rerun_cap;
      J.stats = W.d_stats;
      J.qmode = 1; J.qseq = T.qseq; J.qoff = T.qoff; J.qlen = T.qlen; J.qout = T.qout;
      J.qtab = d_qtab_; J.qflag = d_qflag_;
      if (two_) {
        J.box = W.d_box; J.boxwin = W.d_win; J.box_count = W.d_counts;
        J.box_cap = (int)std::min<size_t>(W.box_cap, 0x7fffffff);
      }
      const bool fork = ls.size() > 1;
      if (fork && (e = cudaEventRecord(W.fork, st)) != cudaSuccess) return cuda_err(e, msg);
      for (size_t x = 0; x < ls.size(); x++) {
        cudaStream_t s2 = fork ? W.side[x] : st;
        if (fork && (e = cudaStreamWaitEvent(s2, W.fork, 0)) != cudaSuccess) return cuda_err(e, msg);
        J.items = W.d_items + ls[x].offset;
        J.nitems = ls[x].count;
        J.counter = W.d_counters + ls[x].b;
        J.mpad = ls[x].mpad;
        J.scratch = W.d_scratch + scr_off[x];
        J.scratch_words = (long long)(W.scratch_bytes / 4) - (long long)scr_off[x];
        J.rowbuf = two_ ? W.d_rowbuf + row_off[x] : nullptr;
        J.rowbuf_words = two_ ? (long long)(W.rowbuf_bytes / 4) - (long long)row_off[x] : 0;
        if ((e = launch_engine_k(ls[x].K, kind, J, grid[x], smem[x], s2)) != cudaSuccess) return cuda_err(e, msg);
        if (fork) {
          if ((e = cudaEventRecord(W.join[x], s2)) != cudaSuccess) return cuda_err(e, msg);
          if ((e = cudaStreamWaitEvent(st, W.join[x], 0)) != cudaSuccess) return cuda_err(e, msg);
        }
      }
    }
    if (two_ && !ls.empty()) {
      // the box step of the wave's score records: query residues against database codes, distances
      // to the query rows; pairs it cannot finish go to the 32-bit lanes below
      BoxJob X;
      std::memset(&X, 0, sizeof(X));
      X.seq = B_.d_code; X.off = P_.off;
      X.qseq = T.qseq; X.qoff = T.qoff; X.qout = T.qout; X.qsc = d_qbsc_; X.qscf = d_qbscf_;
      X.list = W.d_box; X.count = W.d_counts; X.win = W.d_win;
      X.cls[0] = W.d_cls[0]; X.cls[1] = W.d_cls[1]; X.cls_count = W.d_counts + 2;
      X.A = A; X.o = P_.o; X.e = P_.e; X.maxlen = B_.maxcol;
      X.rerun = W.d_rerun; X.rerun_count = W.d_rerun_count; X.rerun_cap = (int)rerun_cap;
      X.stats = W.d_stats;
      X.list_cap = (long long)W.box_cap;
      // pairs whose region is wider than the register step's go to the warp box kernel
      X.spill = W.d_spill; X.spill_count = W.d_counts + 1;
      X.spill_cap = (int)std::min<size_t>(W.spill_cap, 0x7fffffff);
      if (fb) { X.fb = W.d_fb; X.fb_count = W.d_counts + 6; X.fb_cap = (long long)W.box_cap; }
      if ((e = launch_box_scan(X, P_.sms, st)) != cudaSuccess) return cuda_err(e, msg);
      for (int c = 0; c < 4; c++)
        if ((e = launch_box_band(X, c, P_.sms, st)) != cudaSuccess) return cuda_err(e, msg);
      BoxJob Y = X;
      Y.list = W.d_spill; Y.count = W.d_counts + 1; Y.list_cap = (long long)W.spill_cap;
      Y.max_score = kWarpBoxMaxCols * std::max(max_s_, 0);
      Y.budget = 1 << 16;
      if ((e = launch_box(Y, (int)(B_.carry_threads / 128), 128, st)) != cudaSuccess) return cuda_err(e, msg);
      if (fb) {
        // the give-ups bucketed by query slot, then the one-pass counter kernel on them
        int* cnt = W.d_fbq;
        int* start = cnt + W.fbq_cap;
        int* fill = start + W.fbq_cap;
        int* cstart = fill + W.fbq_cap;
        int* total = cstart + W.fbq_cap + 1;
        if ((e = cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)fb_nq, st)) != cudaSuccess) return cuda_err(e, msg);
        const int g4 = std::max(1, P_.sms * 4);
        fb_count_kernel<<<g4, 256, 0, st>>>(W.d_fb, W.d_counts + 6, (long long)W.box_cap, 0, cnt);
        fb_scan_kernel<<<1, 1024, 0, st>>>(cnt, start, fill, cstart, total, fb_nq, fb_grid);
        fb_scatter_kernel<<<g4, 256, 0, st>>>(W.d_fb, W.d_counts + 6, (long long)W.box_cap, 0, start, fill,
                                              W.d_fbsorted);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, msg);
        EngineJob F = J;
        F.fb_cnt = cnt; F.fb_start = start; F.fb_cstart = cstart; F.fb_total = total;
        F.fb_nq = fb_nq; F.fb_lo = 0;
        F.sorted = W.d_fbsorted;
        F.items = nullptr; F.nitems = 0;
        F.counter = W.d_counts + 7;
        F.mpad = fb_mpad;
        F.scratch = W.d_scratch;
        F.scratch_words = (long long)(W.scratch_bytes / 4);
        F.rowbuf = nullptr; F.rowbuf_words = 0;
        F.box = nullptr; F.boxwin = nullptr;
        if ((e = launch_engine_k(kFbK, kKindSw, F, fb_grid, fb_smem, st)) != cudaSuccess) return cuda_err(e, msg);
      }
    }
    // 32-bit lanes: pairs routed there by the static guard and 16-bit lanes that tripped
    PlainJob R;
    std::memset(&R, 0, sizeof(R));
    R.seq = P_.seq; R.off = P_.off;
    R.list = W.d_rerun; R.list_count = W.d_rerun_count;
    R.npairs = (long long)rerun_cap;
    R.scores = P_.scores; R.flags = P_.flags;
    R.o = P_.o; R.e = P_.e; R.mode = P_.mode; R.protein = P_.protein;
    R.dist_fn = P_.dist_fn; R.throws = P_.throws;
    R.carry = B_.d_carry;
    R.qseq = T.qseq; R.qoff = T.qoff; R.qlen = T.qlen; R.qout = T.qout;
    const int g = (big > 0 || two_) ? (int)(B_.carry_threads / 128) : P_.sms;
    // the 32-bit lanes' scratch is shared: after the other buffer's 32-bit kernel
    WaveBuf& other = wb_[(buf & 1) ^ 1];
    if (other.plain_used && (e = cudaStreamWaitEvent(st, other.plain_done, 0)) != cudaSuccess) return cuda_err(e, msg);
    if ((e = launch_plain_block(R, g, 128, st)) != cudaSuccess) return cuda_err(e, msg);
    if ((e = cudaEventRecord(W.plain_done, st)) != cudaSuccess) return cuda_err(e, msg);
    W.plain_used = true;
    return SW_OK;
  }

 private:
  struct WaveBuf {
    int4* d_items = nullptr;
    int4* h_items = nullptr;
    size_t cap_items = 0;
    int2* d_rerun = nullptr;
    int2* h_rerun = nullptr;
    size_t cap_rerun = 0;
    int* d_counters = nullptr;
    int* d_rerun_count = nullptr;
    unsigned long long* d_stats = nullptr;
    // waves of the two buffers may run at once: each has its own scratch, streams and events
    uint32_t* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    cudaEvent_t fork = nullptr, plain_done = nullptr;
    bool plain_used = false;
    cudaStream_t side[kNumK] = {};
    cudaEvent_t join[kNumK] = {};
    // two passes: the score kernels' box records, threshold windows and rows' bounds, the band
    // classes, and the counts ([0] records, [1] spilled, [2..5] classes)
    int4* d_box = nullptr;
    uint32_t* d_win = nullptr;
    int* d_cls[2] = {nullptr, nullptr};
    int* d_counts = nullptr;
    size_t box_cap = 0;
    uint32_t* d_rowbuf = nullptr;
    size_t rowbuf_bytes = 0;
    // third pass: the give-ups (box_cap entries), their partners bucketed by query slot, and per
    // slot counts / offsets / fill (fbq_cap each), chunk offsets (fbq_cap + 1), the chunk count
    // and the chunk size
    int2* d_fb = nullptr;
    int* d_fbsorted = nullptr;
    int* d_fbq = nullptr;
    size_t fbq_cap = 0;
    // the register step's spills for the warp box kernel
    int4* d_spill = nullptr;
    size_t spill_cap = 0;
  };

  int grow_fbq(WaveBuf& W, size_t nq, std::string* msg) {
    if (nq <= W.fbq_cap) return SW_OK;
    const size_t cap = std::max(nq, W.fbq_cap * 2);
    cudaFree(W.d_fbq);
    W.d_fbq = nullptr;
    W.fbq_cap = 0;
    if (cudaMalloc(&W.d_fbq, sizeof(int) * (4 * cap + 3)) != cudaSuccess) {
      cudaGetLastError(); *msg = "cudaMalloc wave third-pass counts"; return SW_E_OOM;
    }
    W.fbq_cap = cap;
    return SW_OK;
  }

  // Two-pass buffers of a wave buffer for `pairs` box records and `rowbuf` bytes of rows' bounds.
  int grow_box(WaveBuf& W, size_t pairs, size_t rowbuf, std::string* msg) {
    if (!W.d_counts && cudaMalloc(&W.d_counts, sizeof(int) * 8) != cudaSuccess) {
      cudaGetLastError(); W.d_counts = nullptr; *msg = "cudaMalloc wave box counts"; return SW_E_OOM;
    }
    if (pairs > W.box_cap) {
      const size_t cap = std::max(pairs, W.box_cap * 2);
      cudaFree(W.d_box); cudaFree(W.d_win); cudaFree(W.d_cls[0]); cudaFree(W.d_cls[1]);
      cudaFree(W.d_fb); cudaFree(W.d_fbsorted); cudaFree(W.d_spill);
      W.d_box = nullptr; W.d_win = nullptr; W.d_cls[0] = W.d_cls[1] = nullptr; W.box_cap = 0;
      W.d_fb = nullptr; W.d_fbsorted = nullptr; W.d_spill = nullptr; W.spill_cap = 0;
      const size_t nspill = std::max<size_t>(cap / 16, 1 << 16);
      if (cudaMalloc(&W.d_spill, sizeof(int4) * nspill) != cudaSuccess ||
          cudaMalloc(&W.d_box, sizeof(int4) * cap) != cudaSuccess ||
          cudaMalloc(&W.d_fb, sizeof(int2) * cap) != cudaSuccess ||
          cudaMalloc(&W.d_fbsorted, sizeof(int) * cap) != cudaSuccess ||
          cudaMalloc(&W.d_win, sizeof(uint32_t) * kRegWinWords * cap) != cudaSuccess ||
          cudaMalloc(&W.d_cls[0], sizeof(int) * cap) != cudaSuccess ||
          cudaMalloc(&W.d_cls[1], sizeof(int) * cap) != cudaSuccess) {
        cudaGetLastError(); *msg = "cudaMalloc wave box lists"; return SW_E_OOM;
      }
      W.box_cap = cap;
      W.spill_cap = nspill;
    }
    if (rowbuf > W.rowbuf_bytes) {
      cudaFree(W.d_rowbuf);
      W.d_rowbuf = nullptr; W.rowbuf_bytes = 0;
      if (cudaMalloc(&W.d_rowbuf, rowbuf) != cudaSuccess) { cudaGetLastError(); *msg = "cudaMalloc wave row bounds"; return SW_E_OOM; }
      W.rowbuf_bytes = rowbuf;
    }
    return SW_OK;
  }

  static int cuda_err(cudaError_t e, std::string* msg) {
    *msg = std::string("query wave: ") + cudaGetErrorString(e);
    return SW_E_CUDA;
  }

  // Wave buffers grow geometrically; a buffer is only regrown when its earlier wave is done.
  int grow(WaveBuf& W, size_t items, size_t rerun, std::string* msg) {
    if (!W.d_counters) {
      if (cudaMalloc(&W.d_counters, sizeof(int) * kNumK) != cudaSuccess ||
          cudaMalloc(&W.d_rerun_count, sizeof(int)) != cudaSuccess ||
          cudaMalloc(&W.d_stats, sizeof(unsigned long long) * kNumStats) != cudaSuccess) {
        cudaGetLastError(); *msg = "cudaMalloc wave counters"; return SW_E_OOM;
      }
    }
    if (items > W.cap_items) {
      const size_t cap = std::max(items, W.cap_items * 2);
      cudaFree(W.d_items); cudaFreeHost(W.h_items);
      W.d_items = nullptr; W.h_items = nullptr; W.cap_items = 0;
      if (cudaMalloc(&W.d_items, cap * sizeof(int4)) != cudaSuccess ||
          cudaMallocHost(&W.h_items, cap * sizeof(int4)) != cudaSuccess) {
        cudaGetLastError(); *msg = "wave item buffers"; return SW_E_OOM;
      }
      W.cap_items = cap;
    }
    if (rerun > W.cap_rerun) {
      const size_t cap = std::max(rerun, W.cap_rerun * 2);
      cudaFree(W.d_rerun); cudaFreeHost(W.h_rerun);
      W.d_rerun = nullptr; W.h_rerun = nullptr; W.cap_rerun = 0;
      if (cudaMalloc(&W.d_rerun, cap * sizeof(int2)) != cudaSuccess ||
          cudaMallocHost(&W.h_rerun, cap * sizeof(int2)) != cudaSuccess) {
        cudaGetLastError(); *msg = "wave pair buffers"; return SW_E_OOM;
      }
      W.cap_rerun = cap;
    }
    return SW_OK;
  }

  EngineParams P_;
  Base B_;
  int N_ = 0;
  bool lanes16_ = false;
  int bias_ = 1, max_s_ = 0, thresh_ = 0;
  int64_t total_len_ = 0;
  std::vector<int> chunk_lo_, chunk_hi_, chunk_max_;
  std::vector<int64_t> chunk_sum_;
  int32_t* d_qtab_ = nullptr;
  uint32_t* d_qflag_ = nullptr;
  bool two_ = false;          // SW-Gotoh with gap costs that suit the box step: two passes
  bool nw_ = false;           // global alignment (the NW kernels)
  bool kim_ = false;          // Kimura2 / JukesCantor on 16-bit lanes (two counter words)
  bool third_ = true;         // two passes: the box step's give-ups on 16-bit lanes (third pass)
  int nw_qmax_ = 0;           // NW: longest query the 16-bit lanes' bias covers
  int32_t* d_qbsc_ = nullptr;   // [128 * (A+1)] box step tables (query residue byte x database code)
  int32_t* d_qbscf_ = nullptr;
  WaveBuf wb_[2];
};

}  // namespace

Engine* Engine::create() { return new (std::nothrow) EngineImpl(); }

QueryRunner* QueryRunner::create(const EngineParams& db, std::string* msg, int* rc) {
  QueryRunnerImpl* q = new (std::nothrow) QueryRunnerImpl();
  if (!q) { *rc = SW_E_OOM; *msg = "query runner"; return nullptr; }
  if ((*rc = q->init(db, msg))) { delete q; return nullptr; }
  return q;
}

}  // namespace swg
