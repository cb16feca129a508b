/*
 * swgb200.h - C ABI of the B200 all-pairs alignment -> distance engine.
 *
 * The engine replaces the per-pair aligner calls inside the reference's block handlers
 * (DSC-SPIDAL/csharp, SalsaTPL/) with CUDA kernels for sm_100a.  Every entry point takes plain
 * pointers and sizes, returns an int status (SW_OK = 0) and never throws; sw_last_error() gives
 * the text of the last failure on a context.  A context is bound to one CUDA device and one
 * stream, is not re-entrant, and distinct contexts may be used from distinct threads.
 *
 * Sequences are byte strings (the upper-cased residue characters, as the reference's FASTA
 * parser produces them: Salsa.CoreTPL/Bio/IO/Parser.cs:140-144).  Scores index the 128 x 128
 * substitution table by those bytes, as ScoringMatrix.Scores[char, char] does
 * (Salsa.CoreTPL/Bio/Algorithms/ScoringMatrix.cs:34, :130-143).
 */
#ifndef SWGB200_H
#define SWGB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference raises exceptions; none cross this boundary) ------------- */
#define SW_OK 0
#define SW_E_ARG 1          /* bad argument (null pointer, range outside the uploaded set, ...) */
#define SW_E_OOM 2          /* device or host allocation failed */
#define SW_E_CUDA 3         /* a CUDA runtime call failed */
#define SW_E_TIMEOUT 4      /* a bounded device-side wait ran out */
#define SW_E_UNSUPPORTED 5  /* configuration the exact integer kernels cannot reproduce */
#define SW_E_STATE 6        /* call order (e.g. compute before sequences were uploaded) */
#define SW_E_IO 7           /* file could not be read or written */
#define SW_E_THROWS 8       /* the reference would throw for this input (JukesCantor log(0)) */

/* AlignmentType (Salsa.CoreTPL/Bio/Algorithms/AlignmentType.cs:3-7) */
#define SW_PROTEIN 0
#define SW_NUCLEIC 1

/* DistanceFunctionType (AlignmentType.cs:9-15) */
#define SW_DIST_PERCENT_IDENTITY 0
#define SW_DIST_KIMURA2 1
#define SW_DIST_JUKES_CANTOR 2
#define SW_DIST_MIN_MAX_NORM_SCORE 3  /* SWG-MS and NW: from the alignment score and the self scores */

/* Which reference application's semantics a context reproduces. */
#define SW_MODE_SWG_MPI 0 /* Salsa.SmithWatermanMPI: NAligner SW-Gotoh, diagonal blocks j < i */
#define SW_MODE_SWG_MS 1  /* Salsa.SmithWatermanMS: SW-Gotoh, full blocks, MBF distance rules */
#define SW_MODE_NW 2      /* Salsa.NeedlemanWunschTPL: global affine alignment, trimmed identity */

/* Score lane width policy. */
#define SW_LANES_AUTO 0   /* 16-bit packed lanes where a pair provably fits, else 32-bit */
#define SW_LANES_32 32    /* 32-bit lanes only */
#define SW_LANES_16 16    /* 16-bit packed lanes; a pair whose scores could leave int16 reruns in 32-bit */

typedef struct sw_ctx sw_ctx;

typedef struct {
  int32_t mode;           /* SW_MODE_* */
  int32_t alignment_type; /* SW_NUCLEIC or SW_PROTEIN (selects identity vs similarity) */
  int32_t distance_fn;    /* SW_DIST_* */
  float gap_open;         /* positive cost of a gap's first column (GapOpenPenalty) */
  float gap_extension;    /* positive cost of each further column (GapExtensionPenalty) */
  int16_t scores[128][128]; /* substitution table indexed by residue bytes */
  int32_t device;         /* CUDA device ordinal */
  int32_t lanes;          /* SW_LANES_* */
} sw_config;

/* One pair's alignment summary: the PairwiseAlignment fields the reference's distance
 * functions read (Salsa.CoreTPL/Bio/Algorithms/Alignment.cs:124-195). */
typedef struct {
  float score;        /* PairwiseAlignment.Score; -inf for an empty input (Cell.cs:43) */
  int32_t end1, end2; /* traceback start cell (Cell.Row, Cell.Column); SW only */
  int32_t start1, start2; /* PairwiseAlignment.Start1/Start2 */
  int32_t identity;   /* identical columns */
  int32_t similarity; /* identical or positive-score columns (NAligner rule) */
  int32_t gaps;       /* gap columns */
  int32_t length;     /* aligned columns (Sequence1.Length) */
  int16_t distance;   /* the context's Int16 distance for this pair */
  int16_t reserved;
} sw_pair_result;

/* ---- context ---------------------------------------------------------------------------- */
/* Replaces the handler's ambient configuration: the static fields _gapOpen, _gapExtension,
 * _scoringMatrixName, _alignmentType and _distanceFunction that ComputeBlock reads
 * (Salsa.SmithWatermanMPI/Program.cs:58-62, :206-207; Salsa.SmithWatermanMS/Program.cs:275-276;
 * Salsa.NeedlemanWunschTPL/Program.cs:210-213).  Non-integer penalties are SW_E_UNSUPPORTED:
 * the reference's float DP is exact only on integers, which the integer kernels reproduce.
 * distance_fn applies to nucleic input (protein uses PercentSimilarity, as the reference does):
 * Kimura2 / JukesCantor in every mode (SWG-MS and NW cap them at 10, as their Program.cs does),
 * MinMaxNormScore in SWG-MS and NW (SWG-MPI's ComputeDistance has no case for it, so its
 * distances are 0, as the reference's are). */
int sw_create(const sw_config* cfg, sw_ctx** out);
int sw_destroy(sw_ctx* ctx);
const char* sw_last_error(const sw_ctx* ctx);
const char* sw_version(void);

/* Replaces the parsed FASTA list _sequences (Salsa.SmithWatermanMPI/Program.cs:94-95): the
 * sequences stay resident on the device for every later call.  concat holds all residues,
 * sequence k is concat[offsets[k] .. offsets[k+1]).  Lengths up to 32767.  A set with the same
 * lengths and the same residue letters as the resident one replaces its residues in place and keeps
 * the engine's work plans and captured graphs (they depend on the lengths and letters only). */
int sw_upload_sequences(sw_ctx* ctx, const uint8_t* concat, const int64_t* offsets, int32_t count);

/* ---- the block handler (drop-in) ---------------------------------------------------------- */
/* Replaces ComputeBlockHandler / ComputeBlock:
 *   Salsa.SmithWatermanMPI/Program.cs:203-257 (delegate :561),
 *   Salsa.SmithWatermanMS/Program.cs:265-387  (delegate :1018),
 *   Salsa.NeedlemanWunschTPL/Program.cs:206-267 (delegate :977).
 * Rows row_start..row_end and columns col_start..col_end are inclusive global sequence indices
 * (Block.RowRange / Block.ColumnRange).  out is the caller's row-major Int16 buffer over the
 * block, element (i, j) at out[(i - row_start) * ld_out + (j - col_start)].  For a diagonal
 * block in SWG-MPI and NW mode only j < i is aligned (s1 = sequence i) and each distance is
 * also written at the mirrored (j, i) position, as `matrix[i, j] = matrix[j, i]` does; SWG-MS
 * mode aligns every (i, j) of the block.  *pairs_computed receives the handler's return value.
 * sw_compute_block copies to host memory and returns when done; sw_compute_block_device writes
 * device memory, is ordered on the context's stream and does not wait. */
int sw_compute_block(sw_ctx* ctx, int32_t row_start, int32_t row_end, int32_t col_start,
                     int32_t col_end, int32_t is_diagonal, int16_t* out, int64_t ld_out,
                     int64_t* pairs_computed);
int sw_compute_block_device(sw_ctx* ctx, int32_t row_start, int32_t row_end, int32_t col_start,
                            int32_t col_end, int32_t is_diagonal, int16_t* d_out, int64_t ld_out,
                            int64_t* pairs_computed);

/* ---- the per-pair aligner ----------------------------------------------------------------- */
/* Replaces SmithWatermanGotoh.Align (Salsa.CoreTPL/Bio/Algorithms/SmithWaterman/
 * SmithWatermanGotoh.cs:52-110) plus the handler's ComputeDistance for that pair
 * (Salsa.SmithWatermanMPI/Program.cs:259-285).  A null sequence pointer with a non-zero length
 * is SW_E_ARG, as Align throws SmithWatermanGotohException for a null sequence (:55-65). */
int sw_align_pair(sw_ctx* ctx, const uint8_t* s1, int32_t m, const uint8_t* s2, int32_t n,
                  sw_pair_result* out);

/* Alignment strings of explicit pairs: what the applications print with WriteAlignments on
 * (Salsa.SmithWatermanMPI/Program.cs:223-246 and WriteAlignment :545-556;
 * Salsa.SmithWatermanMS/Program.cs:682-702; Salsa.NeedlemanWunschTPL/Program.cs:725-735).  Pair k
 * aligns s1 = sequence rows[k] with s2 = sequence cols[k] under the context's mode and penalties;
 * aln1 / aln2 receive the aligned residues ('-' for a gap, as Sequence1 / Sequence2 hold them) at
 * offset offsets[k], results[k].length characters each; offsets has npairs + 1 entries and
 * offsets[k + 1] - offsets[k] must be at least m + n (the longest alignment).  results[k] holds the
 * traceback's fields and the context's Int16 distance for the pair.  A GPU thread per pair keeps one
 * decision byte per DP cell (pairs go in batches of at most 512 MB of such scratch); waits. */
int sw_align_strings(sw_ctx* ctx, const int32_t* rows, const int32_t* cols, int32_t npairs, char* aln1,
                     char* aln2, const int64_t* offsets, sw_pair_result* results);

/* ---- whole-job engine ---------------------------------------------------------------------- */
/* All blocks of one job in one call: the block driver MPIComputeLowerTriangularBlocked.Compute
 * (Salsa.SmithWatermanMPI/Program.cs:618-642) followed by its Scatter (:645-677), which fills
 * the mirrored half, for `ranks` = the MPI world size whose pair orientation is reproduced
 * (checkerboard rule :628-639; ranks = 1 aligns (s_i, s_j) for every i > j).  SWG-MS mode
 * fills every (i, j).  Work is length-binned and scheduled by a persistent kernel from a device
 * work queue; the launch sequence is captured in a CUDA graph and replayed on later calls.
 * d_out is a device N x N row-major Int16 matrix (leading dimension ld_out); the call is
 * ordered on the context's stream and does not wait.  *pairs receives the number of aligned
 * pairs and *cells the DP cells (sum of m*n). */
int sw_all_pairs_device(sw_ctx* ctx, int32_t ranks, int16_t* d_out, int64_t ld_out,
                        int64_t* pairs, int64_t* cells);
/* Host-memory variant: uploads nothing new, copies the N x N result to out and waits. */
int sw_all_pairs(sw_ctx* ctx, int32_t ranks, int16_t* out, int64_t ld_out, int64_t* pairs,
                 int64_t* cells);
/* Pairs whose 16-bit lanes tripped the saturation check and were rerun in 32-bit lanes by the
 * last engine call (diagnostic). */
int sw_last_rerun_count(const sw_ctx* ctx, int64_t* count);
/* Waits for all work on the context's stream. */
int sw_synchronize(sw_ctx* ctx);

/* One rank's share of the job, for one process per GPU: the pairs that rank `rank` of a
 * `world_size`-rank job aligns in MPIComputeLowerTriangularBlocked.Compute (its row block r,
 * diagonal block lower triangle and the checkerboard half of the off-diagonal blocks,
 * Salsa.SmithWatermanMPI/Program.cs:618-642), through the same engine as sw_all_pairs_device.
 * Distances land at (i, j) and, for the symmetric modes, at the mirrored (j, i), so the
 * entries of all ranks are disjoint and sum to the full matrix (the exchange Scatter and
 * WriteFullMatrixOnRank0 do, :645-677 and :786-888).  d_out is a device N x N matrix whose
 * entries this rank does not own are left unchanged; the call is ordered on the context's
 * stream and does not wait. */
int sw_compute_rank_blocks(sw_ctx* ctx, int32_t rank, int32_t world_size, int16_t* d_out,
                           int64_t ld_out, int64_t* pairs);

/* Rows row_start..row_end of a one-rank run: every pair (i, j) with j < i and i in the rows,
 * s1 = sequence i, written at (i, j) and at the mirrored (j, i) of the device N x N matrix d_out
 * (the distances of sw_all_pairs_device with ranks = 1, whatever the rows).  A process's share of a
 * partition of the job into contiguous rows of about equal DP cells; no reference counterpart (the
 * reference partitions by count, sw_compute_rank_blocks).  SWG-MPI and NW; SWG-MS, which aligns
 * both orientations of a pair, is SW_E_UNSUPPORTED.  row_start = row_end + 1: no rows.  Ordered on
 * the context's stream; does not wait. */
int sw_compute_rows(sw_ctx* ctx, int32_t row_start, int32_t row_end, int16_t* d_out, int64_t ld_out,
                    int64_t* pairs);

/* Engine knobs: "stream" (a caller's cudaStream_t as an integer, 0 = the context's own; later
 * calls are ordered on it), "int16_threshold" (best score above which a 16-bit lane is redone in 32-bit
 * lanes; -1 restores the value derived from the lane range), "use_graph" (0/1), "chunk"
 * (database entries per work item, 32..1024; 0, the default: 1024 for 8,192 sequences or more, else
 * 512), "rows_per_lane" (0 = chosen per query, else an even number 4..16),
 * "plan_only" (1: engine calls build their work plans and graphs but launch nothing; 0: run),
 * "two_pass" (SW-Gotoh: a score-only pass, then each pair's counters from the neighbourhood of
 * its best cell; 1, the default: where open >= 3 x the largest substitution score and extend >= 3,
 * the gap costs with which that neighbourhood stays small; 2: whenever open and extend >= 2; 0:
 * never, the one-pass counter kernels), "box_reg" (two passes: 1, the default, finds each pair's
 * counters with one thread per pair and the DP rows in registers, handing pairs whose alignment
 * region is wider to the warp-per-pair box kernel; 0: the warp-per-pair kernel for every pair),
 * "third_pass" (two passes: 1, the default, redoes the pairs the box step cannot finish with the
 * one-pass 16-bit counter kernel, grouped by query; 0: with the 32-bit lanes), "block_engine"
 * (block handler: 1, the default, the batched engine for blocks of at least 4,096 pairs and the
 * one-launch plain kernel below; 2: the engine for every block; 0: the plain kernel for every
 * block).  Every knob gives the same distances.  Unknown keys are SW_E_ARG. */
int sw_set_option(sw_ctx* ctx, const char* key, int64_t value);

/* Autotuner (no reference counterpart; the reference has one aligner loop): times every
 * rows-per-lane choice of the 16-bit engine (4, 6, ..., 16) forced on a sample of this context's
 * queries (the last ones, each against every earlier sequence; their distances are written to
 * d_out, an N x N device matrix), each choice on the sampled queries it would serve in one pass,
 * and installs the measured cost per row if the whole sample then runs faster than with the
 * current costs, so later jobs choose the tile shape per query from this device and this length
 * mix.  weights (optional) receives the installed costs (100 = the cheapest), all 0 when the
 * current costs were kept. */
int sw_autotune(sw_ctx* ctx, int16_t* d_out, int64_t ld_out, int32_t weights[7]);

/* Counters of the last engine call: "launches" (kernels it enqueued), "pairs", "cells",
 * "bins" (rows-per-lane classes used), "alphabet" (distinct residue bytes), "planned_items",
 * and, after waiting for the device, "items" (work items taken), "lane16_pairs" (pairs finished
 * in 16-bit lanes), "tripped" (16-bit lanes handed to 32-bit lanes), "box_spilled" (two-pass pairs
 * the register box step handed to the warp box kernel), "box_fallbacks" (two-pass pairs the box
 * step could not finish) and "box_third_pass" (those of them redone by the one-pass 16-bit counter
 * kernel; the rest go to 32-bit lanes) and "kernel_error" (0, or the first work item or pair the
 * engine kernels' bounds self-checks rejected and skipped: site << 48 | index; the host-output
 * calls return SW_E_CUDA when it is set).  Unknown keys are SW_E_ARG. */
int sw_query(sw_ctx* ctx, const char* key, int64_t* value);

/* ---- block handler without device allocation ------------------------------------------------ */
/* No counterpart in the reference: this entry point serves callers that cannot allocate device
 * memory (a host that gives all GPU memory to its own pool allocator, a plug-in whose process
 * has a fixed device-memory budget).  It aligns the pairs of one block like
 * sw_compute_block_device, with the same ranges, orientation and mirror rule, in all three
 * modes, with PercentIdentity for nucleic input and PercentSimilarity for protein (nucleic
 * Kimura2 / JukesCantor / MinMaxNormScore are SW_E_UNSUPPORTED here; distance_fn outside 0..3 is
 * SW_E_ARG).  It
 * needs no context: the configuration comes in cfg, the residues and offsets
 * (sw_upload_sequences' layout: d_residues holds d_offsets[count] bytes) and the output are the
 * caller's device buffers, and the work is ordered on `stream` (a cudaStream_t of cfg->device,
 * NULL = the legacy default stream).  The call runs on cfg->device, made current for the call;
 * the caller's current device is current again when it returns.  Buffers that are not
 * cfg->device's memory are SW_E_ARG.  It calls no cudaMalloc or cudaFree: the kernels' scratch is
 * a 64 MiB array in the library's device image, present on every GPU that loads the library
 * until the process exits.  Sequences up to 16,383 residues: a longer one in the block returns
 * SW_E_UNSUPPORTED before the alignment kernel is launched.  The first call on a device looks up
 * that array's address with the device current; make that first call before any stream capture.
 * Calls share the array: calls whose kernels overlap on the GPU race and must be ordered by the
 * caller.  The call waits for its input check (one small kernel over the block's sequences and a
 * copy of its two status words) and does not wait for the alignment kernel. */
int sw_compute_block_static(const sw_config* cfg, const uint8_t* d_residues,
                            const int64_t* d_offsets, int32_t count, int32_t row_start,
                            int32_t row_end, int32_t col_start, int32_t col_end,
                            int32_t is_diagonal, int16_t* d_out, int64_t ld_out,
                            int64_t* pairs_computed, void* stream);

/* ---- serving: query batches against a device-resident database --------------------------- */
/* No single reference call: the reference aligns one sequence set against itself.  Here the
 * sequences uploaded with sw_upload_sequences form the database, and a job is a batch of queries
 * each aligned (query = s1, database entry = s2, every entry) with the context's mode, distance
 * rule and penalties, as the MS block handler aligns one row sequence against a column range
 * (Salsa.SmithWatermanMS/Program.cs:341-375).  Jobs run asynchronously on one host scheduler
 * thread per context: a job is admitted once query slots, query-arena bytes and device memory
 * for its result are free ("serve_slots", "serve_arena_mb", "serve_memory_mb"), and every wave
 * of kernels ("serve_wave_us" of estimated GPU time) takes a fair share of the work items of
 * every admitted job, so jobs that arrive while others run join the next wave.  The options are
 * read when the first job of a database is submitted. */
typedef struct {
  int32_t status;   /* SW_OK, or the error that ended the job */
  int32_t queries;
  int64_t pairs;    /* queries x database entries */
  int64_t cells;    /* sum of query length x entry length */
  double submit_s;  /* the scheduler's clock (seconds since it started) at submission, */
  double admit_s;   /* at admission, */
  double done_s;    /* and when the result was in the caller's buffer */
  int32_t waves;    /* kernel waves the job's work took part in */
  int32_t reserved;
} sw_job_info;

typedef struct {
  int64_t submitted, completed, waves, cells;
  int32_t active;      /* jobs admitted and not yet complete */
  int32_t pending;     /* jobs waiting for admission */
  int32_t max_active;  /* the most jobs admitted at once so far */
  int32_t reserved;
} sw_serve_counters;

/* Submits nq queries (concatenated residues, nq + 1 offsets).  The queries are copied before the
 * call returns; out (host, nq x ld_out Int16, ld_out >= database count) must stay valid until
 * sw_poll reports the job done.  out[i * ld_out + j] = distance(align(query i, entry j)). */
int sw_submit_job(sw_ctx* ctx, const uint8_t* q_concat, const int64_t* q_offsets, int32_t nq,
                  int16_t* out, int64_t ld_out, int64_t* ticket);
/* Waits up to timeout_ms (0 = just look) for the job; done = 1 once out holds every distance.
 * info (optional) is filled when done; a ticket is forgotten after it was reported done. */
int sw_poll(sw_ctx* ctx, int64_t ticket, int32_t timeout_ms, int32_t* done, sw_job_info* info);
int sw_serve_stats(sw_ctx* ctx, sw_serve_counters* stats);
/* Waits for every submitted job, then stops the scheduler (the next submit starts it again). */
int sw_serve_drain(sw_ctx* ctx);

/* ---- host-side library (formats the reference reads and writes) --------------------------- */
/* ScoringMatrix.Load (Salsa.CoreTPL/Bio/Algorithms/ScoringMatrix.cs:145-196) over the matrix
 * text (header of column letters, then one "<letter> <scores...>" line per row; '#' comment
 * lines first).  Letters absent from the header score 0.  Non-integer entries are
 * SW_E_UNSUPPORTED. */
int sw_parse_scoring_matrix(const char* text, int64_t text_len, int16_t out[128][128]);
/* The matrices the reference embeds that the engine ships built in: "EDNAFULL", "BLOSUM62",
 * "IDENTITY" and "MATCH" (the reference's Matrices/ resources of those names). */
int sw_builtin_scoring_matrix(const char* name, int16_t out[128][128]);

/* FastaSequenceParser (Salsa.CoreTPL/Bio/IO/FastaRecord.cs:112-118, Parser.cs:123-180):
 * records start at '>', the label is the trimmed rest of that line, residue lines are trimmed,
 * upper-cased and concatenated.  Two-phase: call with concat/offsets NULL to get the sizes. */
int sw_parse_fasta(const char* text, int64_t text_len, uint8_t* concat, int64_t* offsets,
                   int32_t* count, int64_t* residues);

/* RangePartitioner.Partition (Salsa.CoreTPL/RangePartitioner.cs:17-55): starts/ends receive
 * the inclusive ranges; the first length % parts ranges get one extra element. */
int sw_partition_ranges(int32_t start, int32_t length, int32_t parts, int32_t* starts,
                        int32_t* ends);

/* The computing rank of block (r, c) under the SWG-MPI checkerboard (Program.cs:628-639):
 * returns 1 if rank r computes it, else 0. */
int sw_block_is_computed(int32_t r, int32_t c);

/* Full matrix writer: raw row-major little-endian Int16, no header, as WriteFullMatrixOnRank0
 * (Salsa.SmithWatermanMPI/Program.cs:786-888) and MatrixBinaryWriter.Write(Matrix<short>)
 * (Salsa.CoreTPL/Blas/MatrixBinaryWriter.cs:73-92) produce. */
int sw_write_full_matrix(const char* path, const int16_t* m, int64_t rows, int64_t cols,
                         int64_t ld);

/* SWG-MS block file {BlockDir}/{rank}-{cb}.bin (Salsa.SmithWatermanMS/Program.cs:1081-1160):
 * header (u16-length-prefixed ASCII project, u16 rank, system, fasta names, u16 row/col block
 * numbers, u32 row/col range bounds, four length-prefixed sequence IDs) then the block's Int16
 * values row-major. */
typedef struct {
  const char* project;
  const char* system;
  const char* fasta;
  int32_t rank;
  int32_t row_block, col_block;
  int32_t row_start, row_end, col_start, col_end;
  const char* row_start_id;
  const char* row_end_id;
  const char* col_start_id;
  const char* col_end_id;
} sw_ms_block_header;
int sw_write_ms_block(const char* path, const sw_ms_block_header* h, const int16_t* values,
                      int64_t ld);
/* Reads one block file back (two-phase like sw_parse_fasta for the values). */
int sw_read_ms_block_dims(const char* path, int32_t* rank, int32_t* row_block, int32_t* col_block,
                          int32_t* row_start, int32_t* row_end, int32_t* col_start,
                          int32_t* col_end);
int sw_read_ms_block_values(const char* path, int16_t* values, int64_t ld);

/* ---- measurement ----------------------------------------------------------------------------- */
/* Integer-pipe peak on this device: lane-ops per second of a 2-input integer max (the op the
 * cell update is made of), measured by a calibration kernel.  Denominator of the roofline. */
int sw_measure_int_peak(int32_t device, double* max_ops_per_s, double* add_ops_per_s);

#ifdef __cplusplus
}
#endif
#endif /* SWGB200_H */
