// C-ABI implementation: context lifetime, validation, device residency and dispatch.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "../../include/swgb200.h"
#include "swg_log.cuh"
#include "swg_device.cuh"
#include "swg_engine.h"
#include "swg_serve.h"
#include "swg_internal.h"

struct sw_ctx {
  sw_config cfg;
  int o = 0, e = 0;
  cudaStream_t stream = nullptr;
  int sms = 0;
  std::string err;
  // sequences
  uint8_t* d_seq = nullptr;
  int64_t* d_off = nullptr;
  std::vector<int64_t> h_off;
  std::vector<uint8_t> h_seq;
  int32_t nseq = 0;
  int maxlen = 0;
  // tables
  int16_t* d_scores = nullptr;
  uint8_t* d_flags = nullptr;
  int16_t h_scores[128][128];
  uint8_t h_flags[128][128];
  int max_abs_score = 0, max_score = 0;
  // scratch
  void* d_carry = nullptr;
  size_t carry_bytes = 0;
  int16_t* d_stage = nullptr;
  size_t stage_bytes = 0;
  swg::Engine* engine = nullptr;
  int64_t last_reruns = 0;
  cudaStream_t own_stream = nullptr;  // the context's stream while a caller's stream is in use
  int64_t last_pairs = 0, last_cells = 0;
  int* d_throws = nullptr;  // set by a SWG-MPI JukesCantor pair whose log argument is <= 0
  int block_engine = 1;     // block handler: 1 engine for large blocks, 2 always, 0 plain kernel only
  uint64_t letters[2] = {0, 0};  // residue bytes present in the uploaded set
  // serving (query batches against the uploaded sequences)
  swg::Server* server = nullptr;
  swg::ServeOptions serve_opt;
};

namespace {

int fail(sw_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_fail(sw_ctx* c, cudaError_t e, const char* what) {
  return fail(c, SW_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call, what)                              \
  do {                                              \
    cudaError_t _e = (call);                        \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, what); \
  } while (0)

int ensure(sw_ctx* ctx, void** p, size_t* have, size_t need, const char* what) {
  if (*have >= need && *p) return SW_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  cudaError_t e = cudaMalloc(p, need);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(ctx, SW_E_OOM, std::string("cudaMalloc failed for ") + what);
  }
  *have = need;
  return SW_OK;
}

// Column flags: which (c1, c2) pairs count toward the distance's numerator.
void build_flags(sw_ctx* c) {
  const int mode = c->cfg.mode;
  const bool protein = c->cfg.alignment_type == SW_PROTEIN;
  for (int a = 0; a < 128; a++)
    for (int b = 0; b < 128; b++) {
      const int s = c->h_scores[a][b];
      uint32_t f = 0;
      if (a == b) f |= swg::kFlagIdent;
      if (a == b || s > 0) f |= swg::kFlagSimNA;
      bool count;
      if (!protein) {
        count = (a == b);                             // identity (all three apps)
        // Kimura2 / JukesCantor read the aligned strings (Alignment.cs:254-348)
        const bool transition = (a == 'A' && b == 'G') || (a == 'G' && b == 'A') ||
                                (a == 'C' && b == 'T') || (a == 'T' && b == 'C');
        if (c->cfg.distance_fn == SW_DIST_KIMURA2) {
          if (transition) f |= swg::kFlagCntA;
          else if (a != b) f |= swg::kFlagCntB;
        } else if (c->cfg.distance_fn == SW_DIST_JUKES_CANTOR) {
          if (a == b) f |= swg::kFlagCntA;
        }
      }
      else if (mode == SW_MODE_SWG_MPI) count = (a == b || s > 0);  // NAligner similarity
      else count = (s > 0);                           // MBF: non-gap pairs with positive score
      if (count) f |= swg::kFlagCount;
      if (a == swg::kPadCode || b == swg::kPadCode) f = 0;
      c->h_flags[a][b] = (uint8_t)f;
    }
}

}  // namespace

extern "C" {

const char* sw_version(void) { return "swgb200 1.0 (sm_100a)"; }

const char* sw_last_error(const sw_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int sw_create(const sw_config* cfg, sw_ctx** out) {
  if (!cfg || !out) return SW_E_ARG;
  *out = nullptr;
  if (cfg->mode < 0 || cfg->mode > 2) return SW_E_ARG;
  if (cfg->alignment_type != SW_PROTEIN && cfg->alignment_type != SW_NUCLEIC) return SW_E_ARG;
  if (cfg->distance_fn < 0 || cfg->distance_fn > 3) return SW_E_ARG;
  if (cfg->lanes != SW_LANES_AUTO && cfg->lanes != SW_LANES_16 && cfg->lanes != SW_LANES_32) return SW_E_ARG;
  const float o = cfg->gap_open, e = cfg->gap_extension;
  if (!(std::isfinite(o) && std::isfinite(e))) return SW_E_ARG;
  if (o != std::floor(o) || e != std::floor(e)) return SW_E_UNSUPPORTED;
  if (o < 1 || e < 0 || o > 10000 || e > 10000) return SW_E_UNSUPPORTED;
  if (cfg->mode == SW_MODE_NW && !(o > e)) return SW_E_UNSUPPORTED;
  sw_ctx* ctx = new (std::nothrow) sw_ctx();
  if (!ctx) return SW_E_OOM;
  ctx->cfg = *cfg;
  ctx->o = (int)o;
  ctx->e = (int)e;
  std::memcpy(ctx->h_scores, cfg->scores, sizeof(ctx->h_scores));
  for (int a = 0; a < 128; a++)
    for (int b = 0; b < 128; b++) {
      int s = ctx->h_scores[a][b];
      if (s < -16383 || s > 16383) { delete ctx; return SW_E_UNSUPPORTED; }
      if (a == swg::kPadCode || b == swg::kPadCode) ctx->h_scores[a][b] = (int16_t)swg::kPadScore;
      else {
        ctx->max_abs_score = std::max(ctx->max_abs_score, std::abs(s));
        ctx->max_score = std::max(ctx->max_score, s);
      }
    }
  build_flags(ctx);
  cudaError_t err = cudaSetDevice(cfg->device);
  if (err != cudaSuccess) { int r = cuda_fail(ctx, err, "cudaSetDevice"); delete ctx; return r; }
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, cfg->device);
  if ((err = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (err = cudaMalloc(&ctx->d_scores, sizeof(ctx->h_scores))) != cudaSuccess ||
      (err = cudaMalloc(&ctx->d_flags, sizeof(ctx->h_flags))) != cudaSuccess ||
      (err = cudaMalloc(&ctx->d_throws, sizeof(int))) != cudaSuccess ||
      (err = cudaMemset(ctx->d_throws, 0, sizeof(int))) != cudaSuccess ||
      (err = cudaMemcpy(ctx->d_scores, ctx->h_scores, sizeof(ctx->h_scores), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (err = cudaMemcpy(ctx->d_flags, ctx->h_flags, sizeof(ctx->h_flags), cudaMemcpyHostToDevice)) != cudaSuccess) {
    cudaGetLastError();
    sw_destroy(ctx);
    return SW_E_CUDA;
  }
  *out = ctx;
  return SW_OK;
}

int sw_destroy(sw_ctx* ctx) {
  if (!ctx) return SW_E_ARG;
  cudaSetDevice(ctx->cfg.device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->own_stream) ctx->stream = ctx->own_stream;
  delete ctx->server;
  delete ctx->engine;
  cudaFree(ctx->d_seq);
  cudaFree(ctx->d_off);
  cudaFree(ctx->d_scores);
  cudaFree(ctx->d_flags);
  cudaFree(ctx->d_throws);
  cudaFree(ctx->d_carry);
  cudaFree(ctx->d_stage);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return SW_OK;
}

int sw_upload_sequences(sw_ctx* ctx, const uint8_t* concat, const int64_t* offsets, int32_t count) {
  if (!ctx) return SW_E_ARG;
  if (count < 0 || !offsets || (count > 0 && !concat && offsets[count] > 0))
    return fail(ctx, SW_E_ARG, "bad sequence arrays");
  if (offsets[0] != 0) return fail(ctx, SW_E_ARG, "offsets[0] must be 0");
  int maxlen = 0;
  for (int32_t k = 0; k < count; k++) {
    const int64_t len = offsets[k + 1] - offsets[k];
    if (len < 0) return fail(ctx, SW_E_ARG, "offsets must be non-decreasing");
    if (len > 32767) return fail(ctx, SW_E_UNSUPPORTED, "sequence longer than 32767 residues");
    maxlen = std::max(maxlen, (int)len);
  }
  const int64_t total = offsets[count];
  uint64_t letters[2] = {0, 0};
  for (int64_t k = 0; k < total; k++) {
    if (concat[k] >= 127)  // ScoringMatrix.Scores is [127,127]: the reference throws
      return fail(ctx, SW_E_ARG, "residue byte outside the 127-entry scoring table");
    letters[concat[k] >> 6] |= 1ull << (concat[k] & 63);
  }
  // The reference's float DP is exact while every value stays below 2^24.
  const double bound = (double)(ctx->max_abs_score + ctx->e) * 2.0 * maxlen + ctx->o;
  if (bound >= 16777216.0) return fail(ctx, SW_E_UNSUPPORTED, "scores could exceed float's exact range");
  cudaSetDevice(ctx->cfg.device);
  delete ctx->server;  // the database changes: jobs still running end with SW_E_STATE
  ctx->server = nullptr;
  cudaStreamSynchronize(ctx->stream);
  // the same lengths and letters as the resident set: the engine's plans and graphs stay, only the
  // residues (and the engine's codes of them) are replaced
  if (ctx->d_seq && count == ctx->nseq && ctx->h_off.size() == (size_t)count + 1 &&
      std::equal(offsets, offsets + count + 1, ctx->h_off.begin()) && letters[0] == ctx->letters[0] &&
      letters[1] == ctx->letters[1]) {
    if (total) CK(cudaMemcpyAsync(ctx->d_seq, concat, (size_t)total, cudaMemcpyHostToDevice, ctx->stream), "upload sequences");
    if (ctx->engine) {
      std::string msg;
      const int rc = ctx->engine->refresh_codes(ctx->d_seq, total, ctx->stream, &msg);
      if (rc) return fail(ctx, rc, msg);
    }
    CK(cudaStreamSynchronize(ctx->stream), "upload");
    ctx->h_seq.assign(concat, concat + total);
    return SW_OK;
  }
  cudaFree(ctx->d_seq);
  cudaFree(ctx->d_off);
  ctx->d_seq = nullptr;
  ctx->d_off = nullptr;
  ctx->nseq = 0;
  // one padding byte block at the end so vector loads past a sequence stay in bounds
  const size_t seq_bytes = (size_t)total + 64;
  CK(cudaMalloc(&ctx->d_seq, seq_bytes), "cudaMalloc(sequences)");
  CK(cudaMalloc(&ctx->d_off, sizeof(int64_t) * (size_t)(count + 1)), "cudaMalloc(offsets)");
  CK(cudaMemsetAsync(ctx->d_seq, swg::kPadCode, seq_bytes, ctx->stream), "cudaMemset");
  if (total) CK(cudaMemcpyAsync(ctx->d_seq, concat, (size_t)total, cudaMemcpyHostToDevice, ctx->stream), "upload sequences");
  CK(cudaMemcpyAsync(ctx->d_off, offsets, sizeof(int64_t) * (size_t)(count + 1), cudaMemcpyHostToDevice, ctx->stream), "upload offsets");
  CK(cudaStreamSynchronize(ctx->stream), "upload");
  ctx->h_off.assign(offsets, offsets + count + 1);
  ctx->h_seq.assign(concat, concat + total);
  ctx->nseq = count;
  ctx->maxlen = maxlen;
  ctx->letters[0] = letters[0];
  ctx->letters[1] = letters[1];
  if (ctx->engine) ctx->engine->invalidate();
  return SW_OK;
}

static int block_job(sw_ctx* ctx, int32_t rs, int32_t re, int32_t cs, int32_t ce, int32_t diag,
                     swg::PlainJob* J) {
  if (!ctx->d_seq) return fail(ctx, SW_E_STATE, "no sequences uploaded");
  if (rs < 0 || cs < 0 || re >= ctx->nseq || ce >= ctx->nseq || rs > re || cs > ce)
    return fail(ctx, SW_E_ARG, "block outside the uploaded sequences");
  const bool tri = diag && ctx->cfg.mode != SW_MODE_SWG_MS;
  if (tri && (rs != cs || re != ce)) return fail(ctx, SW_E_ARG, "a diagonal block must be square");
  const long long R = re - rs + 1, Cc = ce - cs + 1;
  std::memset(J, 0, sizeof(*J));
  J->seq = ctx->d_seq;
  J->off = ctx->d_off;
  J->rs = rs; J->re = re; J->cs = cs; J->ce = ce;
  J->tri = tri ? 1 : 0;
  J->npairs = tri ? R * (R - 1) / 2 : R * Cc;
  J->mirror = tri ? 1 : 0;
  J->scores = ctx->d_scores;
  J->flags = ctx->d_flags;
  J->o = ctx->o;
  J->e = ctx->e;
  J->mode = ctx->cfg.mode;
  J->protein = ctx->cfg.alignment_type == SW_PROTEIN;
  J->dist_fn = ctx->cfg.distance_fn;
  J->throws = ctx->d_throws;
  return SW_OK;
}

// After the context's stream is idle: SW_E_THROWS if a pair since the last check met the
// reference's JukesCantor Log(Zero) (its entry holds 0), and the flag is cleared.
static int check_throws(sw_ctx* ctx) {
  if (ctx->cfg.distance_fn != SW_DIST_JUKES_CANTOR) return SW_OK;
  int h = 0;
  CK(cudaMemcpy(&h, ctx->d_throws, sizeof(int), cudaMemcpyDeviceToHost), "read throw flag");
  if (!h) return SW_OK;
  CK(cudaMemset(ctx->d_throws, 0, sizeof(int)), "clear throw flag");
  return fail(ctx, SW_E_THROWS, "JukesCantor: the reference throws for Log(Zero) on a pair of this job");
}

static swg::EngineParams db_params(sw_ctx* ctx);

// After the context's stream is idle: SW_E_CUDA if the last engine launch recorded a violation of
// its kernels' self-checks (a work item or pair outside the plan's bounds; it was skipped).
static int check_kernel(sw_ctx* ctx) {
  if (!ctx->engine) return SW_OK;
  const int64_t v = ctx->engine->stat("kernel_error");
  if (v <= 0) return SW_OK;
  char buf[112];
  std::snprintf(buf, sizeof buf, "engine self-check %lld failed at index %lld", (long long)(v >> 48),
                (long long)(v & 0xFFFFFFFFLL));
  return fail(ctx, SW_E_CUDA, buf);
}

// One engine job: the queries row_lo..row_hi of a `ranks`-rank run, or (block 1 / 2) the diagonal /
// off-diagonal block of those rows by the columns col_lo..col_hi, with d_out pointing at the
// block's element (0, 0).
static int run_engine(sw_ctx* ctx, int32_t ranks, int row_lo, int row_hi, int16_t* d_out,
                      int64_t ld, int64_t* pairs, int64_t* cells, int block = 0, int col_lo = 0,
                      int col_hi = -1) {
  if (!ctx->d_seq) return fail(ctx, SW_E_STATE, "no sequences uploaded");
  if (!d_out || ranks < 1 || (!block && ld < ctx->nseq)) return fail(ctx, SW_E_ARG, "bad arguments");
  cudaSetDevice(ctx->cfg.device);
  if (!ctx->engine) {
    ctx->engine = swg::Engine::create();
    if (!ctx->engine) return fail(ctx, SW_E_OOM, "engine");
  }
  swg::EngineParams P;
  P.seq = ctx->d_seq; P.off = ctx->d_off;
  P.h_off = ctx->h_off.data(); P.h_seq = ctx->h_seq.data();
  P.nseq = ctx->nseq; P.maxlen = ctx->maxlen;
  P.scores = ctx->d_scores; P.flags = ctx->d_flags;
  P.h_scores = &ctx->h_scores[0][0]; P.h_flags = &ctx->h_flags[0][0];
  P.max_score = ctx->max_score; P.max_abs_score = ctx->max_abs_score;
  P.o = ctx->o; P.e = ctx->e;
  P.mode = ctx->cfg.mode;
  P.protein = ctx->cfg.alignment_type == SW_PROTEIN;
  P.lanes = ctx->cfg.lanes;
  P.dist_fn = ctx->cfg.distance_fn;
  P.throws = ctx->d_throws;
  P.ranks = ranks;
  P.row_lo = row_lo;
  P.row_hi = row_hi;
  P.block = block;
  P.col_lo = col_lo;
  P.col_hi = col_hi;
  P.out = d_out; P.ld = ld;
  if (block)  // the kernels index the output by global (s1, s2): shift the base to the block's corner
    P.out = reinterpret_cast<int16_t*>(reinterpret_cast<intptr_t>(d_out) -
                                       ((intptr_t)row_lo * ld + col_lo) * (intptr_t)sizeof(int16_t));
  P.sms = ctx->sms;
  P.stream = ctx->stream;
  std::string msg;
  int64_t np = 0, nc = 0;
  int rc = ctx->engine->run(P, &np, &nc, &ctx->last_reruns, &msg);
  if (rc) return fail(ctx, rc, msg);
  ctx->last_pairs = np;
  ctx->last_cells = nc;
  if (pairs) *pairs = np;
  if (cells) *cells = nc;
  return SW_OK;
}

static int run_plain(sw_ctx* ctx, swg::PlainJob& J) {
  const int block = 128;
  long threads = (long)ctx->sms * 8 * block;
  if (J.npairs < threads) threads = ((J.npairs + block - 1) / block) * block;
  if (threads < block) threads = block;
  const int grid = (int)(threads / block);
  int rc = ensure(ctx, &ctx->d_carry, &ctx->carry_bytes,
                  swg::plain_carry_bytes(J.mode, threads, ctx->maxlen, J.dist_fn), "carry scratch");
  if (rc) return rc;
  J.carry = ctx->d_carry;
  CK(swg::launch_plain_block(J, grid, block, ctx->stream), "plain block kernel launch");
  return SW_OK;
}

// The pairs of one block into device memory: the batched engine for blocks of at least
// kBlockEngineMin pairs (option "block_engine" 1, the default; 2: every block; 0: never), else the
// plain kernel (one thread per pair).
constexpr int64_t kBlockEngineMin = 4096;

static int block_device(sw_ctx* ctx, swg::PlainJob& J, int16_t* d_out, int64_t ld) {
  const bool engine = ctx->block_engine == 2 || (ctx->block_engine == 1 && J.npairs >= kBlockEngineMin);
  if (engine && J.npairs > 0) {
    int64_t np = 0, nc = 0;
    return run_engine(ctx, 1, J.rs, J.re, d_out, ld, &np, &nc, J.tri ? 1 : 2, J.cs, J.ce);
  }
  J.out = d_out;
  J.ld = ld;
  J.out_r0 = J.rs;
  J.out_c0 = J.cs;
  return run_plain(ctx, J);
}

int sw_compute_block_device(sw_ctx* ctx, int32_t rs, int32_t re, int32_t cs, int32_t ce,
                            int32_t diag, int16_t* d_out, int64_t ld, int64_t* pairs) {
  if (!ctx) return SW_E_ARG;
  if (!d_out || ld < (int64_t)(ce - cs + 1)) return fail(ctx, SW_E_ARG, "bad output buffer");
  cudaSetDevice(ctx->cfg.device);
  swg::PlainJob J;
  int rc = block_job(ctx, rs, re, cs, ce, diag, &J);
  if (rc) return rc;
  if ((rc = block_device(ctx, J, d_out, ld))) return rc;
  if (pairs) *pairs = J.npairs;
  return SW_OK;
}

int sw_compute_block(sw_ctx* ctx, int32_t rs, int32_t re, int32_t cs, int32_t ce, int32_t diag,
                     int16_t* out, int64_t ld, int64_t* pairs) {
  if (!ctx) return SW_E_ARG;
  if (!out || ld < (int64_t)(ce - cs + 1)) return fail(ctx, SW_E_ARG, "bad output buffer");
  cudaSetDevice(ctx->cfg.device);
  swg::PlainJob J;
  int rc = block_job(ctx, rs, re, cs, ce, diag, &J);
  if (rc) return rc;
  const size_t R = (size_t)(re - rs + 1), Cc = (size_t)(ce - cs + 1);
  void* stage = ctx->d_stage;
  if ((rc = ensure(ctx, &stage, &ctx->stage_bytes, R * Cc * sizeof(int16_t), "block staging"))) {
    ctx->d_stage = nullptr;
    return rc;
  }
  ctx->d_stage = static_cast<int16_t*>(stage);
  // Every entry of the block is written except the diagonal of a triangular block, which the
  // handler leaves as the caller had it: keep those values and put them back after the copy.
  std::vector<int16_t> keep;
  if (J.tri)
    for (size_t k = 0; k < R; k++) keep.push_back(out[k * (size_t)ld + k]);
  if ((rc = block_device(ctx, J, ctx->d_stage, (int64_t)Cc))) return rc;
  CK(cudaMemcpy2DAsync(out, (size_t)ld * 2, ctx->d_stage, Cc * 2, Cc * 2, R, cudaMemcpyDeviceToHost, ctx->stream), "copy block out");
  CK(cudaStreamSynchronize(ctx->stream), "compute block");
  for (size_t k = 0; k < keep.size(); k++) out[k * (size_t)ld + k] = keep[k];
  if (pairs) *pairs = J.npairs;
  if ((rc = check_kernel(ctx))) return rc;
  return check_throws(ctx);
}

int sw_align_pair(sw_ctx* ctx, const uint8_t* s1, int32_t m, const uint8_t* s2, int32_t n,
                  sw_pair_result* out) {
  if (!ctx) return SW_E_ARG;
  if (!out || m < 0 || n < 0) return fail(ctx, SW_E_ARG, "bad arguments");
  if ((!s1 && m > 0) || (!s2 && n > 0)) return fail(ctx, SW_E_ARG, "S1 or S2 is null");
  if (m > 32767 || n > 32767) return fail(ctx, SW_E_UNSUPPORTED, "sequence longer than 32767 residues");
  for (int k = 0; k < m; k++) if (s1[k] >= 127) return fail(ctx, SW_E_ARG, "residue byte outside the scoring table");
  for (int k = 0; k < n; k++) if (s2[k] >= 127) return fail(ctx, SW_E_ARG, "residue byte outside the scoring table");
  if (ctx->cfg.mode == SW_MODE_NW) return fail(ctx, SW_E_UNSUPPORTED, "sw_align_pair is the local aligner (SmithWatermanGotoh.Align)");
  cudaSetDevice(ctx->cfg.device);
  // one scratch block: [result][s1][s2][carry]
  const size_t res_b = 256, s_b = ((size_t)m + (size_t)n + 2 + 255) / 256 * 256;
  const size_t need = res_b + s_b + swg::pair_carry_bytes(n);
  int rc = ensure(ctx, &ctx->d_carry, &ctx->carry_bytes, need, "pair scratch");
  if (rc) return rc;
  char* base = static_cast<char*>(ctx->d_carry);
  swg::sw_pair_result_dev* d_res = reinterpret_cast<swg::sw_pair_result_dev*>(base);
  uint8_t* d_s1 = reinterpret_cast<uint8_t*>(base + res_b);
  uint8_t* d_s2 = d_s1 + m + 1;
  if (m) CK(cudaMemcpyAsync(d_s1, s1, (size_t)m, cudaMemcpyHostToDevice, ctx->stream), "upload s1");
  if (n) CK(cudaMemcpyAsync(d_s2, s2, (size_t)n, cudaMemcpyHostToDevice, ctx->stream), "upload s2");
  swg::PairJob J;
  J.s1 = d_s1; J.s2 = d_s2; J.m = m; J.n = n;
  J.scores = ctx->d_scores; J.flags = ctx->d_flags;
  J.o = ctx->o; J.e = ctx->e;
  J.carry = base + res_b + s_b;
  J.out = d_res;
  CK(swg::launch_align_pair(J, ctx->stream), "align pair launch");
  swg::sw_pair_result_dev r;
  CK(cudaMemcpyAsync(&r, d_res, sizeof(r), cudaMemcpyDeviceToHost, ctx->stream), "copy result");
  CK(cudaStreamSynchronize(ctx->stream), "align pair");
  out->score = r.score_is_neg_inf ? -INFINITY : (float)r.score;
  out->end1 = r.end1; out->end2 = r.end2;
  out->start1 = r.start1; out->start2 = r.start2;
  out->identity = r.identity; out->similarity = r.similarity;
  out->gaps = r.gaps; out->length = r.length;
  out->reserved = 0;
  if (ctx->cfg.alignment_type == SW_NUCLEIC && ctx->cfg.distance_fn == SW_DIST_MIN_MAX_NORM_SCORE) {
    // MinMaxNormScore (SWG-MS Program.cs:544-553) in binary64; SWG-MPI has no case for it: 0
    if (ctx->cfg.mode != SW_MODE_SWG_MS) { out->distance = 0; return SW_OK; }
    long long self1 = 0, self2 = 0;
    for (int k = 0; k < m; k++) self1 += ctx->h_scores[s1[k]][s1[k]];
    for (int k = 0; k < n; k++) self2 += ctx->h_scores[s2[k]][s2[k]];
    const long long s = (m == 0 || n == 0) ? 0 : r.score;
    volatile double x = (double)s / (double)std::max(self1, self2);
    volatile double v = (1.0 - x) * 32767.0;
    const double vv = v;
    out->distance = (vv > -2147483649.0 && vv < 2147483648.0) ? (int16_t)(uint16_t)(uint32_t)(int32_t)vv : 0;
    return SW_OK;
  }
  if (ctx->cfg.alignment_type == SW_NUCLEIC && ctx->cfg.distance_fn != SW_DIST_PERCENT_IDENTITY) {
    // Kimura2 / JukesCantor (Alignment.cs:254-348) in binary64, as the device epilogue
    const double eps = 4.9406564584124654e-324;  // System.Double.Epsilon
    const bool ms = ctx->cfg.mode == SW_MODE_SWG_MS;
    const double length = r.length, gapc = (double)(r.length - r.diag);
    double v;
    if (ctx->cfg.distance_fn == SW_DIST_KIMURA2) {
      volatile double P = (double)r.transitions / (length - gapc), Q = (double)r.transversions / (length - gapc);
      volatile double t1 = 1.0 - (2.0 * P + Q), t2 = 1.0 - 2.0 * Q;
      if (t1 <= eps || t2 <= eps) v = 10.0;
      else {
        volatile double a = 1.0 - 2.0 * P - Q;
        volatile double l1 = -0.5 * swg::cr_log(a), l2 = 0.25 * swg::cr_log(t2);
        v = l1 - l2;
      }
      if (ms && v > 10.0) v = 10.0;
    } else {
      volatile double frac = (double)(r.diag - r.identity) / (length - gapc);
      volatile double d = 1.0 - (4.0 / 3.0) * frac;
      if (d <= eps) {
        if (!ms) {
          out->distance = 0;
          return fail(ctx, SW_E_THROWS, "JukesCantor: the reference throws for Log(Zero)");
        }
        v = 10.0;
      } else {
        v = -0.75 * swg::cr_log(d);
      }
    }
    volatile double x = v * 32767.0;
    out->distance = (x > -2147483649.0 && x < 2147483648.0) ? (int16_t)(uint16_t)(uint32_t)(int32_t)x : 0;
    return SW_OK;
  }
  // ComputeDistance for this pair on the host, in binary32 like the device epilogue.
  int count;
  if (ctx->cfg.alignment_type == SW_NUCLEIC) count = r.identity;
  else count = r.similarity;
  volatile float p = (float)count / (float)r.length;
  volatile float d = (1.0f - p) * 32767.0f;
  const float x = d;
  out->distance = (x > -2147483648.0f && x < 2147483648.0f) ? (int16_t)(int32_t)x : 0;
  out->reserved = 0;
  return SW_OK;
}

// Int16 distance of one traced alignment under the context's rules (the same arithmetic as the
// kernels' epilogues): a, b are the aligned strings of len columns.
static int16_t traced_distance(const sw_ctx* ctx, const char* a, const char* b, int len,
                               const swg::TraceResult& r, int m, int n, long long self1, long long self2,
                               int* throws) {
  const bool protein = ctx->cfg.alignment_type == SW_PROTEIN;
  const int mode = ctx->cfg.mode, fn = ctx->cfg.distance_fn;
  auto conv_f = [](float x) -> int16_t { return (x > -2147483648.0f && x < 2147483648.0f) ? (int16_t)(int32_t)x : 0; };
  auto conv_d = [](double x) -> int16_t {
    return (x > -2147483649.0 && x < 2147483648.0) ? (int16_t)(uint16_t)(uint32_t)(int32_t)x : 0;
  };
  auto fraction = [&](int count, int cols) { volatile float p = (float)count / (float)cols; return conv_f((1.0f - p) * 32767.0f); };
  if (!protein && fn == SW_DIST_MIN_MAX_NORM_SCORE) {  // SWG-MS :544-553, NW :573-581
    if (mode == SW_MODE_SWG_MPI) return 0;               // no case in SWG-MPI's ComputeDistance
    const long long sc = r.valid ? r.score : 0;
    const long long maxS = std::max(self1, self2);
    const long long minS = mode == SW_MODE_NW ? 2LL * ctx->o + (long long)(m + n) * ctx->e : 0LL;
    volatile double x = (double)(sc - minS) / (double)(maxS - minS);
    volatile double v = (1.0 - x) * 32767.0;
    return conv_d(v);
  }
  if (!protein && (fn == SW_DIST_KIMURA2 || fn == SW_DIST_JUKES_CANTOR)) {
    const double eps = 4.9406564584124654e-324;  // System.Double.Epsilon
    const bool capped = mode != SW_MODE_SWG_MPI;
    const double nongap = (double)r.diag;
    double v;
    if (fn == SW_DIST_KIMURA2) {
      volatile double P = (double)r.transitions / nongap, Q = (double)r.transversions / nongap;
      volatile double t1 = 1.0 - (2.0 * P + Q), t2 = 1.0 - 2.0 * Q;
      if (t1 <= eps || t2 <= eps) v = 10.0;
      else {
        volatile double l1 = -0.5 * swg::cr_log(1.0 - 2.0 * P - Q), l2 = 0.25 * swg::cr_log(t2);
        v = l1 - l2;
      }
      if (capped && v > 10.0) v = 10.0;
    } else {
      volatile double d = 1.0 - (4.0 / 3.0) * ((double)(r.diag - r.identity) / nongap);
      if (d <= eps) {
        if (!capped) { *throws = 1; return 0; }
        v = 10.0;
      } else {
        v = -0.75 * swg::cr_log(d);
      }
    }
    volatile double x = v * 32767.0;
    return conv_d(x);
  }
  if (mode == SW_MODE_NW) {
    if (protein) {  // MBF similarity: non-gap pairs with a positive score, over every column
      int sim = 0;
      for (int k = 0; k < len; k++)
        if (a[k] != '-' && b[k] != '-' && ctx->h_scores[(uint8_t)a[k]][(uint8_t)b[k]] > 0) sim++;
      return fraction(sim, len);
    }
    // identity between the last leading and the first trailing end gap (Program.cs:547-571)
    int fa = -1, fb = -1, la = -1, lb = -1;
    for (int k = 0; k < len && fa < 0; k++) if (a[k] != '-') fa = k;
    for (int k = 0; k < len && fb < 0; k++) if (b[k] != '-') fb = k;
    for (int k = len - 1; k >= 0 && la < 0; k--) if (a[k] != '-') la = k;
    for (int k = len - 1; k >= 0 && lb < 0; k--) if (b[k] != '-') lb = k;
    const int first = std::max(fa, fb), last = std::min(la, lb);
    int id = 0;
    for (int k = first; k <= last && k >= 0; k++) if (a[k] == b[k]) id++;
    return fraction(id, last - first + 1);
  }
  if (protein) {
    if (mode == SW_MODE_SWG_MPI) return fraction(r.similarity, r.length);
    int sim = 0;
    for (int k = 0; k < len; k++)
      if (a[k] != '-' && b[k] != '-' && ctx->h_scores[(uint8_t)a[k]][(uint8_t)b[k]] > 0) sim++;
    return fraction(sim, len);
  }
  return fraction(r.identity, r.length);
}

int sw_align_strings(sw_ctx* ctx, const int32_t* rows, const int32_t* cols, int32_t npairs, char* aln1,
                     char* aln2, const int64_t* offsets, sw_pair_result* results) {
  if (!ctx) return SW_E_ARG;
  if (npairs < 0 || (npairs > 0 && (!rows || !cols || !aln1 || !aln2 || !offsets || !results)))
    return fail(ctx, SW_E_ARG, "bad arguments");
  if (!ctx->d_seq) return fail(ctx, SW_E_STATE, "no sequences uploaded");
  // every pair's room: offsets[k + 1] - offsets[k] >= m + n (the longest alignment)
  std::vector<int> len_m(npairs), len_n(npairs);
  for (int32_t k = 0; k < npairs; k++) {
    if (rows[k] < 0 || rows[k] >= ctx->nseq || cols[k] < 0 || cols[k] >= ctx->nseq)
      return fail(ctx, SW_E_ARG, "pair outside the uploaded sequences");
    len_m[k] = (int)(ctx->h_off[rows[k] + 1] - ctx->h_off[rows[k]]);
    len_n[k] = (int)(ctx->h_off[cols[k] + 1] - ctx->h_off[cols[k]]);
    if (offsets[k] < 0 || offsets[k + 1] - offsets[k] < (int64_t)len_m[k] + len_n[k])
      return fail(ctx, SW_E_ARG, "offsets leave less than m + n characters for a pair");
  }
  cudaSetDevice(ctx->cfg.device);
  const bool local = ctx->cfg.mode != SW_MODE_NW;
  constexpr size_t kBudget = size_t(512) << 20;  // scratch of one batch of pairs
  int throws = 0;
  int32_t k0 = 0;
  while (k0 < npairs) {
    // the batch: pairs while their decision bytes and rows fit the budget (at least one pair)
    const long row_ints = 2L * (ctx->maxlen + 1);
    size_t dir_stride = 0;
    int32_t k1 = k0;
    while (k1 < npairs) {
      const size_t st = std::max(dir_stride, (size_t)len_m[k1] * (size_t)len_n[k1]);
      if (k1 > k0 && (st + row_ints * 4) * (size_t)(k1 - k0 + 1) > kBudget) break;
      dir_stride = st;
      k1++;
    }
    dir_stride = (dir_stride + 15) / 16 * 16;
    const int32_t nb = k1 - k0;
    const size_t chars = (size_t)(offsets[k1] - offsets[k0]);
    std::vector<int64_t> rel(nb);
    for (int32_t k = 0; k < nb; k++) rel[k] = offsets[k0 + k] - offsets[k0];
    uint8_t* d_dirs = nullptr;
    int* d_rows = nullptr;
    int32_t* d_pairs = nullptr;
    char* d_a = nullptr;
    int64_t* d_rel = nullptr;
    swg::TraceResult* d_res = nullptr;
    auto release = [&]() {
      cudaFree(d_dirs); cudaFree(d_rows); cudaFree(d_pairs); cudaFree(d_a); cudaFree(d_rel); cudaFree(d_res);
    };
    if (cudaMalloc(&d_dirs, std::max<size_t>(dir_stride * nb, 16)) != cudaSuccess ||
        cudaMalloc(&d_rows, sizeof(int) * (size_t)row_ints * nb) != cudaSuccess ||
        cudaMalloc(&d_pairs, sizeof(int32_t) * 2 * (size_t)nb) != cudaSuccess ||
        cudaMalloc(&d_a, std::max<size_t>(2 * chars, 16)) != cudaSuccess ||
        cudaMalloc(&d_rel, sizeof(int64_t) * (size_t)nb) != cudaSuccess ||
        cudaMalloc(&d_res, sizeof(swg::TraceResult) * (size_t)nb) != cudaSuccess) {
      release();
      cudaGetLastError();
      return fail(ctx, SW_E_OOM, "cudaMalloc alignment strings");
    }
    cudaError_t e = cudaMemcpyAsync(d_pairs, rows + k0, sizeof(int32_t) * nb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_pairs + nb, cols + k0, sizeof(int32_t) * nb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rel, rel.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, ctx->stream);
    swg::TraceJob J;
    std::memset(&J, 0, sizeof(J));
    J.seq = ctx->d_seq; J.off = ctx->d_off;
    J.rows = d_pairs; J.cols = d_pairs + nb; J.npairs = nb;
    J.scores = ctx->d_scores; J.o = ctx->o; J.e = ctx->e;
    J.dirs = d_dirs; J.dir_stride = (long long)dir_stride;
    J.vrow = d_rows; J.row_stride = row_ints;
    J.aln1 = d_a; J.aln2 = d_a + chars; J.out_off = d_rel; J.out = d_res;
    if (e == cudaSuccess) e = swg::launch_traceback(J, local, ctx->stream);
    std::vector<swg::TraceResult> res(nb);
    if (e == cudaSuccess) e = cudaMemcpyAsync(aln1 + offsets[k0], d_a, chars, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(aln2 + offsets[k0], d_a + chars, chars, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(res.data(), d_res, sizeof(swg::TraceResult) * nb, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    release();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "alignment strings");
    for (int32_t k = 0; k < nb; k++) {
      const swg::TraceResult& r = res[k];
      sw_pair_result& o = results[k0 + k];
      o.score = r.valid ? (float)r.score : -INFINITY;
      o.end1 = r.end1; o.end2 = r.end2; o.start1 = r.start1; o.start2 = r.start2;
      o.identity = r.identity; o.similarity = r.similarity; o.gaps = r.gaps; o.length = r.length;
      o.reserved = 0;
      long long self1 = 0, self2 = 0;  // MinMaxNormScore's self scores of the two sequences
      for (int64_t x = ctx->h_off[rows[k0 + k]]; x < ctx->h_off[rows[k0 + k] + 1]; x++) self1 += ctx->h_scores[ctx->h_seq[x]][ctx->h_seq[x]];
      for (int64_t x = ctx->h_off[cols[k0 + k]]; x < ctx->h_off[cols[k0 + k] + 1]; x++) self2 += ctx->h_scores[ctx->h_seq[x]][ctx->h_seq[x]];
      o.distance = traced_distance(ctx, aln1 + offsets[k0 + k], aln2 + offsets[k0 + k], r.length, r,
                                   len_m[k0 + k], len_n[k0 + k], self1, self2, &throws);
    }
    k0 = k1;
  }
  if (throws) return fail(ctx, SW_E_THROWS, "JukesCantor: the reference throws for Log(Zero) on a pair of this call");
  return SW_OK;
}

int sw_synchronize(sw_ctx* ctx) {
  if (!ctx) return SW_E_ARG;
  cudaSetDevice(ctx->cfg.device);
  CK(cudaStreamSynchronize(ctx->stream), "synchronize");
  return check_throws(ctx);
}

int sw_last_rerun_count(const sw_ctx* ctx_, int64_t* count) {
  sw_ctx* ctx = const_cast<sw_ctx*>(ctx_);
  if (!ctx || !count) return SW_E_ARG;
  *count = 0;
  if (!ctx->engine) return SW_OK;
  cudaSetDevice(ctx->cfg.device);
  std::string msg;
  int rc = ctx->engine->rerun_count(ctx->stream, count, &msg);
  return rc ? fail(ctx, rc, msg) : SW_OK;
}

int sw_all_pairs_device(sw_ctx* ctx, int32_t ranks, int16_t* d_out, int64_t ld, int64_t* pairs,
                        int64_t* cells) {
  if (!ctx) return SW_E_ARG;
  return run_engine(ctx, ranks, 0, -1, d_out, ld, pairs, cells);
}

int sw_compute_rank_blocks(sw_ctx* ctx, int32_t rank, int32_t world, int16_t* d_out, int64_t ld,
                           int64_t* pairs) {
  if (!ctx) return SW_E_ARG;
  if (world < 1 || rank < 0 || rank >= world) return fail(ctx, SW_E_ARG, "rank outside the world");
  std::vector<int32_t> st(world), en(world);
  sw_partition_ranges(0, ctx->nseq, world, st.data(), en.data());
  if (st[rank] > en[rank]) {  // an empty row range owns no pairs
    if (pairs) *pairs = 0;
    return SW_OK;
  }
  int64_t cells = 0;
  return run_engine(ctx, world, st[rank], en[rank], d_out, ld, pairs, &cells);
}

int sw_compute_rows(sw_ctx* ctx, int32_t row_start, int32_t row_end, int16_t* d_out, int64_t ld,
                    int64_t* pairs) {
  if (!ctx) return SW_E_ARG;
  if (ctx->cfg.mode == SW_MODE_SWG_MS)
    return fail(ctx, SW_E_UNSUPPORTED, "SWG-MS aligns both orientations of a pair: use its rank blocks");
  if (row_start < 0 || row_end >= ctx->nseq || row_start > row_end + 1)
    return fail(ctx, SW_E_ARG, "rows outside the uploaded sequences");
  if (row_start > row_end) {  // no rows: no pairs
    if (pairs) *pairs = 0;
    return SW_OK;
  }
  int64_t cells = 0;
  return run_engine(ctx, 1, row_start, row_end, d_out, ld, pairs, &cells);
}

int sw_autotune(sw_ctx* ctx, int16_t* d_out, int64_t ld, int32_t weights[7]) {
  if (!ctx) return SW_E_ARG;
  if (!ctx->d_seq) return fail(ctx, SW_E_STATE, "no sequences uploaded");
  if (!d_out || ld < ctx->nseq) return fail(ctx, SW_E_ARG, "bad output buffer");
  cudaSetDevice(ctx->cfg.device);
  if (!ctx->engine) {
    ctx->engine = swg::Engine::create();
    if (!ctx->engine) return fail(ctx, SW_E_OOM, "engine");
  }
  swg::EngineParams P = db_params(ctx);
  P.out = d_out;
  P.ld = ld;
  std::string msg;
  int w[7];
  const int rc = ctx->engine->autotune(P, w, &msg);
  if (rc) return fail(ctx, rc, msg);
  if (weights) for (int x = 0; x < 7; x++) weights[x] = w[x];
  return check_throws(ctx);
}

int sw_query(sw_ctx* ctx, const char* key, int64_t* value) {
  if (!ctx || !key || !value) return SW_E_ARG;
  const std::string k(key);
  if (k == "pairs" || k == "cells") {
    *value = (k == "pairs") ? ctx->last_pairs : ctx->last_cells;
    return SW_OK;
  }
  if (k != "launches" && k != "bins" && k != "alphabet" && k != "items" && k != "lane16_pairs" &&
      k != "tripped" && k != "planned_items" && k != "box_fallbacks" && k != "box_spilled" &&
      k != "box_third_pass" && k != "kernel_error")
    return fail(ctx, SW_E_ARG, "unknown counter " + k);
  *value = ctx->engine ? ctx->engine->stat(key) : 0;
  return SW_OK;
}

int sw_set_option(sw_ctx* ctx, const char* key, int64_t value) {
  if (!ctx || !key) return SW_E_ARG;
  if (!ctx->engine) {
    ctx->engine = swg::Engine::create();
    if (!ctx->engine) return fail(ctx, SW_E_OOM, "engine");
  }
  const std::string k(key);
  if (k == "stream") {  // a caller-owned cudaStream_t; 0 restores the context's own stream
    cudaStreamSynchronize(ctx->stream);
    if (!ctx->own_stream) ctx->own_stream = ctx->stream;
    ctx->stream = value ? reinterpret_cast<cudaStream_t>(value) : ctx->own_stream;
    return SW_OK;
  }
  if (k == "block_engine") {
    if (value < 0 || value > 2) return fail(ctx, SW_E_ARG, "block_engine must be 0, 1 or 2");
    ctx->block_engine = (int)value;
    return SW_OK;
  }
  if (k == "plan_only") {
    ctx->engine->set_plan_only(value ? 1 : 0);
    return SW_OK;
  }
  if (k.compare(0, 6, "serve_") == 0) {
    if (ctx->server) return fail(ctx, SW_E_STATE, "serving options are read when the first job is submitted");
    if (value < 0) return fail(ctx, SW_E_ARG, "serving options are non-negative");
    swg::ServeOptions& so = ctx->serve_opt;
    if (k == "serve_memory_mb") so.memory_bytes = (size_t)value << 20;
    else if (k == "serve_arena_mb") so.arena_bytes = std::max<size_t>(1, (size_t)value) << 20;
    else if (k == "serve_slots") so.slots = (int)std::max<int64_t>(1, std::min<int64_t>(value, 1 << 20));
    else if (k == "serve_wave_us") so.wave_seconds = std::max<int64_t>(100, value) * 1e-6;
    else return fail(ctx, SW_E_ARG, "unknown option " + k);
    return SW_OK;
  }
  swg::EngineOptions& o = ctx->engine->options();
  if (k == "int16_threshold") o.int16_threshold = value;
  else if (k == "use_graph") o.use_graph = value ? 1 : 0;
  else if (k == "two_pass") {
    if (value < 0 || value > 2) return fail(ctx, SW_E_ARG, "two_pass must be 0, 1 or 2");
    o.two_pass = (int)value;
  }
  else if (k == "box_reg") o.box_reg = value ? 1 : 0;
  else if (k == "third_pass") o.third_pass = value ? 1 : 0;
  else if (k == "chunk") {
    if (value != 0 && (value < 32 || value > 1024)) return fail(ctx, SW_E_ARG, "chunk must be 0 or in [32, 1024]");
    o.chunk = (int)value;
  } else if (k == "rows_per_lane") {
    if (value != 0 && (value < 4 || value > 16 || (value & 1))) return fail(ctx, SW_E_ARG, "rows_per_lane must be 0 or an even number from 4 to 16");
    o.k_override = (int)value;
  } else return fail(ctx, SW_E_ARG, "unknown option " + k);
  return SW_OK;
}

int sw_all_pairs(sw_ctx* ctx, int32_t ranks, int16_t* out, int64_t ld, int64_t* pairs,
                 int64_t* cells) {
  if (!ctx) return SW_E_ARG;
  if (!out || ld < ctx->nseq) return fail(ctx, SW_E_ARG, "bad output buffer");
  cudaSetDevice(ctx->cfg.device);
  const size_t N = (size_t)ctx->nseq;
  void* stage = ctx->d_stage;
  int rc = ensure(ctx, &stage, &ctx->stage_bytes, std::max<size_t>(N * N * 2, 2), "result staging");
  if (rc) { ctx->d_stage = nullptr; return rc; }
  ctx->d_stage = static_cast<int16_t*>(stage);
  if ((rc = sw_all_pairs_device(ctx, ranks, ctx->d_stage, (int64_t)N, pairs, cells))) return rc;
  if (N) CK(cudaMemcpy2DAsync(out, (size_t)ld * 2, ctx->d_stage, N * 2, N * 2, N, cudaMemcpyDeviceToHost, ctx->stream), "copy result");
  CK(cudaStreamSynchronize(ctx->stream), "all pairs");
  if ((rc = check_kernel(ctx))) return rc;
  return check_throws(ctx);
}

static swg::EngineParams db_params(sw_ctx* ctx) {
  swg::EngineParams P;
  P.seq = ctx->d_seq; P.off = ctx->d_off;
  P.h_off = ctx->h_off.data(); P.h_seq = ctx->h_seq.data();
  P.nseq = ctx->nseq; P.maxlen = ctx->maxlen;
  P.scores = ctx->d_scores; P.flags = ctx->d_flags;
  P.h_scores = &ctx->h_scores[0][0]; P.h_flags = &ctx->h_flags[0][0];
  P.max_score = ctx->max_score; P.max_abs_score = ctx->max_abs_score;
  P.o = ctx->o; P.e = ctx->e;
  P.mode = ctx->cfg.mode;
  P.protein = ctx->cfg.alignment_type == SW_PROTEIN;
  P.lanes = ctx->cfg.lanes;
  P.dist_fn = ctx->cfg.distance_fn;
  P.throws = ctx->d_throws;
  P.two_pass = ctx->engine ? ctx->engine->current_options().two_pass : 1;
  P.third_pass = ctx->engine ? ctx->engine->current_options().third_pass : 1;
  P.ranks = 1;
  P.out = nullptr; P.ld = 0;
  P.sms = ctx->sms;
  P.stream = ctx->stream;
  return P;
}

int sw_submit_job(sw_ctx* ctx, const uint8_t* q_concat, const int64_t* q_offsets, int32_t nq,
                  int16_t* out, int64_t ld_out, int64_t* ticket) {
  if (!ctx) return SW_E_ARG;
  if (!ctx->d_seq) return fail(ctx, SW_E_STATE, "no database uploaded");
  if (nq < 1 || !q_offsets || !out || !ticket || ld_out < ctx->nseq) return fail(ctx, SW_E_ARG, "bad arguments");
  if (q_offsets[0] != 0) return fail(ctx, SW_E_ARG, "offsets[0] must be 0");
  if (!q_concat && q_offsets[nq] > 0) return fail(ctx, SW_E_ARG, "bad query arrays");
  int maxlen = ctx->maxlen;
  for (int32_t k = 0; k < nq; k++) {
    const int64_t len = q_offsets[k + 1] - q_offsets[k];
    if (len < 0) return fail(ctx, SW_E_ARG, "offsets must be non-decreasing");
    if (len > 32767) return fail(ctx, SW_E_UNSUPPORTED, "query longer than 32767 residues");
    maxlen = std::max(maxlen, (int)len);
  }
  for (int64_t k = 0; k < q_offsets[nq]; k++)
    if (q_concat[k] >= 127) return fail(ctx, SW_E_ARG, "residue byte outside the 127-entry scoring table");
  const double bound = (double)(ctx->max_abs_score + ctx->e) * 2.0 * maxlen + ctx->o;
  if (bound >= 16777216.0) return fail(ctx, SW_E_UNSUPPORTED, "scores could exceed float's exact range");
  cudaSetDevice(ctx->cfg.device);
  std::string msg;
  if (!ctx->server) {
    cudaStreamSynchronize(ctx->stream);
    int rc = 0;
    ctx->server = swg::Server::create(db_params(ctx), ctx->cfg.device, ctx->serve_opt, &msg, &rc);
    if (!ctx->server) return fail(ctx, rc ? rc : SW_E_OOM, msg);
  }
  const int rc = ctx->server->submit(q_concat, q_offsets, nq, out, ld_out, ticket, &msg);
  return rc ? fail(ctx, rc, msg) : SW_OK;
}

int sw_poll(sw_ctx* ctx, int64_t ticket, int32_t timeout_ms, int32_t* done, sw_job_info* info) {
  if (!ctx || !done) return SW_E_ARG;
  if (!ctx->server) return fail(ctx, SW_E_ARG, "unknown ticket");
  int d = 0;
  const int rc = ctx->server->poll(ticket, std::max(0, timeout_ms), &d, info);
  *done = d;
  if (rc == SW_E_ARG) return fail(ctx, rc, "unknown ticket");
  if (rc) return fail(ctx, rc, "job failed");
  return SW_OK;
}

int sw_serve_stats(sw_ctx* ctx, sw_serve_counters* stats) {
  if (!ctx || !stats) return SW_E_ARG;
  std::memset(stats, 0, sizeof(*stats));
  if (ctx->server) ctx->server->stats(stats);
  return SW_OK;
}

int sw_serve_drain(sw_ctx* ctx) {
  if (!ctx) return SW_E_ARG;
  if (!ctx->server) return SW_OK;
  ctx->server->drain();
  delete ctx->server;
  ctx->server = nullptr;
  return SW_OK;
}

int sw_measure_int_peak(int32_t device, double* max_ops, double* add_ops) {
  if (!max_ops || !add_ops) return SW_E_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return SW_E_CUDA;
  return swg::measure_int_peak(max_ops, add_ops) == cudaSuccess ? SW_OK : SW_E_CUDA;
}

}  // extern "C"
