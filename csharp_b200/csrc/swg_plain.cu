// Plain block kernel: the drop-in replacement of one ComputeBlock call
// (SalsaTPL/Salsa.SmithWatermanMPI/Program.cs:203-257, Salsa.SmithWatermanMS/Program.cs:341-375,
// Salsa.NeedlemanWunschTPL/Program.cs:206-267).  One launch per block, one thread per pair,
// int32 score lanes.  A thread walks its pair in strips of K rows held in registers; the row
// below each strip (V, G and their counters per column) is carried to the next strip through a
// per-thread slice of global scratch, interleaved across threads so a warp's accesses coalesce.
// Substitution scores and column flags are staged in shared memory.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <type_traits>
#include "swg_box_reg.cuh"
#include "swg_device.cuh"
#include "swg_internal.h"

namespace swg {

template <class CP>
struct Carry {
  int v, g;
  typename CP::T cv, cg;
};

template <class CP>
struct DpResult {
  int best;  // SW: traceback start score; NW: V(m,n)
  int bi, bj;
  typename CP::T c;
};

// The DP of one pair.  s1 rows (1..m), s2 columns (1..n), both non-empty.
template <bool LOCAL, class CP, int K, bool TRACK_POS>
__device__ __forceinline__ DpResult<CP> dp_pair(const uint8_t* __restrict__ s1, int m,
                                                const uint8_t* __restrict__ s2, int n,
                                                const int16_t* sc, const uint8_t* fl, int o, int e,
                                                Carry<CP>* carry, long stride) {
  typedef typename CP::T T;
  DpResult<CP> res;
  res.best = kNegInf;
  res.bi = res.bj = 0;
  res.c = CP::origin();
  for (int s0 = 0; s0 < m; s0 += K) {
    int c1[K], vl[K], h[K], bv[K], bj[K];
    T cl[K], ch[K], bc[K];
#pragma unroll
    for (int r = 0; r < K; r++) {
      const int i = s0 + r + 1;
      c1[r] = (i <= m) ? (int)s1[i - 1] * kTable : kPadCode * kTable;
      vl[r] = LOCAL ? 0 : (-o - (i - 1) * e);
      cl[r] = LOCAL ? CP::stop(i, 0) : CP::col0(i);
      h[r] = kNegInf;
      ch[r] = CP::origin();
      bv[r] = kNegInf;
      bc[r] = CP::origin();
      bj[r] = 0;
    }
    int vdiag = (LOCAL || s0 == 0) ? 0 : (-o - (s0 - 1) * e);
    T cdiag = LOCAL ? CP::stop(s0, 0) : (s0 == 0 ? CP::origin() : CP::col0(s0));
    for (int j = 1; j <= n; j++) {
      const int c2 = s2[j - 1];
      int vu, gu;
      T cvu, cgu;
      if (s0 == 0) {
        vu = LOCAL ? 0 : (-o - (j - 1) * e);
        gu = kNegInf;
        cvu = LOCAL ? CP::stop(0, j) : CP::row0(j);
        cgu = cvu;
      } else {
        const Carry<CP> cr = carry[(long)j * stride];
        vu = cr.v; gu = cr.g; cvu = cr.cv; cgu = cr.cg;
      }
      int vd = vdiag;
      T cd = cdiag;
      vdiag = vu;
      cdiag = cvu;
#pragma unroll
      for (int r = 0; r < K; r++) {
        const int s = sc[c1[r] + c2];
        const uint32_t f = fl[c1[r] + c2];
        int v, g;
        T cv, cg;
        gotoh_cell<LOCAL, CP>(s, f, vd, cd, vu, gu, cvu, cgu, vl[r], cl[r], h[r], ch[r], o, e,
                              s0 + r + 1, j, v, g, cv, cg);
        vd = vl[r];
        cd = cl[r];
        vl[r] = v;
        cl[r] = cv;
        vu = v; gu = g; cvu = cv; cgu = cg;
        if (LOCAL && v > bv[r]) {
          bv[r] = v;
          bc[r] = cv;
          if (TRACK_POS) bj[r] = j;
        }
      }
      if (s0 + K < m) {
        Carry<CP> cw;
        cw.v = vu; cw.g = gu; cw.cv = cvu; cw.cg = cgu;
        carry[(long)j * stride] = cw;
      }
    }
#pragma unroll
    for (int r = 0; r < K; r++) {
      const int i = s0 + r + 1;
      if (LOCAL) {
        if (i <= m && bv[r] > res.best) {
          res.best = bv[r];
          res.c = bc[r];
          res.bi = i;
          res.bj = bj[r];
        }
      } else if (i == m) {
        res.best = vl[r];
        res.c = cl[r];
        res.bi = m;
        res.bj = n;
      }
    }
  }
  return res;
}

// ---- pair enumeration of a block -----------------------------------------------------------
// tri: rows rs..re, columns cs..i-1 (diagonal blocks of SWG-MPI/NW, cs == rs); else the full
// rectangle.
__device__ __forceinline__ void pair_of(long long p, const PlainJob& J, int& i, int& j) {
  if (J.tri) {
    // p = a(a-1)/2 + b with a = i - rs >= 1, 0 <= b < a
    long long a = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
    while (a * (a - 1) / 2 > p) a--;
    while ((a + 1) * a / 2 <= p) a++;
    i = J.rs + (int)a;
    j = J.cs + (int)(p - a * (a - 1) / 2);
  } else {
    const int cols = J.ce - J.cs + 1;
    i = J.rs + (int)(p / cols);
    j = J.cs + (int)(p % cols);
  }
}

__device__ __forceinline__ void load_tables(const PlainJob& J, int16_t* sc, uint8_t* fl) {
  for (int k = threadIdx.x; k < kTable * kTable; k += blockDim.x) {
    sc[k] = J.scores[k];
    fl[k] = J.flags[k];
  }
  __syncthreads();
}

// NW distance (Salsa.NeedlemanWunschTPL/Program.cs:547-571): identity over the aligned region
// with the leading and trailing same-type gap runs removed; protein: similarity over the full
// aligned length (:583-604).
__device__ __forceinline__ int16_t nw_distance(const NwCnt::T& c, int m, int n, int protein) {
  const int count = (int)(c.w0 & 0xFFFFu), len = (int)(c.w0 >> 16);
  if (protein) return fraction_distance(count, len);
  const int lead = (int)(c.w1 >> 16);
  const int run = (int)(int16_t)(c.w1 & 0xFFFFu);
  int trimmed = len - lead - (run < 0 ? -run : run);
  if (m == 0 || n == 0) trimmed = 0;  // a single gap run: first non-gap index > last
  return fraction_distance(count, trimmed);
}

// Sum of the matrix's diagonal over a sequence's residues (MinMaxNormScore's self score).
__device__ __forceinline__ int self_score(const uint8_t* s, int n, const int16_t* sc) {
  int t = 0;
  for (int k = 0; k < n; k++) t += sc[(int)s[k] * (kTable + 1)];
  return t;
}

template <bool LOCAL, class CP, int K>
__global__ void __launch_bounds__(128) plain_block_kernel(PlainJob J) {
  __shared__ int16_t sc[kTable * kTable];
  __shared__ uint8_t fl[kTable * kTable];
  load_tables(J, sc, fl);
  const long stride = (long)gridDim.x * blockDim.x;
  const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  Carry<CP>* carry = reinterpret_cast<Carry<CP>*>(J.carry) + tid;
  long long np = J.npairs;
  if (J.list) np = min(np, (long long)*J.list_count);
  for (long long p = tid; p < np; p += stride) {
    int i, j;
    if (J.list) {
      const int2 pr = J.list[p];
      i = pr.x;
      j = pr.y;
    } else {
      pair_of(p, J, i, j);
    }
    const uint8_t* s1 = J.qoff ? J.qseq + J.qoff[i] : J.seq + J.off[i];
    const uint8_t* s2 = J.seq + J.off[j];
    const int m = J.qoff ? J.qlen[i] : (int)(J.off[i + 1] - J.off[i]);
    const int n = (int)(J.off[j + 1] - J.off[j]);
    int16_t d;
    const bool minmax = J.dist_fn == 3 && !J.protein;  // MinMaxNormScore: from the score alone
    if constexpr (std::is_same<CP, KimCnt>::value) {
      // Kimura2 / JukesCantor; SWG-MS and NW cap them at 10 (and JukesCantor's Log(Zero) is 10)
      KimCnt::T c = KimCnt::origin();
      if (m > 0 && n > 0) c = dp_pair<LOCAL, CP, K, false>(s1, m, s2, n, sc, fl, J.o, J.e, carry, stride).c;
      d = kim_distance(c, J.dist_fn, J.mode != kModeSwgMpi, J.throws);
    } else if (LOCAL) {
      if (m == 0 || n == 0) {
        d = minmax ? minmax_distance(0, self_score(s1, m, sc), self_score(s2, n, sc), m, n, J.o, J.e, J.mode)
                   : fraction_distance(0, 0);
      } else {
        DpResult<CP> r = dp_pair<LOCAL, CP, K, false>(s1, m, s2, n, sc, fl, J.o, J.e, carry, stride);
        const uint32_t w = *reinterpret_cast<const uint32_t*>(&r.c);
        d = minmax ? minmax_distance(r.best, self_score(s1, m, sc), self_score(s2, n, sc), m, n, J.o, J.e, J.mode)
                   : fraction_distance((int)(w & 0xFFFFu), (int)(w >> 16));
      }
    } else if constexpr (std::is_same<CP, NwCnt>::value) {
      NwCnt::T c;
      long long score;  // V(m, n): the global alignment's score
      if (m == 0 && n == 0) { c = NwCnt::origin(); score = 0; }
      else if (m == 0) { c = NwCnt::row0(n); score = -(long long)J.o - (long long)(n - 1) * J.e; }
      else if (n == 0) { c = NwCnt::col0(m); score = -(long long)J.o - (long long)(m - 1) * J.e; }
      else {
        DpResult<CP> r = dp_pair<LOCAL, CP, K, false>(s1, m, s2, n, sc, fl, J.o, J.e, carry, stride);
        c = *reinterpret_cast<const NwCnt::T*>(&r.c);
        score = r.best;
      }
      d = minmax ? minmax_distance(score, self_score(s1, m, sc), self_score(s2, n, sc), m, n, J.o, J.e, J.mode)
                 : nw_distance(c, m, n, J.protein);
    }
    if (J.qoff) {
      J.qout[i][j] = d;
      continue;
    }
    J.out[(long long)(i - J.out_r0) * J.ld + (j - J.out_c0)] = d;
    if (J.mirror) J.out[(long long)(j - J.out_r0) * J.ld + (i - J.out_c0)] = d;
  }
}

// ---- box kernel: the counters of the best cell from a confined DP --------------------------------
// The first pass gives, per pair, the best score S and the reference's traceback start cell
// (ie, je) (first maximum in row-major order).  Every optimal local alignment ending there has,
// at each of its cells, a suffix score (from that cell to (ie, je)) >= 0: its prefix up to the
// cell scores at most the best V there, which is at most S.  A reverse DP anchored at (ie, je),
// with every state below 0 pruned, therefore keeps all such alignments and finds all their first
// pairs (the cells whose reverse score plus their own pair score equals S).  The box from the
// smallest such row and column to (ie, je) contains the reference's traceback path, and a local
// DP confined to the box (zero boundary) reproduces its values and pointer choices along that
// path (each value on the path is reached inside the box, and off-path competitors can only be
// lower than in the full matrix), so the counters of the box's first maximum, which is (ie, je)
// with score S, are the traceback's.  Pairs whose scan or box exceed the budget, or whose box
// does not end at S, go to the 32-bit full DP.
// One warp per pair.  The reverse scan goes row by row (rows ie-1 .. 0) with the lanes on a
// window of 64 positions (two chunks of 32) ending at the row's rightmost live position; within
// a row the gap chain RHs(j) = max(X(j), RHs(j+1) - min(e, o)) is a max-plus prefix scan over
// the lanes.  The box DP is a warp wavefront (lane = box row, 32 rows per pass).
constexpr int kBoxWarps = 4;
constexpr int kBoxMaxW = kWarpBoxMaxCols;  // box columns (else 32-bit full DP)
constexpr int kBoxMaxH = kWarpBoxMaxCols;  // box rows
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int scan_max_up(int y, int lane) {
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    const int t = __shfl_up_sync(kFull, y, k);
    if (lane >= k) y = max(y, t);
  }
  return y;
}

constexpr int kBoxMaxA1 = 33;  // letters + padding of the dense codes
// Rows of the box tables: one per residue byte of s1 in query mode, else one per code.
constexpr int kBoxTabRows = 128;

// A pair the box step cannot finish: the full DP with counters, on the 16-bit lanes of the
// one-pass kernel (J.fb) where the engine runs that third pass, else on the 32-bit lanes.
__device__ __forceinline__ void box_give_up(const BoxJob& J, int q, int d) {
  atomicAdd(J.stats + 3, 1ull);
  atomicAdd(J.stats + 1, ~0ull);  // not finished yet (the third pass counts it again)
  if (J.fb) {
    const int w = atomicAdd(J.fb_count, 1);
    if (w < J.fb_cap) {
      J.fb[w] = make_int2(q, d);
      atomicAdd(J.stats + 5, 1ull);
      return;
    }
  }
  const int wr = atomicAdd(J.rerun_count, 1);
  if (wr < J.rerun_cap) J.rerun[wr] = make_int2(q, d);
}

__global__ void __launch_bounds__(kBoxWarps * 32) box_kernel(BoxJob J) {
  // S(a, b) << 8 | counted flag; rows: s1's dense codes, or its residue bytes in query mode
  __shared__ int scf[kBoxTabRows * kBoxMaxA1];
  __shared__ int4 rowbuf[kBoxWarps * kBoxMaxW];
  const int A1 = J.A + 1;
  for (int k = threadIdx.x; k < (J.qseq ? kBoxTabRows : A1) * A1; k += blockDim.x)
    scf[k] = J.qseq ? J.qscf[k]
                    : (int)(((uint32_t)(J.lettab[k] - J.o) << 8) | (J.flagtab[k] & kFlagCount));
  __syncthreads();
  constexpr int NEG = kNegInf;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // bottom row of a box pass: V, G, and the two counter words per column
  int4* buf = rowbuf + warp * kBoxMaxW;
  const long nwarps = (long)gridDim.x * kBoxWarps;
  const long long np = min((long long)*J.count, J.list_cap);
  const int o = J.o, e = J.e, dchain = min(J.e, J.o);
  for (long p = (long)blockIdx.x * kBoxWarps + warp; p < np; p += nwarps) {
    const int4 rec = J.list[p];
    const int q = rec.x, d = rec.y, S = rec.z & 0xFFFF;
    const int ie = (int)((uint32_t)rec.w >> 16), je = rec.w & 0xFFFF;
    const uint8_t* a = J.qseq ? J.qseq + J.qoff[q] : J.seq + J.off[q];
    const uint8_t* b = J.seq + J.off[d];
    // ---- reverse scan: positions (i, j) = residues consumed ----
    int hi = je, lo = je;
    int rwb0 = lane == 0 ? 0 : NEG, rwb1 = NEG, rgb0 = NEG, rgb1 = NEG;  // row below, pos lane / 32+lane
    int cand_i = 1 << 30, cand_j = 1 << 30;
    // S needs at least S / max S diagonal columns: beyond max_score the box cannot fit
    bool ok = S <= J.max_score;
    long long cells = 0;
    for (int i = ie - 1; ok && i >= 0; i--) {
      const int arow = (int)a[i] * A1;
      // chunk 0: pos = lane, j = hi - lane
      const int j0 = hi - lane;
      int rwn0 = __shfl_up_sync(kFull, rwb0, 1);  // RW(i+1, j0+1)
      if (lane == 0) rwn0 = NEG;
      int pair0 = NEG;
      if (rwn0 > NEG && j0 >= 0 && j0 < je) {
        pair0 = (scf[arow + b[j0]] >> 8) + rwn0;
        if (pair0 == S) { cand_i = min(cand_i, i + 1); cand_j = min(cand_j, j0 + 1); }
      }
      const int x0 = max(pair0, rgb0 > NEG ? rgb0 - o : NEG);
      int y0 = scan_max_up(x0 > NEG ? x0 + dchain * lane : NEG, lane);
      int rh0 = (y0 > NEG && j0 >= 0) ? y0 - dchain * lane : NEG;  // RHs(i, j0)
      int rhp0 = __shfl_up_sync(kFull, rh0, 1);                     // RHs(i, j0+1)
      if (lane == 0) rhp0 = NEG;
      int rw0 = max(x0, rhp0 > NEG ? rhp0 - o : NEG);
      int rg0 = max(rgb0 > NEG ? rgb0 - e : NEG, rw0);
      if (j0 < 0) rw0 = rg0 = NEG;
      if (rw0 < 0) rw0 = NEG;
      if (rg0 < 0) rg0 = NEG;
      if (rh0 < 0) rh0 = NEG;
      // chunk 1 (pos 32 + lane): when the row below reaches it or the gap chain runs into it
      const int rh31 = __shfl_sync(kFull, rh0, 31);
      int rw1 = NEG, rg1 = NEG;
      if (hi - lo >= 31 || rh31 >= dchain) {
        const int j1 = hi - 32 - lane;
        int rwn1 = __shfl_up_sync(kFull, rwb1, 1);
        const int last0 = __shfl_sync(kFull, rwb0, 31);
        if (lane == 0) rwn1 = last0;
        int pair1 = NEG;
        if (rwn1 > NEG && j1 >= 0 && j1 < je) {
          pair1 = (scf[arow + b[j1]] >> 8) + rwn1;
          if (pair1 == S) { cand_i = min(cand_i, i + 1); cand_j = min(cand_j, j1 + 1); }
        }
        const int x1 = max(pair1, rgb1 > NEG ? rgb1 - o : NEG);
        int y1 = scan_max_up(x1 > NEG ? x1 + dchain * (32 + lane) : NEG, lane);
        y1 = max(y1, __shfl_sync(kFull, y0, 31));  // the chain from chunk 0
        int rh1 = (y1 > NEG && j1 >= 0) ? y1 - dchain * (32 + lane) : NEG;
        int rhp1 = __shfl_up_sync(kFull, rh1, 1);
        if (lane == 0) rhp1 = rh31;
        rw1 = max(x1, rhp1 > NEG ? rhp1 - o : NEG);
        rg1 = max(rgb1 > NEG ? rgb1 - e : NEG, rw1);
        if (j1 < 0) rw1 = rg1 = NEG;
        if (rw1 < 0) rw1 = NEG;
        if (rg1 < 0) rg1 = NEG;
        if (rh1 < 0) rh1 = NEG;
        if (__shfl_sync(kFull, rh1, 31) >= dchain) ok = false;  // the chain leaves the window
      }
      cells += 64;
      const unsigned b0 = __ballot_sync(kFull, rw0 > NEG || rg0 > NEG);
      const unsigned b1 = __ballot_sync(kFull, rw1 > NEG || rg1 > NEG);
      if (!ok || cells > J.budget) { ok = false; break; }
      if (!b0 && !b1) break;  // nothing above can still reach (ie, je)
      const int minpos = b0 ? __ffs(b0) - 1 : 32 + __ffs(b1) - 1;
      const int maxpos = b1 ? 63 - __clz(b1) : 31 - __clz(b0);
      // next row: positions relative to the new rightmost live column
      const int sft = minpos, src = (lane + sft) & 31;
      const int a0 = __shfl_sync(kFull, rw0, src), a1 = __shfl_sync(kFull, rw1, src);
      const int g0 = __shfl_sync(kFull, rg0, src), g1 = __shfl_sync(kFull, rg1, src);
      rwb0 = lane + sft < 32 ? a0 : (lane + sft < 64 ? a1 : NEG);
      rgb0 = lane + sft < 32 ? g0 : (lane + sft < 64 ? g1 : NEG);
      rwb1 = lane + sft < 32 ? a1 : NEG;
      rgb1 = lane + sft < 32 ? g1 : NEG;
      lo = hi - maxpos;
      hi = hi - minpos;
    }
#pragma unroll
    for (int k = 16; k >= 1; k >>= 1) {
      cand_i = min(cand_i, __shfl_xor_sync(kFull, cand_i, k));
      cand_j = min(cand_j, __shfl_xor_sync(kFull, cand_j, k));
    }
    const int ilo = cand_i, jlo = cand_j;
    const int h = ie - ilo + 1, w = je - jlo + 1;
    if (ilo > ie || jlo > je || h > kBoxMaxH || w > kBoxMaxW) ok = false;
    // ---- box DP: rows ilo..ie (lanes), columns jlo..je (steps); local, zero boundary ----
    int vcap = NEG;
    uint32_t ccap = 0u;
    if (ok) {
      const int passes = (h + 31) / 32;
      for (int ps = 0; ps < passes; ps++) {
        const int t = ps * 32 + lane;  // box row of this lane
        const bool row_ok = t < h;
        const int arow = row_ok ? (int)a[ilo - 1 + t] * A1 : 0;
        int vl = 0, hh = NEG;
        uint32_t cl = 0u, ch = 0u;
        int uv = 0, ug = NEG, dv = 0;
        uint32_t ucv = 0u, ucg = 0u, dcv = 0u;
        for (int s2 = 0; s2 < w + 31; s2++) {
          const int bv = __shfl_up_sync(kFull, uv, 1), bg = __shfl_up_sync(kFull, ug, 1);
          const uint32_t bcv = __shfl_up_sync(kFull, ucv, 1), bcg = __shfl_up_sync(kFull, ucg, 1);
          const int c = s2 - lane;
          int vu, gu;
          uint32_t cvu, cgu;
          if (lane == 0) {
            if (ps == 0 || c < 0 || c >= w) { vu = 0; gu = NEG; cvu = cgu = 0u; }
            else { const int4 x = buf[c]; vu = x.x; gu = x.y; cvu = (uint32_t)x.z; cgu = (uint32_t)x.w; }
          } else {
            vu = bv; gu = bg; cvu = bcv; cgu = bcg;
          }
          const int vd = dv;
          const uint32_t cd = dcv;
          dv = vu;
          dcv = cvu;
          if (row_ok && c >= 0 && c < w) {
            const int col = (int)b[jlo - 1 + c];
            int v, g;
            uint32_t cv, cg;
            const int sf = scf[arow + col];
            gotoh_cell<true, SwCnt>(sf >> 8, (uint32_t)sf & 0xFFu, vd, cd, vu, gu, cvu, cgu,
                                    vl, cl, hh, ch, o, e, 0, 0, v, g, cv, cg);
            vl = v;
            cl = cv;
            uv = v; ug = g; ucv = cv; ucg = cg;
            if (t == h - 1 && c == w - 1) { vcap = v; ccap = cv; }
          } else {
            uv = 0; ug = NEG; ucv = ucg = 0u;  // outside the box: the zero boundary
          }
          if (lane == 31 && ps + 1 < passes && c >= 0 && c < w) buf[c] = make_int4(uv, ug, (int)ucv, (int)ucg);
        }
        __syncwarp();
      }
      const int holder = (h - 1) & 31;
      vcap = __shfl_sync(kFull, vcap, holder);
      ccap = __shfl_sync(kFull, ccap, holder);
      if (vcap != S) ok = false;
    }
    if (lane == 0) {
      if (!ok) {
        box_give_up(J, q, d);
      } else {
        const int16_t dist = fraction_distance((int)(ccap & 0xFFFFu), (int)(ccap >> 16));
        if (J.qout) {
          J.qout[q][d] = dist;
        } else {
          J.out[(long long)q * J.ld + d] = dist;
          if (J.mirror) J.out[(long long)d * J.ld + q] = dist;
        }
      }
    }
    __syncwarp();
  }
}

// ---- box step, one pair per thread with the DP rows in registers (swg_box_reg.cuh) -------------
constexpr int kRegThreads = 128;

__global__ void __launch_bounds__(kRegThreads) box_scan_kernel(BoxJob J) {
  __shared__ int sc[kBoxTabRows * kBoxMaxA1];
  const int A1 = J.A + 1;
  for (int k = threadIdx.x; k < (J.qseq ? kBoxTabRows : A1) * A1; k += blockDim.x) {
    const int a = k / A1, c = k - a * A1;
    sc[k] = J.qseq ? J.qsc[k] : (a == J.A || c == J.A) ? kRegPadScore : J.lettab[k] - J.o;
  }
  __syncthreads();
  const long long np = min((long long)*J.count, J.list_cap);
  auto emit = [&](long long p, const int4& rec, int rc, const RegBox& bx) {
    const int bw = bx.bhi - bx.blo + 1;
    if (rc == kRegScanOk && bw <= 32) {
      // the thresholds are used up: the window's first words keep the box for the band DP
      *reinterpret_cast<int4*>(J.win + p * kRegWinWords) = make_int4(bx.ci, bx.cj, bx.blo, bx.bhi);
      const int c = bw <= 8 ? 0 : bw <= 16 ? 1 : bw <= 24 ? 2 : 3;
      const int pos = atomicAdd(J.cls_count + c, 1);
      J.cls[c >> 1][(c & 1) ? J.list_cap - 1 - pos : pos] = (int)p;
      return;
    }
    // a wider window or band: the warp box kernel (its 64-column windows), else the 32-bit lanes
    const int w = J.spill_cap > 0 ? atomicAdd(J.spill_count, 1) : 0;
    if (w < J.spill_cap) {
      J.spill[w] = rec;
      atomicAdd(J.stats + 4, 1ull);
      return;
    }
    box_give_up(J, rec.x, rec.y);
  };
  reg_scan_run(J.list, J.win, (long long)blockIdx.x * kRegThreads + threadIdx.x, np,
               (long long)gridDim.x * kRegThreads, J.qseq ? J.qseq : J.seq, J.qseq ? J.qoff : J.off, J.seq,
               J.off, sc, A1, J.o, J.e, emit);
}

template <int B>
__global__ void __launch_bounds__(kRegThreads) box_band_kernel(BoxJob J, int c) {
  __shared__ int scf[kBoxTabRows * kBoxMaxA1];
  const int A1 = J.A + 1;
  for (int k = threadIdx.x; k < (J.qseq ? kBoxTabRows : A1) * A1; k += blockDim.x) {
    const int a = k / A1, x = k - a * A1;
    scf[k] = J.qseq ? J.qscf[k]
           : (a == J.A || x == J.A) ? (int)((uint32_t)kRegPadScore << 8)
                                    : (int)(((uint32_t)(J.lettab[k] - J.o) << 8) | (J.flagtab[k] & kFlagCount));
  }
  __syncthreads();
  const long long np = min((long long)J.cls_count[c], J.list_cap);
  const int* idx = (c & 1) ? J.cls[c >> 1] + (J.list_cap - 1) : J.cls[c >> 1];
  auto emit = [&](int, const int4& rec, bool ok, uint32_t cnt) {
    if (!ok) {
      box_give_up(J, rec.x, rec.y);
      return;
    }
    const int16_t dist = fraction_distance((int)(cnt & 0xFFFFu), (int)(cnt >> 16));
    if (J.qout) {
      J.qout[rec.x][rec.y] = dist;
      return;
    }
    J.out[(long long)rec.x * J.ld + rec.y] = dist;
    if (J.mirror) J.out[(long long)rec.y * J.ld + rec.x] = dist;
  };
  reg_band_run<B>(idx, (c & 1) ? -1 : 1, (long long)blockIdx.x * kRegThreads + threadIdx.x, np,
                  (long long)gridDim.x * kRegThreads, J.list, J.win, J.qseq ? J.qseq : J.seq,
                  J.qseq ? J.qoff : J.off, J.seq, J.off, scf, A1, J.o, J.e, emit);
}

// Resident CTAs per SM of a kernel with kRegThreads threads (its registers decide), looked up once.
template <class Kern>
int reg_ctas_per_sm(Kern k) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kRegThreads, 0) != cudaSuccess) {
    cudaGetLastError();
    n = 1;
  }
  return std::max(n, 1);
}

cudaError_t launch_box_scan(const BoxJob& J, int sms, cudaStream_t st) {
  if (J.A + 1 > kBoxMaxA1) return cudaErrorInvalidValue;
  static const int per_sm = reg_ctas_per_sm(box_scan_kernel);
  box_scan_kernel<<<std::max(sms, 1) * per_sm, kRegThreads, 0, st>>>(J);
  return cudaGetLastError();
}

cudaError_t launch_box_band(const BoxJob& J, int c, int sms, cudaStream_t st) {
  if (J.A + 1 > kBoxMaxA1 || c < 0 || c > 3) return cudaErrorInvalidValue;
  static const int per_sm[4] = {reg_ctas_per_sm(box_band_kernel<8>), reg_ctas_per_sm(box_band_kernel<16>),
                                reg_ctas_per_sm(box_band_kernel<24>), reg_ctas_per_sm(box_band_kernel<32>)};
  const int grid = std::max(sms, 1) * per_sm[c];
  switch (c) {
    case 0: box_band_kernel<8><<<grid, kRegThreads, 0, st>>>(J, c); break;
    case 1: box_band_kernel<16><<<grid, kRegThreads, 0, st>>>(J, c); break;
    case 2: box_band_kernel<24><<<grid, kRegThreads, 0, st>>>(J, c); break;
    default: box_band_kernel<32><<<grid, kRegThreads, 0, st>>>(J, c); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_box(const BoxJob& J, int grid, int block, cudaStream_t st) {
  if (J.A + 1 > kBoxMaxA1) return cudaErrorInvalidValue;
  (void)block;
  box_kernel<<<grid, kBoxWarps * 32, 0, st>>>(J);
  return cudaGetLastError();
}

// Single pair with every PairwiseAlignment field (SmithWatermanGotoh.Align).
__global__ void __launch_bounds__(32) align_pair_kernel(PairJob J) {
  __shared__ int16_t sc[kTable * kTable];
  __shared__ uint8_t fl[kTable * kTable];
  for (int k = threadIdx.x; k < kTable * kTable; k += blockDim.x) {
    sc[k] = J.scores[k];
    fl[k] = J.flags[k];
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  sw_pair_result_dev out;
  if (J.m == 0 || J.n == 0) {
    out.score_is_neg_inf = 1;
    out.score = 0;
    out.end1 = out.end2 = out.start1 = out.start2 = 0;
    out.identity = out.similarity = out.gaps = out.length = 0;
    out.diag = out.transitions = out.transversions = 0;
  } else {
    DpResult<FullCnt> r = dp_pair<true, FullCnt, 4, true>(J.s1, J.m, J.s2, J.n, sc, fl, J.o, J.e,
                                                          reinterpret_cast<Carry<FullCnt>*>(J.carry), 1);
    out.score_is_neg_inf = 0;
    out.score = r.best;
    out.end1 = r.bi;
    out.end2 = r.bj;
    out.start1 = r.c.si;
    out.start2 = r.c.sj;
    out.identity = r.c.id;
    out.similarity = r.c.sim;
    out.length = r.c.len;
    out.diag = r.c.diag;
    out.transitions = r.c.ts;
    out.transversions = r.c.tv;
    out.gaps = r.c.len - ((r.bi - r.c.si) + (r.bj - r.c.sj) - r.c.len);
  }
  *J.out = out;
}

// ---- launchers -----------------------------------------------------------------------------
size_t plain_carry_bytes(int mode, long threads, int maxlen, int dist_fn) {
  static_assert(sizeof(Carry<KimCnt>) >= sizeof(Carry<NwCnt>), "carry sizes");
  const size_t per = dist_fn ? sizeof(Carry<KimCnt>) : (mode == kModeNw) ? sizeof(Carry<NwCnt>) : sizeof(Carry<SwCnt>);
  return per * (size_t)threads * (size_t)(maxlen + 1);
}

cudaError_t launch_plain_block(const PlainJob& J, int grid, int block, cudaStream_t st) {
  if (J.npairs == 0) return cudaSuccess;
  const bool kim = (J.dist_fn == 1 || J.dist_fn == 2) && !J.protein;
  if (J.mode == kModeNw && kim) plain_block_kernel<false, KimCnt, 8><<<grid, block, 0, st>>>(J);
  else if (J.mode == kModeNw) plain_block_kernel<false, NwCnt, 8><<<grid, block, 0, st>>>(J);
  else if (kim) plain_block_kernel<true, KimCnt, 8><<<grid, block, 0, st>>>(J);
  else plain_block_kernel<true, SwCnt, 8><<<grid, block, 0, st>>>(J);
  return cudaGetLastError();
}

size_t pair_carry_bytes(int n) { return sizeof(Carry<FullCnt>) * (size_t)(n + 1); }

cudaError_t launch_align_pair(const PairJob& J, cudaStream_t st) {
  align_pair_kernel<<<1, 32, 0, st>>>(J);
  return cudaGetLastError();
}

// ---- integer-pipe calibration --------------------------------------------------------------
// Eight ring-coupled chains of a 2-input op per thread (no chain folds because each op reads a
// different neighbour).  Used as the roofline denominator of the cell-update kernels.
template <int OP>
__global__ void int_peak_kernel(int* out, int seed, int iters) {
  int x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = seed * (k + 1) + (int)threadIdx.x * 7 + k;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      int r;
      if (OP == 0) asm volatile("max.s32 %0, %1, %2;" : "=r"(r) : "r"(x[k]), "r"(x[(k + 1) & 7]));
      else asm volatile("add.s32 %0, %1, %2;" : "=r"(r) : "r"(x[k]), "r"(x[(k + 1) & 7]));
      x[k] = r;
    }
  }
  int s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= x[k];
  out[(long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

cudaError_t measure_int_peak(double* max_ops, double* add_ops) {
  int dev;
  cudaGetDevice(&dev);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  int* d = nullptr;
  cudaError_t err = cudaMalloc(&d, sizeof(int) * (size_t)blocks * threads);
  if (err != cudaSuccess) return err;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double res[2];
  for (int op = 0; op < 2; op++) {
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
      cudaEventRecord(e0);
      if (op == 0) int_peak_kernel<0><<<blocks, threads>>>(d, rep + 1, iters);
      else int_peak_kernel<1><<<blocks, threads>>>(d, rep + 1, iters);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && ms < best) best = ms;
    }
    res[op] = (double)blocks * threads * iters * 8.0 / (best * 1e-3);
  }
  err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  *max_ops = res[0];
  *add_ops = res[1];
  return err;
}

}  // namespace swg
