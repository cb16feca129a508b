// Box step of the two-pass SW-Gotoh path, one pair per thread, DP state in registers.
//
// The first pass (the score-only wavefront kernel) gives, per pair, the best score S and the
// reference's traceback start cell (ie, je) (the first maximum in row-major order,
// SmithWatermanGotoh.cs:211-214), plus an upper bound U(i) of the forward value V(i, j) of every
// row i in the 128 rows above ie (and one bound for all rows further up).  The counters of the
// traceback path (aligned columns and identity or similarity, Traceback :229-332) come from two
// small DPs near (ie, je):
//
//  1. Reverse scan (reg_scan_run).  RW(i, j) = best score of a path from the V state after
//     consuming i residues of s1 and j of s2 to the V state at (ie, je); RG / RH the same from the
//     vertical / horizontal gap states:
//        RW(i,j) = max(S(s1[i], s2[j]) + RW(i+1,j+1), RG(i+1,j) - o, RH(i,j+1) - o)
//        RG(i,j) = max(RW(i,j), RG(i+1,j) - e),   RH(i,j) = max(RW(i,j), RH(i,j+1) - e)
//     with RW(ie, je) = 0, row by row upwards.  A state on an optimal alignment ending at
//     (ie, je) has a prefix scoring at most V(i, j) <= U(i) and a completion scoring S minus that,
//     so its completion is at least T(i) = S - U(i) >= 0: states below T(i) are pruned.  The first
//     aligned pair of such an alignment is a cell (i+1, j+1) with S(s1[i], s2[j]) +
//     RW(i+1, j+1) == S; the smallest row ci and column cj of all of them bound a box that holds
//     every optimal alignment ending at (ie, je), the traceback's among them, and the diagonals
//     (j - i) of the live states in rows ci..ie bound a band that holds them too.
//  2. Band DP (reg_band_run).  The local Gotoh DP with counters, in the reference's comparison
//     order, on the cells of the box inside the band, with a zero boundary (V = 0, gaps
//     -infinity, counters 0) outside.  The region holds the traceback path; along it every value
//     equals the full matrix's (values inside never exceed the full matrix's and the path's are
//     reached inside), and every pointer and gap-size decision on the path compares path values
//     with values no larger than the full matrix's, so the DP follows the same path and its
//     counters at (ie, je) are the traceback's.  The value there must come out as S.
//
// Both DPs keep one row of states in registers, indexed by diagonal: slot k of a row holds the
// diagonal base + k, so the diagonal predecessor of a cell is its own slot in the row before, the
// vertical one the neighbouring slot, and the horizontal one the slot just computed; the
// unrolled row code indexes registers statically.  The scan's window of kRegWin diagonals moves
// by kRegShift when the live states reach an edge; a pair whose live states need a wider window
// is handed on (to the warp box kernel, which works on 64-column windows).  The band DP runs with
// B slots for a band of at most B diagonals.
//
// Each thread runs its pairs as one flattened loop, one DP row per iteration: a thread whose pair
// ends takes its next pair in the same iteration, so the threads of a warp keep issuing the
// same row code.
#pragma once
#include <cstdint>
#include <vector_types.h>

#ifdef __CUDACC__
#define SWG_REG_FN __host__ __device__ __forceinline__
#else
#define SWG_REG_FN inline
#endif

namespace swg {

constexpr int kRegDead = -(1 << 28);       // pruned state / -infinity
constexpr int kRegPadScore = -(1 << 20);   // score of the padding code: no alignment uses it
constexpr int kRegWin = 32;                // reverse-scan window (diagonals; one bit each in a mask)
constexpr int kRegShift = 4;               // window move when the live states reach an edge
constexpr int kRegLeft = 12;               // slot of the end cell's diagonal when the scan starts
constexpr int kRegWinRows = 128;           // rows above ie with their own bound
constexpr int kRegWinWords = kRegWinRows / 8;  // 4-bit bound codes, eight per word

// Threshold of a 4-bit bound code q: the largest T = S - U(i) the code stands for is at least
// this, so pruning below it keeps every state an optimal alignment uses.
SWG_REG_FN int reg_thr_of(int q) {
  return q <= 8 ? 4 * q : q <= 12 ? 40 + 8 * (q - 9) : q == 13 ? 96 : q == 14 ? 128 : 192;
}
// The largest code whose threshold does not exceed t (t >= 0).
SWG_REG_FN int reg_code_of(int t) {
  return t < 32 ? (t >> 2) : t < 40 ? 8 : t < 48 ? 9 : t < 56 ? 10 : t < 64 ? 11 : t < 96 ? 12 : t < 128 ? 13 : t < 192 ? 14 : 15;
}

SWG_REG_FN int reg_max(int a, int b) { return a > b ? a : b; }
SWG_REG_FN int reg_min(int a, int b) { return a < b ? a : b; }

#ifdef __CUDACC__
SWG_REG_FN uint32_t reg_shl8(uint32_t lo, uint32_t hi) {
#ifdef __CUDA_ARCH__
  return __funnelshift_l(lo, hi, 8);
#else
  return (hi << 8) | (lo >> 24);
#endif
}
SWG_REG_FN uint32_t reg_shr8(uint32_t lo, uint32_t hi) {
#ifdef __CUDA_ARCH__
  return __funnelshift_r(lo, hi, 8);
#else
  return (lo >> 8) | (hi << 24);
#endif
}
SWG_REG_FN int reg_ctz(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __ffs((int)x) - 1;
#else
  return __builtin_ctz(x);
#endif
}
SWG_REG_FN int reg_hibit(uint32_t x) {
#ifdef __CUDA_ARCH__
  return 31 - __clz((int)x);
#else
  return 31 - __builtin_clz(x);
#endif
}
#else
inline uint32_t reg_shl8(uint32_t lo, uint32_t hi) { return (hi << 8) | (lo >> 24); }
inline uint32_t reg_shr8(uint32_t lo, uint32_t hi) { return (lo >> 8) | (hi << 24); }
inline int reg_ctz(uint32_t x) { return __builtin_ctz(x); }
inline int reg_hibit(uint32_t x) { return 31 - __builtin_clz(x); }
#endif

// A pair record of the box step: x = s1 index, y = s2 index, z = S | T_rest << 16 (the threshold
// of the rows above the 128-row window), w = ie << 16 | je (1-based).  Its window (kRegWinWords
// words) holds the 4-bit codes of the thresholds of rows ie-1, ie-2, ..., ie-128 (nibble k of the
// window = row ie-1-k, eight per word from the low bits).
// The scan's result: box rows ci..ie and columns cj..je, band diagonals blo..bhi (clipped to
// the box).
struct RegBox {
  int ci, cj, blo, bhi;
};

// Outcomes of the scan: box found, window too narrow, no first pair (bad input).
enum { kRegScanOk = 0, kRegScanWide = 1, kRegScanNone = 2 };

// Reverse scans of pairs list[first], list[first + stride], ... below np, each with its window
// win + p * kRegWinWords.  aseq + aoff[k] are the residues of s1 = sequence k (a row index of sc),
// seq + off[k] the codes of s2 = sequence k (0..A1-2; A1-1 is the padding code); sc[a * A1 + b]
// the substitution score of s1 residue a and s2 code b (the padding code's column
// kRegPadScore).  emit(p, rec, outcome, box) receives each pair's outcome.
template <class ScT, class Emit>
SWG_REG_FN void reg_scan_run(const int4* list, const uint32_t* win, long long first, long long np,
                             long long stride, const uint8_t* aseq, const int64_t* aoff, const uint8_t* seq,
                             const int64_t* off, const ScT* sc, int A1, int o, int e, Emit& emit) {
  constexpr int W = kRegWin;
  constexpr int D = kRegDead;
  const uint32_t pad = (uint32_t)(A1 - 1);
  int RW[W], RG[W];
  uint32_t cw[W / 4];
  long long p = first;
  bool active = false;
  int4 rec;
  rec.x = rec.y = rec.z = rec.w = 0;
  const uint8_t* a = seq;
  const uint8_t* b = seq;
  const uint32_t* wp = win;
  int S = 0, trest = 0, ie = 0, je = 0, i = 0, base = 0, ci = 0, cj = 0, dlo = 0, dhi = 0, blo = 0, bhi = -1;
  // codes of slots k..k+3 of row i: s2 residues at columns i + base + k.., padding outside [0, je)
  auto load_codes = [&]() {
#pragma unroll
    for (int t = 0; t < W / 4; t++) {
      uint32_t x = 0;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int j = i + base + 4 * t + u;
        const uint32_t c = (j >= 0 && j < je) ? (uint32_t)b[j] : pad;
        x |= c << (8 * u);
      }
      cw[t] = x;
    }
  };
  for (;;) {
    if (!active) {
      if (p >= np) break;
      rec = list[p];
      S = rec.z & 0xFFFF;
      trest = (rec.z >> 16) & 0xFFFF;
      ie = (int)((uint32_t)rec.w >> 16);
      je = rec.w & 0xFFFF;
      a = aseq + aoff[rec.x];
      b = seq + off[rec.y];
      wp = win + p * kRegWinWords;
#pragma unroll
      for (int k = 0; k < W; k++) {
        RW[k] = D;
        RG[k] = D;
      }
      RW[kRegLeft] = 0;  // row ie: RW(ie, je) = 0
      base = je - ie - kRegLeft;
      i = ie - 1;
      ci = cj = 1 << 30;
      dlo = dhi = je - ie;
      blo = 0;
      bhi = -1;
      load_codes();
      active = true;
    }
    // ---- row i: slots from the right (columns descending) ----
    const int kr = ie - 1 - i;
    const int thr = kr < kRegWinRows ? reg_thr_of((int)((wp[kr >> 3] >> ((kr & 7) * 4)) & 15u)) : trest;
    const ScT* srow = sc + (int)a[i] * A1;
    int rh = D, cand = -1;
    uint32_t live = 0u;
#pragma unroll
    for (int k = W - 1; k >= 0; k--) {
      const int c = (int)((cw[k >> 2] >> ((k & 3) * 8)) & 0xFFu);
      const int pr = (int)srow[c] + RW[k];
      if (pr == S) cand = k;
      const int gu = k > 0 ? RG[k - 1] : D;
      const int x = reg_max(pr, gu - o);
      const int rw = reg_max(x, rh - o);
      rh = reg_max(rw, rh - e);
      const int rg = reg_max(rw, gu - e);
      const bool lv = rg >= thr;  // rg >= rw: the slot is live iff its RG survives
      RW[k] = rw >= thr ? rw : D;
      RG[k] = lv ? rg : D;
      live |= lv ? (1u << k) : 0u;
    }
    const int j0 = i + base;  // column of slot 0
    if (j0 < 0) {             // slots left of column 0 are no positions
      const int kv = -j0;
      live &= kv >= W ? 0u : (~0u << kv);
#pragma unroll
      for (int k = 0; k < W; k++)
        if (k < kv) {
          RW[k] = D;
          RG[k] = D;
        }
    }
    if (cand >= 0) {
      ci = i + 1;
      cj = reg_min(cj, j0 + cand + 1);
      blo = dlo;  // the live diagonals of rows i+1 .. ie
      bhi = dhi;
    }
    int outcome = -1;
    if (j0 > 0 && rh - o >= thr) outcome = kRegScanWide;  // a live state left of the window
    if (live) {
      dlo = reg_min(dlo, base + reg_ctz(live));
      dhi = reg_max(dhi, base + reg_hibit(live));
    }
    if (outcome < 0 && (!live || i == 0)) {
      if (ci > ie || cj > je || bhi < blo) {
        outcome = kRegScanNone;
      } else {
        outcome = kRegScanOk;
        blo = reg_max(blo, cj - ie);
        bhi = reg_min(bhi, je - ci);
      }
    }
    if (outcome < 0) {
      // the next row: its live states reach at most one slot further right (a vertical gap)
      const int kmin = reg_ctz(live), kmax = reg_hibit(live);
      int shift = 0;
      if (kmax >= W - 2) {
        if (kmin >= kRegShift) shift = kRegShift;
        else if (kmax == W - 1) outcome = kRegScanWide;
      } else if (kmin < 6 && kmax < W - kRegShift - 1 && j0 > 0) {
        shift = -kRegShift;
      }
      i--;
      if (shift > 0) {
#pragma unroll
        for (int k = 0; k < W; k++) {
          RW[k] = k + kRegShift < W ? RW[k + kRegShift] : D;
          RG[k] = k + kRegShift < W ? RG[k + kRegShift] : D;
        }
        base += kRegShift;
        load_codes();
      } else if (shift < 0) {
#pragma unroll
        for (int k = W - 1; k >= 0; k--) {
          RW[k] = k >= kRegShift ? RW[k - kRegShift] : D;
          RG[k] = k >= kRegShift ? RG[k - kRegShift] : D;
        }
        base -= kRegShift;
        load_codes();
      } else {
        // every slot's column moves one to the left: codes move up one slot
#pragma unroll
        for (int t = W / 4 - 1; t > 0; t--) cw[t] = reg_shl8(cw[t - 1], cw[t]);
        const int j = i + base;
        cw[0] = (cw[0] << 8) | ((j >= 0 && j < je) ? (uint32_t)b[j] : pad);
      }
    }
    if (outcome >= 0) {
      RegBox bx;
      bx.ci = ci;
      bx.cj = cj;
      bx.blo = blo;
      bx.bhi = bhi;
      emit(p, rec, outcome, bx);
      active = false;
      p += stride;
    }
  }
}

// Band DPs of the records list[idx[k * step]] for k = first, first + stride, ... below np (band
// width at most B); the scan's result of record r, (ci, cj, blo, bhi), is the first four words of
// its window win + r * kRegWinWords (the scan writes it there once the thresholds are used).
// scf[a * A1 + b] = S(a, b) << 8 | counted flag (a: an s1 residue of aseq, b: an s2 code of seq).
// emit(r, rec, ok, counters) receives each pair's
// outcome: ok with counters = aligned columns << 16 | counted columns, or not ok (the value at
// (ie, je) was not S).
template <int B, class Emit>
SWG_REG_FN void reg_band_run(const int* idx, long long step, long long first, long long np, long long stride,
                             const int4* list, const uint32_t* win, const uint8_t* aseq, const int64_t* aoff,
                             const uint8_t* seq, const int64_t* off, const int* scf, int A1, int o, int e,
                             Emit& emit) {
  constexpr int D = kRegDead;
  const uint32_t pad = (uint32_t)(A1 - 1);
  int V[B], G[B];
  uint32_t CV[B], CG[B];
  uint32_t cw[B / 4];
  long long p = first;
  bool active = false;
  int q = 0;
  int4 rec, bx;
  rec.x = rec.y = rec.z = rec.w = 0;
  bx = rec;
  const uint8_t* a = seq;
  const uint8_t* b = seq;
  int S = 0, ie = 0, je = 0, i = 0, blo = 0, bhi = 0, ci = 0, cj = 0;
  // codes of slots k..k+3 of row i: s2 residues of cells (i, i + blo + k), padding outside the box
  auto load_codes = [&]() {
#pragma unroll
    for (int t = 0; t < B / 4; t++) {
      uint32_t x = 0;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int j = i + blo + 4 * t + u;
        const uint32_t c = (j >= cj && j <= je) ? (uint32_t)b[j - 1] : pad;
        x |= c << (8 * u);
      }
      cw[t] = x;
    }
  };
  for (;;) {
    if (!active) {
      if (p >= np) break;
      q = idx[p * step];
      rec = list[q];
      bx = *reinterpret_cast<const int4*>(win + (long long)q * kRegWinWords);
      S = rec.z & 0xFFFF;
      ie = (int)((uint32_t)rec.w >> 16);
      je = rec.w & 0xFFFF;
      ci = bx.x;
      cj = bx.y;
      blo = bx.z;
      bhi = bx.w;
      a = aseq + aoff[rec.x];
      b = seq + off[rec.y];
#pragma unroll
      for (int k = 0; k < B; k++) {  // the row above the box: zero boundary
        V[k] = 0;
        G[k] = D;
        CV[k] = 0u;
        CG[k] = 0u;
      }
      i = ci;
      load_codes();
      active = true;
    }
    // ---- row i: slots from the left (columns ascending) ----
    const int j0 = i + blo;  // column of slot 0
    const int klo = cj - j0, khi = reg_min(je - j0, bhi - blo);  // the box's columns, the band
    const int* srow = scf + (int)a[i - 1] * A1;
    int vl = 0, hh = D;
    uint32_t cl = 0u, ch = 0u;
#pragma unroll
    for (int k = 0; k < B; k++) {
      const int c = (int)((cw[k >> 2] >> ((k & 3) * 8)) & 0xFFu);
      const int sf = srow[c];
      const int vd = V[k];
      const uint32_t cd = CV[k];
      const int vu = k + 1 < B ? V[k + 1] : 0;
      const int gu = k + 1 < B ? G[k + 1] : D;
      const uint32_t cvu = k + 1 < B ? CV[k + 1] : 0u;
      const uint32_t cgu = k + 1 < B ? CG[k + 1] : 0u;
      const int f = vd + (sf >> 8);
      const uint32_t cf = cd + 0x10000u + ((uint32_t)sf & 1u);
      const int g1 = gu - e, g2 = vu - o;
      const bool gext = g1 > g2;
      int g = gext ? g1 : g2;
      uint32_t cg = (gext ? cgu : cvu) + 0x10000u;
      const int h1 = hh - e, h2 = vl - o;
      const bool hext = h1 > h2;
      hh = hext ? h1 : h2;
      ch = (hext ? ch : cl) + 0x10000u;
      int v = reg_max(reg_max(f, g), reg_max(hh, 0));
      uint32_t cv = v == 0 ? 0u : v == f ? cf : v == g ? cg : ch;
      if (k < klo || k > khi) {  // outside the box or the band: the zero boundary
        v = 0;
        g = D;
        hh = D;
        cv = cg = ch = 0u;
      }
      V[k] = v;
      G[k] = g;
      CV[k] = cv;
      CG[k] = cg;
      vl = v;
      cl = cv;
    }
    if (i == ie) {
      // (ie, je) lies on the diagonal je - ie, in the band
      const int kje = je - ie - blo;
      int v = 0;
      uint32_t c = 0u;
#pragma unroll
      for (int k = 0; k < B; k++)
        if (k == kje) {
          v = V[k];
          c = CV[k];
        }
      emit(q, rec, v == S, c);
      active = false;
      p += stride;
    } else {
      i++;
      // every slot's column moves one to the right: codes move down one slot
#pragma unroll
      for (int t = 0; t + 1 < B / 4; t++) cw[t] = reg_shr8(cw[t], cw[t + 1]);
      const int j = i + blo + B - 1;
      cw[B / 4 - 1] = (cw[B / 4 - 1] >> 8) | (((j >= cj && j <= je) ? (uint32_t)b[j - 1] : pad) << 24);
    }
  }
}

}  // namespace swg
