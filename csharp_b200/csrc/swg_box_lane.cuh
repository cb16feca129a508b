// Box step of the two-pass SW-Gotoh path, one pair per thread.
//
// The first pass gives, per pair, the best score S and the reference's traceback start cell
// (ie, je) (the first maximum in row-major order, SmithWatermanGotoh.cs:211-214).  The counters of
// the traceback path (identity and aligned columns, Traceback :229-332) are found here from two
// small DPs, both local to the neighbourhood of (ie, je):
//
//  1. Reverse scan.  RW(i, j) = best score of a path from the V state after consuming i residues
//     of s1 and j of s2 to the V state at (ie, je); RG / RH the same from the vertical /
//     horizontal gap states:
//        RW(i,j) = max(S(s1[i], s2[j]) + RW(i+1,j+1), RG(i+1,j) - o, RH(i,j+1) - o)
//        RG(i,j) = max(RW(i,j), RG(i+1,j) - e),   RH(i,j) = max(RW(i,j), RH(i,j+1) - e)
//     with RW(ie, je) = 0.  Every state on an alignment of score S ending at (ie, je) has a
//     completion score >= 0 (its prefix scores at most S there), so states below 0 are pruned.
//     The first aligned pair of such an alignment is a cell (i+1, j+1) with
//     S(s1[i], s2[j]) + RW(i+1, j+1) == S; the smallest row and column of all of them bound a box
//     that holds every optimal alignment ending at (ie, je), the traceback's among them.
//  2. Band DP.  The local Gotoh DP with counters, in the reference's comparison order, on the
//     cells of that box that lie on the diagonals (j - i) its rows' live states span, with a zero
//     boundary (V = 0, gaps -infinity, counters 0) outside them.  Every cell of those alignments
//     is live (a gap run lies between two live cells of its row or column), so the region holds
//     the traceback path.  Along that path every value equals the full matrix's (the path is
//     inside the region, and values inside never exceed the full matrix's), and each pointer and
//     gap-size decision on the path compares path values against values no larger than the full
//     matrix's, so the band DP follows the same path and its counters at (ie, je) are the
//     traceback's.  The value at (ie, je) must come out as S; anything else gives up.
//
// Scratch per thread: kLaneWords 32-bit words, word k at base[k * stride] (the kernel interleaves
// threads so a warp's accesses hit 32 distinct banks).  The reverse scan keeps row i+1's RW | RG
// (two int16) in word j % kLaneWin; the band DP keeps the row above's V | G and its two 16-bit
// counter words (aligned << 8 | counted) of column j in words j % kLaneBand and kLaneBand +
// j % kLaneBand.  The pair is given up (nonzero return) when the scan exceeds kLaneMaxRows rows or
// a row's live span exceeds kLaneWin columns, or the band exceeds kLaneBand diagonals or the box
// 254 rows + columns (the counters' range).
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define SWG_LANE_FN __host__ __device__ __forceinline__
#else
#define SWG_LANE_FN inline
#endif

namespace swg {

constexpr int kLaneWin = 64;       // reverse-scan window (columns)
constexpr int kLaneBand = 48;      // band DP: diagonals
constexpr int kLaneMaxRows = 400;  // reverse-scan rows
constexpr int kLaneWords = 96;     // words per thread: max(kLaneWin, 2 * kLaneBand)
constexpr int kLaneDead = -16384;  // pruned / -infinity state
constexpr uint32_t kLaneFlagCount = 1u;  // counted-column bit of the flag table

static_assert(kLaneWords >= kLaneWin && kLaneWords >= 2 * kLaneBand, "lane scratch");

struct LaneMem {
  uint32_t* base;
  int stride;
  SWG_LANE_FN uint32_t& operator[](int k) const {
#ifdef SWG_LANE_CHECK
    if (k < 0 || k >= kLaneWords) swg_lane_check_failed(k);
#endif
    return base[(long)k * stride];
  }
};

SWG_LANE_FN uint32_t lane_pack(int lo, int hi) {
  return (uint32_t)(uint16_t)(int16_t)lo | ((uint32_t)(uint16_t)(int16_t)hi << 16);
}
SWG_LANE_FN int lane_lo(uint32_t w) { return (int)(int16_t)(uint16_t)(w & 0xFFFFu); }
SWG_LANE_FN int lane_hi(uint32_t w) { return (int)(int16_t)(uint16_t)(w >> 16); }
SWG_LANE_FN int lane_max(int a, int b) { return a > b ? a : b; }
SWG_LANE_FN int lane_min(int a, int b) { return a < b ? a : b; }

// a, b: residue codes of s1 and s2 (indices into the tables' rows and columns, row stride A1);
// sc: substitution scores S(x, y); fl: flags (bit 0 = counted column).  Requires 1 <= S <= 32767,
// 1 <= ie <= m, 1 <= je <= n, o + e < 8192.  Returns 0 with *cnt = aligned << 8 | counted, or the
// reason it gave up: 1 scan rows, 2 scan window, 3 no first pair found, 4 band or box size,
// 5 score.
template <class ScT, class FlT>
SWG_LANE_FN int lane_box_pair(const uint8_t* a, const uint8_t* b, int S, int ie, int je, const ScT* sc,
                              const FlT* fl, int A1, int o, int e, LaneMem mem, uint32_t* cnt) {
  constexpr int D = kLaneDead;
  // ---- reverse scan, rows ie-1 .. 0; [lo, hi] = live columns of the row below ----
  int lo = je, hi = je;
  mem[je % kLaneWin] = lane_pack(0, D);
  int ci = 1 << 30, cj = 1 << 30;
  // diagonals (j - i) spanned by the live states of the rows below the current one, and their
  // value when the topmost first pair so far was found (the band of the rows ci..ie)
  int dlo = je - ie, dhi = je - ie, blo = 0, bhi = -1;
  for (int i = ie - 1; i >= 0; i--) {
    if (ie - i > kLaneMaxRows) return 1;
    const ScT* srow = sc + (int)a[i] * A1;
    int rh = D;   // RH(i, j+1)
    int drw = D;  // RW(i+1, j+1)
    int nlo = 0, nhi = -1;
    bool first_pair = false;
    for (int j = hi; j >= 0; j--) {
      if (nhi >= 0 && nhi - j >= kLaneWin) return 2;  // the row's span would exceed the window
      int rwb = D, rgb = D;
      if (j >= lo) {
        const uint32_t w = mem[j % kLaneWin];
        rwb = lane_lo(w);
        rgb = lane_hi(w);
      }
      int x = rgb - o;
      if (drw >= 0) {
        const int pr = (int)srow[b[j]] + drw;
        if (pr == S) {
          ci = lane_min(ci, i + 1);
          cj = lane_min(cj, j + 1);
          first_pair = true;
        }
        x = lane_max(x, pr);
      }
      int rw = lane_max(x, rh - o);
      rh = lane_max(rw, rh - e);
      int rg = lane_max(rw, rgb - e);
      if (rw < 0) rw = D;
      if (rg < 0) rg = D;
      if (rh < 0) rh = D;
      mem[j % kLaneWin] = lane_pack(rw, rg);
      if (rw >= 0 || rg >= 0) {
        nlo = j;
        if (nhi < 0) nhi = j;
      }
      drw = rwb;
      if (j < lo && rh < 0) break;  // nothing further left in this row can be live
    }
    if (first_pair) { blo = dlo; bhi = dhi; }  // the rows i+1 .. ie
    if (nhi < 0) break;  // no live state: nothing above can reach (ie, je)
    lo = nlo;
    hi = nhi;
    dlo = lane_min(dlo, lo - i);
    dhi = lane_max(dhi, hi - i);
  }
  if (ci > ie || cj > je || bhi < blo) return 3;
  const int h = ie - ci + 1, w = je - cj + 1;
  blo = lane_max(blo, cj - ie);  // clipped to the box's own diagonals
  bhi = lane_min(bhi, je - ci);
  if (bhi - blo + 1 > kLaneBand || h + w > 254) return 4;
  // ---- band DP: rows ci..ie, columns cj..je with blo <= j - i <= bhi, zero boundary ----
  int vlast = 0;
  uint32_t clast = 0u;
  int plo = 1, phi = 0;  // columns of the row above (none: the top boundary)
  for (int i = ci; i <= ie; i++) {
    const int jl = lane_max(cj, i + blo), jr = lane_min(je, i + bhi);
    const int arow = (int)a[i - 1] * A1;
    const ScT* srow = sc + arow;
    const FlT* frow = fl + arow;
    int vl = 0, hh = D, vd = 0;
    uint32_t cl = 0u, ch = 0u, cd = 0u;
    if (jl - 1 >= plo && jl - 1 <= phi) {
      const int k = (jl - 1) % kLaneBand;
      vd = lane_lo(mem[k]);
      cd = mem[kLaneBand + k] & 0xFFFFu;
    }
    for (int j = jl; j <= jr; j++) {
      const int k = j % kLaneBand;
      int vu = 0, gu = D;
      uint32_t cvu = 0u, cgu = 0u;
      if (j >= plo && j <= phi) {
        const uint32_t wv = mem[k], wc = mem[kLaneBand + k];
        vu = lane_lo(wv);
        gu = lane_hi(wv);
        cvu = wc & 0xFFFFu;
        cgu = wc >> 16;
      }
      const int y = b[j - 1];
      const int f = vd + (int)srow[y];
      const uint32_t cf = cd + 0x100u + ((uint32_t)frow[y] & kLaneFlagCount);
      const int g1 = gu - e, g2 = vu - o;
      int g;
      uint32_t cg;
      if (g1 > g2) { g = g1; cg = cgu + 0x100u; } else { g = g2; cg = cvu + 0x100u; }
      const int h1 = hh - e, h2 = vl - o;
      if (h1 > h2) { hh = h1; ch = ch + 0x100u; } else { hh = h2; ch = cl + 0x100u; }
      const int v = lane_max(lane_max(f, g), lane_max(hh, 0));
      const uint32_t cv = (v == 0) ? 0u : (v == f) ? cf : (v == g) ? cg : ch;
      mem[k] = lane_pack(v, lane_max(g, D));
      mem[kLaneBand + k] = cv | (cg << 16);
      vd = vu;
      cd = cvu;
      vl = v;
      cl = cv;
      vlast = v;
      clast = cv;
    }
    plo = jl;
    phi = jr;
  }
  if (vlast != S) return 5;
  *cnt = clast;
  return 0;
}

}  // namespace swg
