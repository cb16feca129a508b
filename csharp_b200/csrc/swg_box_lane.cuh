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
// j % kLaneBand.  A pair is given up when the scan exceeds kLaneMaxRows rows or a row's live span
// exceeds kLaneWin columns, or the band exceeds kLaneBand diagonals or the box 254 rows + columns
// (the counters' range).
#pragma once
#include <cstdint>
#include <vector_types.h>

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

// Runs the two DPs for the pairs list[first], list[first + stride], ... below np, flattened into
// one loop whose every iteration does one cell (of the reverse scan or of the band DP) of the
// current pair: lanes of a warp that hold pairs of different shapes still issue the same loop body
// together, and a lane that finishes a pair takes its next one in the following iteration.  Each
// record is (s1 index, s2 index, S, ie << 16 | je) with 1 <= S <= 32767, 1 <= ie <= m and
// 1 <= je <= n; seq + off[k] are the residue codes of sequence k (indices into the tables' rows
// and columns, row stride A1); sc holds the substitution scores S(x, y) and fl the flags (bit 0 =
// counted column); o + e < 8192.  emit(record, reason, counters) receives every pair's outcome:
// reason 0 with counters = aligned << 8 | counted, or the reason the pair was given up: 1 scan
// rows, 2 scan window, 3 no first pair found, 4 band or box size (or S above max_score), 5 score.
template <class ScT, class FlT, class Emit>
SWG_LANE_FN void lane_box_run(const int4* list, long long first, long long np, long long stride,
                              const uint8_t* seq, const int64_t* off, const ScT* sc, const FlT* fl,
                              int A1, int o, int e, int max_score, LaneMem mem, Emit& emit) {
  constexpr int D = kLaneDead;
  constexpr int kFetch = 0, kScan = 1, kBand = 2;
  int phase = kFetch;
  long long p = first;
  int4 nrec;  // the next pair's record, loaded one pair ahead
  nrec.x = nrec.y = nrec.z = nrec.w = 0;
  if (p < np) nrec = list[p];
  int4 rec = nrec;
  const uint8_t* a = seq;
  const uint8_t* b = seq;
  int S = 0, ie = 0, je = 0;
  // reverse scan
  int i = 0, j = 0, lo = 0, hi = 0, nlo = 0, nhi = -1, rh = D, drw = D;
  int ci = 0, cj = 0, dlo = 0, dhi = 0, blo = 0, bhi = -1;
  bool first_pair = false;
  const ScT* srow = sc;
  // band DP
  int jl = 0, jr = -1, plo = 1, phi = 0, vl = 0, hh = D, vd = 0, vlast = 0;
  uint32_t cl = 0u, ch = 0u, cd = 0u, clast = 0u;
  const FlT* frow = fl;
  for (;;) {
    int rc = -1;  // >= 0: the current pair is finished with this outcome
    if (phase == kFetch) {
      if (p >= np) break;
      rec = nrec;
      if (p + stride < np) nrec = list[p + stride];
      S = rec.z;
      ie = (int)((uint32_t)rec.w >> 16);
      je = rec.w & 0xFFFF;
      if (S > max_score) {
        rc = 4;
      } else {
        a = seq + off[rec.x];
        b = seq + off[rec.y];
        lo = hi = je;
        mem[je % kLaneWin] = lane_pack(0, D);
        ci = cj = 1 << 30;
        dlo = dhi = je - ie;
        blo = 0;
        bhi = -1;
        i = ie - 1;
        j = hi;
        rh = drw = D;
        nlo = 0;
        nhi = -1;
        first_pair = false;
        srow = sc + (int)a[i] * A1;
        phase = kScan;
      }
    } else if (phase == kScan) {
      // cell (i, j) of the reverse scan
      if (nhi >= 0 && nhi - j >= kLaneWin) {
        rc = 2;  // the row's span would exceed the window
      } else {
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
        const bool row_end = (j < lo && rh < 0) || j == 0;
        j--;
        if (row_end) {
          if (first_pair) { blo = dlo; bhi = dhi; }  // the rows i+1 .. ie
          if (nhi >= 0 && i > 0) {
            lo = nlo;
            hi = nhi;
            dlo = lane_min(dlo, lo - i);
            dhi = lane_max(dhi, hi - i);
            i--;
            if (ie - i > kLaneMaxRows) {
              rc = 1;
            } else {
              j = hi;
              rh = drw = D;
              nlo = 0;
              nhi = -1;
              first_pair = false;
              srow = sc + (int)a[i] * A1;
            }
          } else if (ci > ie || cj > je || bhi < blo) {
            rc = 3;  // the scan is over: the box of the first pairs
          } else {
            const int h = ie - ci + 1, w = je - cj + 1;
            blo = lane_max(blo, cj - ie);
            bhi = lane_min(bhi, je - ci);
            if (bhi - blo + 1 > kLaneBand || h + w > 254) {
              rc = 4;
            } else {
              i = ci;
              plo = 1;
              phi = 0;
              jl = 1;
              jr = 0;
              j = 1;  // past the empty row: the row set-up below runs first
              phase = kBand;
            }
          }
        }
      }
    } else {
      // cell (i, j) of the band DP, after the set-up of row i when j has left the row
      if (j > jr) {
        if (jl <= jr) {  // the row just finished becomes the row above
          plo = jl;
          phi = jr;
          i++;
        }
        for (;;) {  // rows whose band lies outside the box are empty (never row ie)
          jl = lane_max(cj, i + blo);
          jr = lane_min(je, i + bhi);
          if (jl <= jr) break;
          plo = jl;
          phi = jr;
          i++;
        }
        const int arow = (int)a[i - 1] * A1;
        srow = sc + arow;
        frow = fl + arow;
        vl = 0;
        hh = D;
        vd = 0;
        cl = ch = cd = 0u;
        if (jl - 1 >= plo && jl - 1 <= phi) {
          const int k = (jl - 1) % kLaneBand;
          vd = lane_lo(mem[k]);
          cd = mem[kLaneBand + k] & 0xFFFFu;
        }
        j = jl;
      }
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
      j++;
      if (i == ie && j > jr) rc = (vlast == S) ? 0 : 5;  // (ie, je) was the last cell
    }
    if (rc >= 0) {
      emit(rec, rc, clast);
      phase = kFetch;
      p += stride;
    }
  }
}

}  // namespace swg
