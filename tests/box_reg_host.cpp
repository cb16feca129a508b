// Host build of the two-pass box step (csharp_b200/csrc/swg_box_reg.cuh) for the CPU tests: the
// same source the box_scan_kernel and box_band_kernel run, driven for a list of pairs as `threads`
// emulated lanes (lane t takes pairs t, t + threads, ...).  The first pass's outputs (best score,
// first-maximum cell, row bounds) come from a plain forward DP here; `slack` > 0 loosens each row
// bound by a pseudo-random amount in [0, slack] (any bound >= the row's maximum must give the
// same counters).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../csharp_b200/csrc/swg_box_reg.cuh"

namespace {

// Forward SW-Gotoh scores of one pair (codes are residue bytes, table 128 x 128): best score,
// its first cell in row-major order (1-based) and each row's maximum V (row 0 = 0).
void forward(const uint8_t* a, int m, const uint8_t* b, int n, const int32_t* sc, int o, int e, int* S,
             int* ie, int* je, std::vector<int>& rowmax) {
  const int NEG = -(1 << 28);
  std::vector<int> V(n + 1, 0), G(n + 1, NEG);
  rowmax.assign(m + 1, 0);
  *S = NEG;
  *ie = *je = 0;
  for (int i = 1; i <= m; i++) {
    int vdiag = 0, vleft = 0, h = NEG, rm = 0;
    for (int j = 1; j <= n; j++) {
      const int f = vdiag + sc[a[i - 1] * 128 + b[j - 1]];
      const int g1 = G[j] - e, g2 = V[j] - o;
      G[j] = g1 > g2 ? g1 : g2;
      const int h1 = h - e, h2 = vleft - o;
      h = h1 > h2 ? h1 : h2;
      int v = f;
      if (G[j] > v) v = G[j];
      if (h > v) v = h;
      if (v < 0) v = 0;
      vdiag = V[j];
      V[j] = v;
      vleft = v;
      if (v > rm) rm = v;
      if (v > *S) {
        *S = v;
        *ie = i;
        *je = j;
      }
    }
    rowmax[i] = rm;
  }
}

}  // namespace

// outcome: 0 solved (counters = aligned << 16 | counted), 1 the scan's window was too narrow,
// 2 no first pair, 3 band wider than 32 diagonals, 4 band DP value not S, 5 not a box pair
// (empty or S <= 0); S / ie / je receive the forward DP's best score and cell.
extern "C" int box_reg_run(const uint8_t* seqs, const int64_t* off, const int32_t* q, const int32_t* d, long np,
                           const int32_t* scores, const uint32_t* flags, int o, int e, int threads, int slack,
                           int32_t* S_out, int32_t* ie_out, int32_t* je_out, int32_t* outcome, uint32_t* counters,
                           int32_t* band_width) {
  const int A1 = 128;
  std::vector<int32_t> sc(A1 * A1), scf(A1 * A1);
  for (int a = 0; a < A1; a++)
    for (int b = 0; b < A1; b++) {
      const bool pad = a == A1 - 1 || b == A1 - 1;
      const int s = pad ? swg::kRegPadScore : scores[a * 128 + b];
      sc[a * A1 + b] = s;
      scf[a * A1 + b] = (int32_t)((uint32_t)s << 8) | (int32_t)(pad ? 0u : (flags[a * 128 + b] & 1u));
    }
  std::vector<int4> list;
  std::vector<uint32_t> win;
  std::vector<long> src;  // list entry -> pair
  uint32_t rng = 12345u;
  std::vector<int> rowmax;
  for (long p = 0; p < np; p++) {
    const uint8_t* a = seqs + off[q[p]];
    const uint8_t* b = seqs + off[d[p]];
    const int m = (int)(off[q[p] + 1] - off[q[p]]), n = (int)(off[d[p] + 1] - off[d[p]]);
    int S = 0, ie = 0, je = 0;
    outcome[p] = 5;
    counters[p] = 0;
    band_width[p] = 0;
    S_out[p] = ie_out[p] = je_out[p] = 0;
    if (m == 0 || n == 0) continue;
    forward(a, m, b, n, scores, o, e, &S, &ie, &je, rowmax);
    S_out[p] = S;
    ie_out[p] = ie;
    je_out[p] = je;
    if (S <= 0) continue;
    auto bound = [&](int i) {
      int u = i >= 1 ? rowmax[i] : 0;
      if (slack > 0) {
        rng = rng * 1664525u + 1013904223u;
        u += (int)((rng >> 8) % (uint32_t)(slack + 1));
      }
      return u;
    };
    uint32_t w[swg::kRegWinWords] = {};
    for (int k = 0; k < swg::kRegWinRows; k++) {
      const int i = ie - 1 - k;
      const int u = i >= 0 ? bound(i) : 0;
      const int t = S - (u < S ? u : S);
      w[k >> 3] |= (uint32_t)swg::reg_code_of(t) << ((k & 7) * 4);
    }
    int umax = 0;
    for (int i = 0; i <= ie - 1 - swg::kRegWinRows; i++) {
      const int u = bound(i);
      if (u > umax) umax = u;
    }
    const int trest = S - (umax < S ? umax : S);
    int4 r;
    r.x = q[p];
    r.y = d[p];
    r.z = S | (trest << 16);
    r.w = (int)(((uint32_t)ie << 16) | (uint32_t)je);
    list.push_back(r);
    win.insert(win.end(), w, w + swg::kRegWinWords);
    src.push_back(p);
  }
  const long nl = (long)list.size();
  std::vector<std::vector<int>> cls(4);
  int dup = 0;
  std::vector<char> seen(nl > 0 ? nl : 1, 0);
  for (int t = 0; t < threads; t++) {
    auto emit = [&](long long p, const int4&, int rc, const swg::RegBox& bx) {
      if (p < 0 || p >= nl || seen[p]) {
        dup = 1;
        return;
      }
      seen[p] = 1;
      const long pp = src[p];
      if (rc != swg::kRegScanOk) {
        outcome[pp] = rc;
        return;
      }
      const int bw = bx.bhi - bx.blo + 1;
      band_width[pp] = bw;
      int4 v;
      v.x = bx.ci;
      v.y = bx.cj;
      v.z = bx.blo;
      v.w = bx.bhi;
      memcpy(&win[p * swg::kRegWinWords], &v, sizeof(v));  // as the scan kernel stores it
      if (bw > 32) {
        outcome[pp] = 3;
        return;
      }
      cls[bw <= 8 ? 0 : bw <= 16 ? 1 : bw <= 24 ? 2 : 3].push_back((int)p);
    };
    swg::reg_scan_run(list.data(), win.data(), t, nl, threads, seqs, off, seqs, off, sc.data(), A1, o, e, emit);
  }
  for (long p = 0; p < nl; p++)
    if (!seen[p]) dup = 1;
  std::vector<char> done(nl > 0 ? nl : 1, 0);
  for (int c = 0; c < 4; c++) {
    const long nc = (long)cls[c].size();
    for (int t = 0; t < threads; t++) {
      auto emit = [&](int qi, const int4&, bool ok, uint32_t cnt) {
        if (qi < 0 || qi >= nl || done[qi]) {
          dup = 1;
          return;
        }
        done[qi] = 1;
        outcome[src[qi]] = ok ? 0 : 4;
        counters[src[qi]] = cnt;
      };
      switch (c) {
        case 0: swg::reg_band_run<8>(cls[c].data(), 1, t, nc, threads, list.data(), win.data(), seqs, off, seqs, off, scf.data(), A1, o, e, emit); break;
        case 1: swg::reg_band_run<16>(cls[c].data(), 1, t, nc, threads, list.data(), win.data(), seqs, off, seqs, off, scf.data(), A1, o, e, emit); break;
        case 2: swg::reg_band_run<24>(cls[c].data(), 1, t, nc, threads, list.data(), win.data(), seqs, off, seqs, off, scf.data(), A1, o, e, emit); break;
        default: swg::reg_band_run<32>(cls[c].data(), 1, t, nc, threads, list.data(), win.data(), seqs, off, seqs, off, scf.data(), A1, o, e, emit); break;
      }
    }
  }
  return dup;
}
