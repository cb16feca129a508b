// Alignment strings for requested pairs (the reference's WriteAlignments output:
// Salsa.SmithWatermanMPI/Program.cs:223-246 and :545-556, Salsa.SmithWatermanMS/Program.cs:682-702,
// Salsa.NeedlemanWunschTPL/Program.cs:725-735).
//
// One thread per pair.  The thread runs the pair's DP row by row (the row above in global scratch)
// and keeps one decision byte per cell: the source of V (stop, diagonal, up, left, in the
// reference's priority) and whether the vertical / horizontal gap state extended its run (extend
// only when strictly better than reopening).  The traceback then walks from the start cell (the
// first maximum for local alignment, (m, n) for global) as SmithWatermanGotoh.Traceback does
// (SmithWatermanGotoh.cs:229-332): a diagonal step aligns two residues, an up or left step opens a
// gap run whose length is the number of consecutive extensions plus one -- the gap-size arrays of
// the reference hold exactly that count.  It writes both aligned strings ('-' for a gap) and the
// alignment's counts.
#include <cuda_runtime.h>
#include <cstdint>

#include "swg_device.cuh"
#include "swg_internal.h"

namespace swg {

enum : uint8_t { kDirStop = 0, kDirDiag = 1, kDirUp = 2, kDirLeft = 3, kGExt = 4, kHExt = 8 };

template <bool LOCAL>
__global__ void __launch_bounds__(128) traceback_kernel(TraceJob J) {
  __shared__ int16_t sc[kTable * kTable];
  for (int k = threadIdx.x; k < kTable * kTable; k += blockDim.x) sc[k] = J.scores[k];
  __syncthreads();
  const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= J.npairs) return;
  const int i1 = J.rows[tid], i2 = J.cols[tid];
  const uint8_t* s1 = J.seq + J.off[i1];
  const uint8_t* s2 = J.seq + J.off[i2];
  const int m = (int)(J.off[i1 + 1] - J.off[i1]), n = (int)(J.off[i2 + 1] - J.off[i2]);
  uint8_t* dir = J.dirs + tid * J.dir_stride;
  int* V = J.vrow + tid * (long)J.row_stride;
  int* G = V + (J.row_stride >> 1);
  TraceResult r;
  r.score = 0; r.valid = 1; r.end1 = r.end2 = r.start1 = r.start2 = 0;
  r.identity = r.similarity = r.gaps = r.length = r.diag = r.transitions = r.transversions = 0;
  char* a1 = J.aln1 + J.out_off[tid];
  char* a2 = J.aln2 + J.out_off[tid];
  if (m == 0 || n == 0) {
    if (LOCAL) {  // Cell.Score stays -infinity: the alignment is empty
      r.valid = 0;
    } else {      // one gap run along the boundary
      for (int k = 0; k < m; k++) { a1[k] = (char)s1[k]; a2[k] = '-'; }
      for (int k = 0; k < n; k++) { a1[k] = '-'; a2[k] = (char)s2[k]; }
      r.length = r.gaps = m + n;
      r.score = (m + n) ? -J.o - (m + n - 1) * J.e : 0;
      r.end1 = m; r.end2 = n;
    }
    J.out[tid] = r;
    return;
  }
  // ---- the DP with a decision byte per cell (rows 1..m, columns 1..n) ----
  for (int j = 0; j <= n; j++) {
    V[j] = LOCAL ? 0 : (j == 0 ? 0 : -J.o - (j - 1) * J.e);
    G[j] = kNegInf;
  }
  int best = kNegInf, bi = 0, bj = 0;
  for (int i = 1; i <= m; i++) {
    const int arow = (int)s1[i - 1] * kTable;
    int vdiag = V[0];
    int vleft = LOCAL ? 0 : -J.o - (i - 1) * J.e;
    V[0] = vleft;
    int h = kNegInf;
    uint8_t* drow = dir + (long)(i - 1) * n;
    for (int j = 1; j <= n; j++) {
      const int f = vdiag + sc[arow + s2[j - 1]];
      const int g1 = G[j] - J.e, g2 = V[j] - J.o;
      const bool gext = g1 > g2;
      const int g = gext ? g1 : g2;
      const int h1 = h - J.e, h2 = vleft - J.o;
      const bool hext = h1 > h2;
      h = hext ? h1 : h2;
      int v = max(max(f, g), h);
      if (LOCAL) v = max(v, 0);
      uint8_t d = (LOCAL && v == 0) ? kDirStop : v == f ? kDirDiag : v == g ? kDirUp : kDirLeft;
      d |= (gext ? kGExt : 0) | (hext ? kHExt : 0);
      drow[j - 1] = d;
      vdiag = V[j];
      V[j] = v;
      G[j] = g;
      vleft = v;
      if (LOCAL && v > best) { best = v; bi = i; bj = j; }
    }
  }
  if (!LOCAL) { best = V[n]; bi = m; bj = n; }
  r.score = best;
  r.end1 = bi;
  r.end2 = bj;
  // ---- traceback, reversed strings first ----
  int i = bi, j = bj, len = 0;
  int state = 0;  // 0: V, 1: vertical gap run, 2: horizontal gap run
  while (LOCAL ? true : (i > 0 || j > 0)) {
    if (LOCAL && (i == 0 || j == 0)) break;  // row 0 and column 0 hold STOP
    if (!LOCAL && (i == 0 || j == 0)) {  // global: the rest is one gap run along the boundary
      if (i > 0) { a1[len] = (char)s1[--i]; a2[len] = '-'; len++; r.gaps++; continue; }
      a1[len] = '-'; a2[len] = (char)s2[--j]; len++; r.gaps++;
      continue;
    }
    const uint8_t d = dir[(long)(i - 1) * n + (j - 1)];
    if (state == 0) {
      const uint8_t src = d & 3;
      if (src == kDirStop) break;
      if (src == kDirDiag) {
        const uint8_t x = s1[--i], y = s2[--j];
        a1[len] = (char)x; a2[len] = (char)y; len++;
        r.diag++;
        if (x == y) r.identity++;
        if (x == y || sc[(int)x * kTable + y] > 0) r.similarity++;
        const bool ts = (x == 'A' && y == 'G') || (x == 'G' && y == 'A') || (x == 'C' && y == 'T') || (x == 'T' && y == 'C');
        if (ts) r.transitions++;
        else if (x != y) r.transversions++;
        continue;
      }
      state = src == kDirUp ? 1 : 2;
    }
    if (state == 1) {  // this cell's vertical gap state: one row of s1 against a gap
      a1[len] = (char)s1[i - 1]; a2[len] = '-'; len++; r.gaps++;
      if (!(d & kGExt)) state = 0;
      i--;
    } else {
      a1[len] = '-'; a2[len] = (char)s2[j - 1]; len++; r.gaps++;
      if (!(d & kHExt)) state = 0;
      j--;
    }
  }
  r.start1 = i;
  r.start2 = j;
  r.length = len;
  for (int k = 0; k < len / 2; k++) {
    const char x = a1[k], y = a2[k];
    a1[k] = a1[len - 1 - k]; a2[k] = a2[len - 1 - k];
    a1[len - 1 - k] = x; a2[len - 1 - k] = y;
  }
  J.out[tid] = r;
}

size_t trace_scratch_bytes(int m, int n) {
  return (size_t)m * n + 2 * sizeof(int) * ((size_t)n + 1);
}

cudaError_t launch_traceback(const TraceJob& J, bool local, cudaStream_t st) {
  if (J.npairs <= 0) return cudaSuccess;
  const int block = 128;
  const int grid = (int)((J.npairs + block - 1) / block);
  if (local) traceback_kernel<true><<<grid, block, 0, st>>>(J);
  else traceback_kernel<false><<<grid, block, 0, st>>>(J);
  return cudaGetLastError();
}

}  // namespace swg
