// Device-side building blocks shared by the alignment kernels.
//
// The recurrences are those of SmithWatermanGotoh.Construct (SalsaTPL/Salsa.CoreTPL/Bio/
// Algorithms/SmithWaterman/SmithWatermanGotoh.cs:119-219), evaluated on integers: with integer
// substitution scores and penalties every float the reference computes is an exact small
// integer, so int32 (or range-checked int16) arithmetic reproduces it bit for bit.
//
//   G(i,j) (vertical gap, consumes s1)  = G(i-1,j)-e  if that is strictly greater than V(i-1,j)-o
//   H(i,j) (horizontal gap, consumes s2) = H(i,j-1)-e if strictly greater than V(i,j-1)-o
//   F(i,j) = V(i-1,j-1) + S(s1[i-1], s2[j-1])
//   V(i,j) = max(F, G, H, 0)            (local; global alignment drops the 0)
//   pointer priority STOP (V == 0) > DIAGONAL (V == F) > UP (V == G) > LEFT
//   traceback start = first V strictly greater than all before it in row-major order
//
// Instead of the reference's direction and gap-size matrices plus Traceback (:229-332), every
// state carries the counters of the path that reaches it ("in-DP" bookkeeping): the gap-size
// arrays follow exactly the G/H extension chains, so the counters of the traceback start cell
// equal what the traceback would count.
#pragma once
#include <cstdint>

#include "swg_log.cuh"

namespace swg {

constexpr int kNegInf = -(1 << 28);  // -infinity of the float DP (only ever loses a max)
constexpr int kPadCode = 127;        // residue code of padding rows/columns
constexpr int kPadScore = -16384;    // score of any pair involving kPadCode
constexpr int kTable = 128;          // substitution tables are [128][128]

// Bits of the per-(c1,c2) flag table.
constexpr uint32_t kFlagCount = 1u;  // the context's counted column (identity or similarity)
constexpr uint32_t kFlagIdent = 2u;  // c1 == c2
constexpr uint32_t kFlagSimNA = 4u;  // NAligner similarity: c1 == c2 or S > 0
constexpr uint32_t kFlagCntA = 8u;   // Kimura2: transition (A<->G, C<->T); JukesCantor: c1 == c2
constexpr uint32_t kFlagCntB = 16u;  // Kimura2: transversion (any other mismatch)

// ---- counter policies --------------------------------------------------------------------------
// SwCnt: one 32-bit word, aligned columns in bits 16..31, counted columns in bits 0..15.
struct SwCnt {
  typedef uint32_t T;
  __device__ __forceinline__ static T stop(int, int) { return 0u; }
  __device__ __forceinline__ static T origin() { return 0u; }
  __device__ __forceinline__ static T row0(int) { return 0u; }
  __device__ __forceinline__ static T col0(int) { return 0u; }
  __device__ __forceinline__ static T diag(T c, uint32_t fl) { return c + 0x10000u + (fl & kFlagCount); }
  __device__ __forceinline__ static T up_ext(T c) { return c + 0x10000u; }
  __device__ __forceinline__ static T up_open(T c) { return c + 0x10000u; }
  __device__ __forceinline__ static T left_ext(T c) { return c + 0x10000u; }
  __device__ __forceinline__ static T left_open(T c) { return c + 0x10000u; }
};

// NwCnt: global alignment.  w0 as SwCnt; w1 = leading same-type gap run (bits 16..31) and the
// signed length of the current trailing gap run (bits 0..15: +k = k UP columns, -k = k LEFT
// columns, 0 after a DIAGONAL column).  With open > extend a gap never reopens right after a
// gap of the same type, so an UP run is exactly the current G chain.
struct NwCnt {
  struct T { uint32_t w0, w1; };
  __device__ __forceinline__ static T origin() { return T{0u, 0u}; }
  __device__ __forceinline__ static T stop(int, int) { return T{0u, 0u}; }
  // V(i,0): i UP columns from (0,0); V(0,j): j LEFT columns.
  __device__ __forceinline__ static T col0(int i) { return T{(uint32_t)i << 16, ((uint32_t)i << 16) | (uint32_t)(i & 0xFFFF)}; }
  __device__ __forceinline__ static T row0(int j) { return T{(uint32_t)j << 16, ((uint32_t)j << 16) | (uint32_t)((-j) & 0xFFFF)}; }
  __device__ __forceinline__ static T diag(T c, uint32_t fl) { return T{c.w0 + 0x10000u + (fl & kFlagCount), c.w1 & 0xFFFF0000u}; }
  __device__ __forceinline__ static T up_ext(T c) { return T{c.w0 + 0x10000u, c.w1 + 1u}; }
  __device__ __forceinline__ static T up_open(T c) { return T{c.w0 + 0x10000u, (c.w1 & 0xFFFF0000u) | 1u}; }
  __device__ __forceinline__ static T left_ext(T c) { return T{c.w0 + 0x10000u, c.w1 - 1u}; }
  __device__ __forceinline__ static T left_open(T c) { return T{c.w0 + 0x10000u, (c.w1 & 0xFFFF0000u) | 0xFFFFu}; }
};

// KimCnt: the Kimura2 / JukesCantor counts of the aligned strings (Alignment.cs:254-348).
// w0 = aligned columns << 16 | A-flagged columns, w1 = diagonal (non-gap) columns << 16 |
// B-flagged columns, with A/B = transitions/transversions (Kimura2) or identical/none
// (JukesCantor), as the flag table marks them.
struct KimCnt {
  struct T { uint32_t w0, w1; };
  __device__ __forceinline__ static T origin() { return T{0u, 0u}; }
  __device__ __forceinline__ static T stop(int, int) { return T{0u, 0u}; }
  __device__ __forceinline__ static T row0(int) { return T{0u, 0u}; }
  __device__ __forceinline__ static T col0(int) { return T{0u, 0u}; }
  __device__ __forceinline__ static T diag(T c, uint32_t fl) {
    return T{c.w0 + 0x10000u + ((fl >> 3) & 1u), c.w1 + 0x10000u + ((fl >> 4) & 1u)};
  }
  __device__ __forceinline__ static T up_ext(T c) { return T{c.w0 + 0x10000u, c.w1}; }
  __device__ __forceinline__ static T up_open(T c) { return T{c.w0 + 0x10000u, c.w1}; }
  __device__ __forceinline__ static T left_ext(T c) { return T{c.w0 + 0x10000u, c.w1}; }
  __device__ __forceinline__ static T left_open(T c) { return T{c.w0 + 0x10000u, c.w1}; }
};

// FullCnt: every PairwiseAlignment field the path reads, for the single-pair aligner, plus the
// transition / transversion counts of Kimura2.
struct FullCnt {
  struct T { int id, sim, len, si, sj, diag, ts, tv; };
  __device__ __forceinline__ static T stop(int i, int j) { return T{0, 0, 0, i, j, 0, 0, 0}; }
  __device__ __forceinline__ static T origin() { return T{0, 0, 0, 0, 0, 0, 0, 0}; }
  __device__ __forceinline__ static T row0(int j) { return T{0, 0, 0, 0, j, 0, 0, 0}; }
  __device__ __forceinline__ static T col0(int i) { return T{0, 0, 0, i, 0, 0, 0, 0}; }
  __device__ __forceinline__ static T diag(T c, uint32_t fl) {
    return T{c.id + (int)((fl >> 1) & 1u), c.sim + (int)((fl >> 2) & 1u), c.len + 1, c.si, c.sj,
             c.diag + 1, c.ts + (int)((fl >> 3) & 1u), c.tv + (int)((fl >> 4) & 1u)};
  }
  __device__ __forceinline__ static T up_ext(T c) { c.len++; return c; }
  __device__ __forceinline__ static T up_open(T c) { c.len++; return c; }
  __device__ __forceinline__ static T left_ext(T c) { c.len++; return c; }
  __device__ __forceinline__ static T left_open(T c) { c.len++; return c; }
};

// One cell of the Gotoh recurrence with counters, in the reference's comparison order.
template <bool LOCAL, class CP>
__device__ __forceinline__ void gotoh_cell(int s, uint32_t fl, int vd, typename CP::T cd, int vu,
                                           int gu, typename CP::T cvu, typename CP::T cgu, int vl,
                                           typename CP::T cl, int& h, typename CP::T& ch, int o,
                                           int e, int i, int j, int& v, int& g,
                                           typename CP::T& cv, typename CP::T& cg) {
  const int f = vd + s;
  const typename CP::T cf = CP::diag(cd, fl);
  const int g1 = gu - e, g2 = vu - o;
  const bool gext = g1 > g2;
  g = gext ? g1 : g2;
  cg = gext ? CP::up_ext(cgu) : CP::up_open(cvu);
  const int h1 = h - e, h2 = vl - o;
  const bool hext = h1 > h2;
  h = hext ? h1 : h2;
  ch = hext ? CP::left_ext(ch) : CP::left_open(cl);
  if (LOCAL) {
    v = max(max(f, g), max(h, 0));
    cv = (v == 0) ? CP::stop(i, j) : (v == f) ? cf : (v == g) ? cg : ch;
  } else {
    v = max(max(f, g), h);
    cv = (v == f) ? cf : (v == g) ? cg : ch;
  }
}

// .NET x64 conv.i2 of a float: truncation toward zero through int32 (NaN and out-of-range
// values become 0x80000000), then the low 16 bits.
__device__ __forceinline__ int16_t cs_conv_i2(float x) {
  if (!(x > -2147483648.0f && x < 2147483648.0f)) return 0;
  return (int16_t)__float2int_rz(x);
}

// (short)((1.0f - count / (len * 1.0f)) * short.MaxValue) in IEEE binary32 round-to-nearest
// (PercentIdentity/PercentSimilarity, Alignment.cs:187-195; ComputeDistance Program.cs:259-285).
__device__ __forceinline__ int16_t fraction_distance(int count, int len) {
  const float p = __fdiv_rn(__int2float_rn(count), __int2float_rn(len));
  return cs_conv_i2(__fmul_rn(__fsub_rn(1.0f, p), 32767.0f));
}

// .NET x64 conv.i2 of a double (cvttsd2si to int32, then the low 16 bits).
__device__ __forceinline__ int16_t cs_conv_i2_d(double x) {
  if (!(x > -2147483649.0 && x < 2147483648.0)) return 0;
  return (int16_t)(uint16_t)(uint32_t)__double2int_rz(x);
}

constexpr double kDoubleEpsilon = 4.9406564584124654e-324;  // System.Double.Epsilon

// Kimura2 (Alignment.cs:254-302) of an alignment with len columns, diag of them non-gap, ts
// transitions and tv transversions; in binary64 without contraction, like the reference.
__device__ __forceinline__ double kimura2_value(int len, int diag, int ts, int tv) {
  const double length = (double)len, gapc = (double)(len - diag);
  const double P = __ddiv_rn((double)ts, __dsub_rn(length, gapc));
  const double Q = __ddiv_rn((double)tv, __dsub_rn(length, gapc));
  if (__dsub_rn(1.0, __dadd_rn(__dmul_rn(2.0, P), Q)) <= kDoubleEpsilon) return 10.0;
  if (__dsub_rn(1.0, __dmul_rn(2.0, Q)) <= kDoubleEpsilon) return 10.0;
  return __dsub_rn(__dmul_rn(-0.5, cr_log(__dsub_rn(__dsub_rn(1.0, __dmul_rn(2.0, P)), Q))),
                   __dmul_rn(0.25, cr_log(__dsub_rn(1.0, __dmul_rn(2.0, Q)))));
}

// JukesCantor (Alignment.cs:314-348): 1 - (4/3)(diff / non-gap columns); false where the
// reference's log would see a value <= Double.Epsilon (it throws "Log(Zero)").
__device__ __forceinline__ bool jukes_cantor_value(int len, int diag, int identical, double* out) {
  const double length = (double)len, gapc = (double)(len - diag);
  const double d = __dsub_rn(1.0, __dmul_rn(4.0 / 3.0, __ddiv_rn((double)(diag - identical), __dsub_rn(length, gapc))));
  if (d <= kDoubleEpsilon) return false;
  *out = __dmul_rn(-0.75, cr_log(d));
  return true;
}

// Int16 distance of KimCnt counters: SWG-MPI ComputeDistance (Program.cs:271-276) or, with
// ms, the SWG-MS rules (Program.cs:555-668: Kimura2 capped at 10, undefined JukesCantor = 10).
// A JukesCantor that SWG-MPI would throw on sets *throws and gives 0.
__device__ __forceinline__ int16_t kim_distance(const KimCnt::T& c, int dist_fn, bool ms, int* throws) {
  const int len = (int)(c.w0 >> 16), a = (int)(c.w0 & 0xFFFFu);
  const int diag = (int)(c.w1 >> 16), b = (int)(c.w1 & 0xFFFFu);
  double v;
  if (dist_fn == 1) {
    v = kimura2_value(len, diag, a, b);
    if (ms && v > 10.0) v = 10.0;
  } else if (!jukes_cantor_value(len, diag, a, &v)) {
    if (!ms) {
      if (throws) atomicExch(throws, 1);
      return 0;
    }
    v = 10.0;
  }
  return cs_conv_i2_d(__dmul_rn(v, 32767.0));
}

// MinMaxNormScore of an alignment scoring s between sequences whose self scores (the sum of the
// matrix's diagonal over their residues) are self1 and self2: (1 - (s - minS) / (maxS - minS)) *
// 32767 in binary64, maxS = max(self1, self2), minS = 0 for SWG-MS (Salsa.SmithWatermanMS/
// Program.cs:544-553) and 2 open + (m + n) extend for NW (Salsa.NeedlemanWunschTPL/Program.cs:
// 573-581).  SWG-MPI's ComputeDistance has no case for it (Program.cs:259-285): its result stays 0.
// mode: 0 SWG-MPI, 1 SWG-MS, 2 NW.
__device__ __forceinline__ int16_t minmax_distance(long long s, int self1, int self2, int m, int n, int o, int e,
                                                   int mode) {
  if (mode == 0) return 0;
  const long long maxS = self1 > self2 ? self1 : self2;
  const long long minS = mode == 2 ? 2LL * o + (long long)(m + n) * e : 0LL;
  const double x = __ddiv_rn((double)(s - minS), (double)(maxS - minS));
  return cs_conv_i2_d(__dmul_rn(__dsub_rn(1.0, x), 32767.0));
}

}  // namespace swg
