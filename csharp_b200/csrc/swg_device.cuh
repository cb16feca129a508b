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

namespace swg {

constexpr int kNegInf = -(1 << 28);  // -infinity of the float DP (only ever loses a max)
constexpr int kPadCode = 127;        // residue code of padding rows/columns
constexpr int kPadScore = -16384;    // score of any pair involving kPadCode
constexpr int kTable = 128;          // substitution tables are [128][128]

// Bits of the per-(c1,c2) flag table.
constexpr uint32_t kFlagCount = 1u;  // the context's counted column (identity or similarity)
constexpr uint32_t kFlagIdent = 2u;  // c1 == c2
constexpr uint32_t kFlagSimNA = 4u;  // NAligner similarity: c1 == c2 or S > 0

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

// FullCnt: every PairwiseAlignment field the path reads, for the single-pair aligner.
struct FullCnt {
  struct T { int id, sim, len, si, sj; };
  __device__ __forceinline__ static T stop(int i, int j) { return T{0, 0, 0, i, j}; }
  __device__ __forceinline__ static T origin() { return T{0, 0, 0, 0, 0}; }
  __device__ __forceinline__ static T row0(int j) { return T{0, 0, 0, 0, j}; }
  __device__ __forceinline__ static T col0(int i) { return T{0, 0, 0, i, 0}; }
  __device__ __forceinline__ static T diag(T c, uint32_t fl) {
    return T{c.id + (int)((fl >> 1) & 1u), c.sim + (int)((fl >> 2) & 1u), c.len + 1, c.si, c.sj};
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

}  // namespace swg
