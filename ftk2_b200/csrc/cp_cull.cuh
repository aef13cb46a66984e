// Per-vertex cull words shared by the regular-mesh and extruded-mesh
// extraction kernels: a 32-bit summary of a vertex's field value from which
// the AND over the vertices of a simplex (or of a whole hypercube) proves that
// the reference's barycentric solve (zero_crossing.hpp:20-90) rejects every
// simplex spanned by those vertices.
#pragma once

#include <cuda_runtime.h>

// loop unrolling in device code only (the word is also compiled for the
// host by its check)
#ifdef __CUDA_ARCH__
#define FTK2B_UNROLL _Pragma("unroll")
#else
#define FTK2B_UNROLL
#endif

namespace ftk2b {

// ---------------------------------------------------------------------------
// Per-vertex cull word (32 bits), computed with integer operations on the
// high 32 bits of each value (the whole value for float).
//
//   bits 0..2   component j strongly positive:  v_j >  kappa' * b,  b = max_k |v_k|
//   bits 3..5   component j strongly negative:  v_j < -kappa' * b
//   bit  6      tiny: b < 4e-13
//   bits 7..31  magnitude-band mask {n-1, n, n+1}, n = (exponent(b) - E_LO) / B
//
// The AND of the words of a set S of vertices is "culled" when
//   (a) a sign bit survives and the band mask is non-zero: then every vertex
//       has component j of one strict sign with |v_ij| > kappa' * b_i, and
//       the exponents of the b_i differ by at most 3B-1, so
//       min_i |v_ij| > kappa' * 2^-(3B) * max_i b_i = kappa * M.  An accepted
//       simplex needs lambda_i >= -1e-9, sum lambda = 1 and a residual
//       sum_i lambda_i v_ij bounded by the backward error of partial-pivot
//       elimination (|r| <= 72 gamma_9 M); with kappa = 2^-24 (double) and
//       2^-12 (float) that is impossible, so no simplex inside S is accepted.
//   (b) or the tiny bit survives: the first pivot of the solve is below 1e-12
//       (zero_crossing.hpp:72), so the solve rejects.
// Each predicate is evaluated on high words so that it can only err towards
// "not strong" / "not tiny": a strictly larger high word of a non-negative
// IEEE value implies a strictly larger value, and kappa' * b only shifts the
// exponent field.  Infinite or NaN components give a word without band and
// tiny bits (never culled).  Vertices outside the mesh get ~0 (neutral under
// AND).
template <typename T> struct CullParams;
template <> struct CullParams<double> {
  static constexpr int mant = 20;          // mantissa bits in the high word
  static constexpr unsigned expmask = 0x7FF00000u;
  static constexpr int bias = 1023;
  static constexpr int kappa_exp = 12;     // kappa' = 2^-12
  static constexpr int band = 4;           // exponents per band: kappa = 2^-24
  static constexpr unsigned tiny_hi = 0x3D5C25C2u;  // high word of 4e-13 (rounded down)
};
template <> struct CullParams<float> {
  static constexpr int mant = 23;
  static constexpr unsigned expmask = 0x7F800000u;
  static constexpr int bias = 127;
  static constexpr int kappa_exp = 3;      // kappa' = 2^-3
  static constexpr int band = 3;           // kappa = 2^-12
  static constexpr unsigned tiny_hi = 0x2AE12E13u;  // 4e-13f (3.99999993e-13)
};
constexpr int kElo = -42;      // 2^-42 < 4e-13: smaller magnitudes are "tiny"
constexpr int kBands = 25;
constexpr unsigned kAbsent = ~0u;

template <typename T> __device__ __forceinline__ unsigned hi_word(T v);
template <> __device__ __forceinline__ unsigned hi_word<double>(double v) {
  return (unsigned)__double2hiint(v);
}
template <> __device__ __forceinline__ unsigned hi_word<float>(float v) {
  return __float_as_uint(v);
}

// Band masks by magnitude exponent: band_table[rel + 1] for rel = biased
// exponent - bias - E_LO; 0 outside the banded window (and at index 0).
constexpr int kBandTable = 128;

template <typename T>
__host__ __device__ __forceinline__ void fill_band_table(unsigned* tbl, int tid, int nthreads) {
  using P = CullParams<T>;
  for (int i = tid; i < kBandTable; i += nthreads) {
    const int rel = i - 1;
    unsigned w = 0;
    if (rel >= 0 && rel < kBands * P::band) {
      const int n = rel / P::band;
      w = (((7u << n) >> 1) & ((1u << kBands) - 1u)) << 7;  // bits n-1, n, n+1
    }
    tbl[i] = w;
  }
}

template <typename T, int M>
__host__ __device__ __forceinline__ unsigned vertex_word_hi(const unsigned h[M], const unsigned* band_tbl) {
  using P = CullParams<T>;
  unsigned a[M], b = 0;
FTK2B_UNROLL
  for (int j = 0; j < M; ++j) {
    a[j] = h[j] & 0x7FFFFFFFu;
    b = b > a[j] ? b : a[j];
  }
  const unsigned kexp = (unsigned)P::kappa_exp << P::mant;
  const unsigned thr = (b > kexp ? b : kexp) - kexp;  // high word of kappa' * b (0 below kappa')
  // component j strong: |v_j| > thr, as the sign of thr - |v_j| (both below
  // 2^31, so the difference does not overflow); the value's sign then picks
  // bit j (positive) or bit 3 + j (negative)
  unsigned w = 0;
FTK2B_UNROLL
  for (int j = 0; j < M; ++j) {
    const unsigned strong = (unsigned)((int)(thr - a[j]) >> 31);
    const unsigned neg = (unsigned)((int)h[j] >> 31);
    w |= strong & ((neg & (8u << j)) | (~neg & (1u << j)));
  }
  w |= (b < P::tiny_hi ? 1u : 0u) << 6;
  const int rel1 = (int)(b >> P::mant) - P::bias - kElo + 1;
  // inf or nan somewhere: the exponent lies past the banded window, so the
  // word gets no band bit (and no tiny bit) and no set of vertices holding
  // it is ever culled
  const unsigned ri = (unsigned)rel1 < (unsigned)(kBandTable - 1) ? (unsigned)rel1 : (unsigned)(kBandTable - 1);
  w |= band_tbl[ri];
  return w;
}

__device__ __forceinline__ bool word_culled(unsigned w) {
  return (((w & 0x3Fu) != 0) && ((w >> 7) != 0)) || ((w & 0x40u) != 0);
}

}  // namespace ftk2b
