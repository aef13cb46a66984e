// Classification of a critical point from the spatial Jacobian J (m x m,
// J[j][a] = d v_j / d x_a) of the linear interpolant on a top cell that
// contains the feature simplex.  The reference stores type = 0 for every
// feature (predicate.hpp:80, 119); this classification is reported in a
// separate field.
//
// Eigen-signature of J:
//   m = 2: det < 0 saddle; det > 0 with real eigenvalues (disc = tr^2 - 4 det
//          >= 0) source (tr > 0) / sink (tr < 0); complex eigenvalues spiral
//          source / spiral sink / centre by the sign of tr; det = 0 degenerate
//   m = 3: characteristic polynomial l^3 + a2 l^2 + a1 l + a0 (a2 = -tr,
//          a1 = sum of principal 2x2 minors, a0 = -det).  The sign changes of
//          the Routh column (1, a2, h / a2, a0), h = a2 a1 - a0, count the
//          eigenvalues with positive real part: 3 source, 0 sink, otherwise
//          saddle; complex eigenvalues (cubic discriminant < 0) make a source
//          or sink a spiral one.  det = 0 is degenerate; h = 0 factors the
//          polynomial as (l + a2)(l^2 + a1): saddle for a1 < 0, centre for
//          a1 > 0; tr = 0 with h, det != 0 is a saddle.
// For a gradient field J is the Hessian: source = minimum, sink = maximum.
//
// Precision: the invariants are evaluated in FP32 on J scaled by a power of
// two (exact) together with a magnitude scale S (the sum of the absolute
// values of the terms).  FP32 rounding moves an invariant by far less than
// 2^-10 S, so a sign is trusted when |x| > 2^-10 S; otherwise all invariants
// are evaluated again in FP64 with every operation rounded separately, in the
// order written below, and the FP64 signs decide.
#pragma once

#include <cuda_runtime.h>

#include "../../include/ftk2b.h"

namespace ftk2b {

constexpr float kClassBand = 1.0f / 1024.0f;

template <typename R> struct cr;
template <> struct cr<double> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};
template <> struct cr<float> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};

template <typename R> __device__ __forceinline__ int sgn_of(R x) { return x > R(0) ? 1 : (x < R(0) ? -1 : 0); }

__device__ __forceinline__ unsigned decide2(int sdet, int str, int sdisc) {
  if (sdet == 0) return FTK2B_CLASS_DEGENERATE;
  if (sdet < 0) return FTK2B_CLASS_SADDLE;
  if (sdisc >= 0) return str > 0 ? FTK2B_CLASS_SOURCE : (str < 0 ? FTK2B_CLASS_SINK : FTK2B_CLASS_DEGENERATE);
  return str > 0 ? FTK2B_CLASS_SPIRAL_SOURCE : (str < 0 ? FTK2B_CLASS_SPIRAL_SINK : FTK2B_CLASS_CENTER);
}

__device__ __forceinline__ unsigned decide3(int sa2, int sa1, int sh, int sa0, int sdelta) {
  if (sa0 == 0) return FTK2B_CLASS_DEGENERATE;  // a zero eigenvalue
  // h = 0: the polynomial is (l + a2)(l^2 + a1): a real pair +-r (saddle) or
  // an imaginary pair +-iw (centre)
  if (sh == 0) return sa1 < 0 ? FTK2B_CLASS_SADDLE : (sa1 > 0 ? FTK2B_CLASS_CENTER : FTK2B_CLASS_DEGENERATE);
  // trace 0, det != 0, no imaginary pair: the real parts have mixed signs
  if (sa2 == 0) return FTK2B_CLASS_SADDLE;
  // Routh column signs: 1, a2, h / a2, a0
  const int c1 = sa2, c2 = sh * sa2, c3 = sa0;
  const int npos = (c1 < 0) + (c1 != c2) + (c2 != c3);
  const bool complex_pair = sdelta < 0;
  if (npos == 3) return complex_pair ? FTK2B_CLASS_SPIRAL_SOURCE : FTK2B_CLASS_SOURCE;
  if (npos == 0) return complex_pair ? FTK2B_CLASS_SPIRAL_SINK : FTK2B_CLASS_SINK;
  return FTK2B_CLASS_SADDLE;
}

// Invariants of a 2x2 Jacobian in precision R, each with its scale.
template <typename R>
__device__ __forceinline__ void invariants2(const R J[2][2], R& det, R& tr, R& disc, R& sdet, R& str,
                                            R& sdisc) {
  using O = cr<R>;
  const R ad = O::mul(J[0][0], J[1][1]), bc = O::mul(J[0][1], J[1][0]);
  det = O::sub(ad, bc);
  tr = O::add(J[0][0], J[1][1]);
  disc = O::sub(O::mul(tr, tr), O::mul(R(4), det));
  sdet = fabs(ad) + fabs(bc);
  str = fabs(J[0][0]) + fabs(J[1][1]);
  sdisc = str * str + R(4) * sdet;
}

template <typename R>
__device__ __forceinline__ void invariants3(const R J[3][3], R& a2, R& a1, R& h, R& a0, R& delta, R& s_a2,
                                            R& s_a1, R& s_h, R& s_a0, R& s_delta) {
  using O = cr<R>;
  const R p0 = O::mul(J[1][1], J[2][2]), q0 = O::mul(J[1][2], J[2][1]);
  const R p1 = O::mul(J[0][0], J[2][2]), q1 = O::mul(J[0][2], J[2][0]);
  const R p2 = O::mul(J[0][0], J[1][1]), q2 = O::mul(J[0][1], J[1][0]);
  const R m0 = O::sub(p0, q0), m1 = O::sub(p1, q1), m2 = O::sub(p2, q2);
  const R r1 = O::mul(J[1][0], J[2][2]), u1 = O::mul(J[1][2], J[2][0]);
  const R r2 = O::mul(J[1][0], J[2][1]), u2 = O::mul(J[1][1], J[2][0]);
  const R c1 = O::sub(r1, u1), c2 = O::sub(r2, u2);
  const R tr = O::add(O::add(J[0][0], J[1][1]), J[2][2]);
  a1 = O::add(O::add(m0, m1), m2);
  const R det = O::add(O::sub(O::mul(J[0][0], m0), O::mul(J[0][1], c1)), O::mul(J[0][2], c2));
  a2 = -tr;
  a0 = -det;
  h = O::sub(O::mul(a2, a1), a0);
  const R b = a2, c = a1, d = a0;
  const R t1 = O::mul(O::mul(O::mul(R(18), b), c), d);
  const R t2 = O::mul(O::mul(O::mul(O::mul(R(4), b), b), b), d);
  const R t3 = O::mul(O::mul(O::mul(b, b), c), c);
  const R t4 = O::mul(O::mul(O::mul(R(4), c), c), c);
  const R t5 = O::mul(O::mul(R(27), d), d);
  delta = O::sub(O::sub(O::add(O::sub(t1, t2), t3), t4), t5);
  // magnitude scales
  s_a2 = fabs(J[0][0]) + fabs(J[1][1]) + fabs(J[2][2]);
  s_a1 = fabs(p0) + fabs(q0) + fabs(p1) + fabs(q1) + fabs(p2) + fabs(q2);
  s_a0 = fabs(J[0][0]) * (fabs(p0) + fabs(q0)) + fabs(J[0][1]) * (fabs(r1) + fabs(u1)) +
         fabs(J[0][2]) * (fabs(r2) + fabs(u2));
  s_h = s_a2 * s_a1 + s_a0;
  s_delta = R(18) * s_a2 * s_a1 * s_a0 + R(4) * s_a2 * s_a2 * s_a2 * s_a0 + s_a2 * s_a2 * s_a1 * s_a1 +
            R(4) * s_a1 * s_a1 * s_a1 + R(27) * s_a0 * s_a0;
}

__device__ __forceinline__ bool in_band(float x, float s) { return !(fabsf(x) > kClassBand * s); }

// J in the field precision T.  Scaled by 2^-e (e = exponent of max |J|) so
// that FP32 neither overflows nor underflows on the invariants' products.
template <int M, typename T>
__device__ unsigned classify_jacobian(const T Jt[M][M]) {
  double mx = 0.0;
  bool finite = true;
#pragma unroll
  for (int j = 0; j < M; ++j)
#pragma unroll
    for (int a = 0; a < M; ++a) {
      const double v = (double)Jt[j][a];
      finite &= isfinite(v);
      mx = fmax(mx, fabs(v));
    }
  if (!finite || mx == 0.0) return FTK2B_CLASS_DEGENERATE;
  int e;
  frexp(mx, &e);
  double Jd[M][M];
  float Jf[M][M];
#pragma unroll
  for (int j = 0; j < M; ++j)
#pragma unroll
    for (int a = 0; a < M; ++a) {
      Jd[j][a] = ldexp((double)Jt[j][a], -e);
      Jf[j][a] = (float)Jd[j][a];
    }
  if constexpr (M == 2) {
    float det, tr, disc, sd, st, sdc;
    invariants2<float>(Jf, det, tr, disc, sd, st, sdc);
    if (!in_band(det, sd) && !in_band(tr, st) && !in_band(disc, sdc))
      return decide2(sgn_of(det), sgn_of(tr), sgn_of(disc));
    double dd, dt, dc, xd, xt, xc;
    invariants2<double>(Jd, dd, dt, dc, xd, xt, xc);
    return decide2(sgn_of(dd), sgn_of(dt), sgn_of(dc));
  } else {
    float a2, a1, h, a0, dl, s2, s1, sh, s0, sdl;
    invariants3<float>(Jf, a2, a1, h, a0, dl, s2, s1, sh, s0, sdl);
    if (!in_band(a2, s2) && !in_band(a1, s1) && !in_band(h, sh) && !in_band(a0, s0) && !in_band(dl, sdl))
      return decide3(sgn_of(a2), sgn_of(a1), sgn_of(h), sgn_of(a0), sgn_of(dl));
    double da2, da1, dh, da0, ddl, x2, x1, xh, x0, xdl;
    invariants3<double>(Jd, da2, da1, dh, da0, ddl, x2, x1, xh, x0, xdl);
    return decide3(sgn_of(da2), sgn_of(da1), sgn_of(dh), sgn_of(da0), sgn_of(ddl));
  }
}

}  // namespace ftk2b
