// Device-side arithmetic of the critical-point predicate: quantisation, the
// integer Simulation-of-Simplicity inside tests and the partial-pivot
// barycentric solve, each rounding exactly like the reference's CPU build.
//
// Reference semantics (file:line in the reference tree):
//   quantisation        sos.hpp:15,25,75   (int128)((double)v*Q + (v > 0 ? .5 : -.5))
//   2D inside test      sos.hpp:22-35, 222-232
//   3D inside test      sos.hpp:72-200, 234-254
//   barycentric solve   zero_crossing.hpp:20-90 (precision T, no FMA)
//   accept              predicate.hpp:66-99 (inside AND solve succeeds)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ftk2b {

typedef __int128 i128;

// ---------------------------------------------------------------------------
// rounding-explicit scalar ops: the reference is compiled for x86-64 without
// FMA, so every multiply and add rounds separately

template <typename T> struct fp;
template <> struct fp<double> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double abs(double a) { return fabs(a); }
};
template <> struct fp<float> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float abs(float a) { return fabsf(a); }
};

// ---------------------------------------------------------------------------
// quantisation to the fixed-point lattice

// Exact truncating conversion of an integral double of magnitude >= 2^63.
__device__ __forceinline__ i128 big_double_to_i128(double p) {
  unsigned long long bits = (unsigned long long)__double_as_longlong(p);
  int e = (int)((bits >> 52) & 0x7FF) - 1075;  // value = mant * 2^e
  unsigned long long mant = (bits & 0xFFFFFFFFFFFFFull) | (1ull << 52);
  if (((bits >> 52) & 0x7FF) == 0x7FF) return 0;  // inf / nan: undefined in the reference
  i128 r = (e >= 75) ? (i128)0 : ((i128)mant << e);  // beyond 2^127 is undefined there too
  return (bits >> 63) ? -r : r;
}

// q(v) = trunc((double)v * Q + (v > 0 ? 0.5 : -0.5)), the product and the sum
// each rounded to nearest.
__device__ __forceinline__ long long quant64(double v, double Q, bool& big) {
  double p = __dadd_rn(__dmul_rn(v, Q), v > 0.0 ? 0.5 : -0.5);
  big = !(fabs(p) < 4.0e18);
  return __double2ll_rz(p);
}

__device__ __forceinline__ i128 quant128(double v, double Q) {
  double p = __dadd_rn(__dmul_rn(v, Q), v > 0.0 ? 0.5 : -0.5);
  if (fabs(p) < 4.0e18) return (i128)__double2ll_rz(p);
  return big_double_to_i128(p);
}

__device__ __forceinline__ int sgn(i128 x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }
__device__ __forceinline__ int sgn(long long x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

// ---------------------------------------------------------------------------
// 2D inside test (M = 2).  idx[] are the sorted vertex ids, so the tie-break
// of det2(va, vb) is +1 for (0,1) and (1,2) and -1 for (2,0).

template <typename T>
__device__ __forceinline__ bool sos_inside2(const T v[3][2], double Q) {
  long long q[3][2];
  bool big = false;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      bool b;
      q[i][j] = quant64((double)v[i][j], Q, b);
      big |= b;
      big |= (q[i][j] >= (1ll << 31)) || (q[i][j] <= -(1ll << 31));
    }
  int s[3];
  const int tie[3] = {1, 1, -1};
  if (!big) {
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int a = e, b = (e + 1) % 3;
      long long d = q[a][0] * q[b][1] - q[a][1] * q[b][0];
      s[e] = d ? sgn(d) : tie[e];
    }
  } else {
    i128 w[3][2];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 2; ++j) w[i][j] = quant128((double)v[i][j], Q);
    for (int e = 0; e < 3; ++e) {
      const int a = e, b = (e + 1) % 3;
      i128 d = w[a][0] * w[b][1] - w[a][1] * w[b][0];
      s[e] = d ? sgn(d) : tie[e];
    }
  }
  return s[0] == s[1] && s[1] == s[2];
}

// ---------------------------------------------------------------------------
// 3D inside test (M = 3).  det3(r0, r1, r2) is the sign of the 4x4
// determinant [r0 1; r1 1; r2 1; origin 1] with 13 sub-determinant fallback
// levels and a final +1 (sos.hpp:72-200).  The origin row quantises to 0, so
// level 0 is det[r0; r1; r2] and every level collapses to a small polynomial
// of the three rows; exact integer arithmetic gives the reference's value for
// any expansion of the same polynomial (and wraps identically on overflow).

static __device__ __noinline__ int sos_det3_levels(const i128 a[3], const i128 b[3], const i128 c[3]) {
  i128 d;
  if ((d = b[0] * c[1] - b[1] * c[0])) return sgn(d);     // 1
  if ((d = -(b[0] * c[2] - b[2] * c[0]))) return sgn(d);  // 2
  if ((d = b[1] * c[2] - b[2] * c[1])) return sgn(d);     // 3
  if ((d = -(a[0] * c[1] - a[1] * c[0]))) return sgn(d);  // 4
  if ((d = c[0])) return sgn(d);                          // 5
  if ((d = -c[1])) return sgn(d);                         // 6
  if ((d = a[0] * c[2] - a[2] * c[0])) return sgn(d);     // 7
  if ((d = c[2])) return sgn(d);                          // 8
  if ((d = -(a[1] * c[2] - a[2] * c[1]))) return sgn(d);  // 9
  if ((d = a[0] * b[1] - a[1] * b[0])) return sgn(d);     // 10
  if ((d = -b[0])) return sgn(d);                         // 11
  if ((d = b[1])) return sgn(d);                          // 12
  if ((d = a[0])) return sgn(d);                          // 13
  return 1;                                               // 14
}

__device__ __forceinline__ i128 det3_i128(const i128 a[3], const i128 b[3], const i128 c[3]) {
  return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
         a[2] * (b[0] * c[1] - b[1] * c[0]);
}

__device__ __forceinline__ long long det3_i64(const long long a[3], const long long b[3],
                                              const long long c[3]) {
  return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
         a[2] * (b[0] * c[1] - b[1] * c[0]);
}

// Argument order of the four oriented faces (sos.hpp:247-250).
__device__ __forceinline__ void face_rows(int f, int& r0, int& r1, int& r2) {
  // d0 = det3(v1,v3,v2)  d1 = det3(v0,v2,v3)  d2 = det3(v0,v3,v1)  d3 = det3(v0,v1,v2)
  const int tab[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};
  r0 = tab[f][0];
  r1 = tab[f][1];
  r2 = tab[f][2];
}

template <typename T>
__device__ bool sos_inside3(const T v[4][3], double Q) {
  long long q[4][3];
  bool big = false;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      bool b;
      q[i][j] = quant64((double)v[i][j], Q, b);
      big |= b;
      big |= (q[i][j] >= (1ll << 20)) || (q[i][j] <= -(1ll << 20));
    }
  int s[4];
  if (!big) {
    // |q| < 2^20: every level-0 term fits in int64 without overflow
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      int r0, r1, r2;
      face_rows(f, r0, r1, r2);
      long long d = det3_i64(q[r0], q[r1], q[r2]);
      if (d) {
        s[f] = sgn(d);
      } else {
        i128 a[3], b[3], c[3];
        for (int k = 0; k < 3; ++k) {
          a[k] = q[r0][k];
          b[k] = q[r1][k];
          c[k] = q[r2][k];
        }
        s[f] = sos_det3_levels(a, b, c);
      }
    }
  } else {
    i128 w[4][3];
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 3; ++j) w[i][j] = quant128((double)v[i][j], Q);
    for (int f = 0; f < 4; ++f) {
      int r0, r1, r2;
      face_rows(f, r0, r1, r2);
      i128 d = det3_i128(w[r0], w[r1], w[r2]);
      s[f] = d ? sgn(d) : sos_det3_levels(w[r0], w[r1], w[r2]);
    }
  }
  return s[0] == s[1] && s[1] == s[2] && s[2] == s[3];
}

// ---------------------------------------------------------------------------
// The same inside tests from values quantised once per hypercube vertex: a
// value enters as q when |q| < 2^31 (and the 64-bit conversion did not
// overflow), else as kQBig, and a simplex holding a kQBig value is tested by
// the functions above from its field values.  Below 2^31 every 2x2 minor is
// exact in 64 bits and a 3x3 determinant in 128, so the signs, and with them
// the decision, are those of the functions above.

constexpr int kQBig = -2147483647 - 1;

// p = (double)v * Q + (v > 0 ? 0.5 : -0.5), each operation rounded to
// nearest; the quantised value is trunc(p)
__device__ __forceinline__ double quant_p(double v, double Q) {
  return __dadd_rn(__dmul_rn(v, Q), v > 0.0 ? 0.5 : -0.5);
}

__device__ __forceinline__ int quant_small_p(double p) {
  if (!(fabs(p) < 2147483648.0)) return kQBig;  // |q| >= 2^31, or not finite
  return (int)__double2ll_rz(p);
}

__device__ __forceinline__ bool sos_inside2_q(const int q[3][2]) {
  const int tie[3] = {1, 1, -1};
  int s[3];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const int a = e, b = (e + 1) % 3;
    const long long d = (long long)q[a][0] * q[b][1] - (long long)q[a][1] * q[b][0];
    s[e] = d ? sgn(d) : tie[e];
  }
  return s[0] == s[1] && s[1] == s[2];
}

// 2x2 minor x0*y1 - x1*y0 of entries below 2^31: each product below 2^62
__device__ __forceinline__ long long minor2_q(int x0, int x1, int y0, int y1) {
  return (long long)x0 * y1 - (long long)x1 * y0;
}

// det3 of rows with entries below 2^20: minors below 2^41, the sum below 2^63
__device__ __forceinline__ long long det3_q20(const int a[3], const int b[3], const int c[3]) {
  return a[0] * minor2_q(b[1], b[2], c[1], c[2]) - a[1] * minor2_q(b[0], b[2], c[0], c[2]) +
         a[2] * minor2_q(b[0], b[1], c[0], c[1]);
}

// det3 of rows with entries below 2^31: the sum below 2^96, in 128 bits
__device__ __forceinline__ i128 det3_q31(const int a[3], const int b[3], const int c[3]) {
  return (i128)a[0] * minor2_q(b[1], b[2], c[1], c[2]) - (i128)a[1] * minor2_q(b[0], b[2], c[0], c[2]) +
         (i128)a[2] * minor2_q(b[0], b[1], c[0], c[1]);
}

// sos_det3_levels for entries below 2^31: every level is a 2x2 minor or a
// single entry, exact in 64 bits
static __device__ __noinline__ int sos_det3_levels_q(const int a[3], const int b[3], const int c[3]) {
  long long d;
  if ((d = minor2_q(b[0], b[1], c[0], c[1]))) return sgn(d);    // 1
  if ((d = -minor2_q(b[0], b[2], c[0], c[2]))) return sgn(d);   // 2
  if ((d = minor2_q(b[1], b[2], c[1], c[2]))) return sgn(d);    // 3
  if ((d = -minor2_q(a[0], a[1], c[0], c[1]))) return sgn(d);   // 4
  if ((d = c[0])) return sgn(d);                                // 5
  if ((d = -(long long)c[1])) return sgn(d);                    // 6
  if ((d = minor2_q(a[0], a[2], c[0], c[2]))) return sgn(d);    // 7
  if ((d = c[2])) return sgn(d);                                // 8
  if ((d = -minor2_q(a[1], a[2], c[1], c[2]))) return sgn(d);   // 9
  if ((d = minor2_q(a[0], a[1], b[0], b[1]))) return sgn(d);    // 10
  if ((d = -(long long)b[0])) return sgn(d);                    // 11
  if ((d = b[1])) return sgn(d);                                // 12
  if ((d = a[0])) return sgn(d);                                // 13
  return 1;                                                     // 14
}

__device__ __forceinline__ bool sos_inside3_q(const int q[4][3]) {
  // entries all below 2^20: the determinants in 64 bits
  unsigned wide = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) wide |= ((unsigned)q[k][j] + (1u << 20)) >> 21;
  int s[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    int r0, r1, r2;
    face_rows(f, r0, r1, r2);
    int sg;
    if (!wide) {
      const long long d = det3_q20(q[r0], q[r1], q[r2]);
      sg = sgn(d);
    } else {
      const i128 d = det3_q31(q[r0], q[r1], q[r2]);
      sg = sgn(d);
    }
    s[f] = sg ? sg : sos_det3_levels_q(q[r0], q[r1], q[r2]);
  }
  return s[0] == s[1] && s[1] == s[2] && s[2] == s[3];
}

// ---------------------------------------------------------------------------
// ZeroCrossingSolver<K,T>::solve, operation for operation

template <int K, typename T>
__device__ bool solve_exact(const T vals[K + 1][K], T lam[K + 1]) {
  using F = fp<T>;
  T A[K][K], x[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
#pragma unroll
    for (int i = 0; i < K; ++i) A[j][i] = F::sub(vals[i][j], vals[K][j]);
    x[j] = -vals[K][j];
  }
#pragma unroll
  for (int i = 0; i < K; ++i) {
    // first row with the strictly largest magnitude, as the reference's scan
    int p = i;
    T best = F::abs(A[i][i]);
#pragma unroll
    for (int j = i + 1; j < K; ++j) {
      const T a = F::abs(A[j][i]);
      if (a > best) {
        best = a;
        p = j;
      }
    }
#pragma unroll
    for (int r = i + 1; r < K; ++r) {
      if (p == r) {
#pragma unroll
        for (int l = 0; l < K; ++l) {
          T t = A[i][l];
          A[i][l] = A[r][l];
          A[r][l] = t;
        }
        T t = x[i];
        x[i] = x[r];
        x[r] = t;
      }
    }
    if (F::abs(A[i][i]) < T(1e-12)) return false;
#pragma unroll
    for (int j = i + 1; j < K; ++j) {
      T f = F::div(A[j][i], A[i][i]);
      x[j] = F::sub(x[j], F::mul(f, x[i]));
#pragma unroll
      for (int l = i + 1; l < K; ++l) A[j][l] = F::sub(A[j][l], F::mul(f, A[i][l]));
    }
  }
#pragma unroll
  for (int i = K - 1; i >= 0; --i) {
    T s = T(0);
#pragma unroll
    for (int j = i + 1; j < K; ++j) s = F::add(s, F::mul(A[i][j], x[j]));
    x[i] = F::div(F::sub(x[i], s), A[i][i]);
  }
  T sum = T(0);
#pragma unroll
  for (int i = 0; i < K; ++i) {
    lam[i] = x[i];
    sum = F::add(sum, lam[i]);
  }
  lam[K] = F::sub(T(1.0), sum);
  const T eps = T(1e-9);
  const T hi = T(1.0) + eps;  // folds in T: 1 + 1e-9 in double, exactly 1 in float
#pragma unroll
  for (int i = 0; i <= K; ++i)
    if (lam[i] < -eps || lam[i] > hi) return false;
  return true;
}

// FP32 solve followed by one FP64 residual-refinement step, for reporting
// positions close to the FP64 solution of the same simplex.  Returns false
// when the FP32 factorisation meets a zero pivot (callers then keep the
// exact-path lambda).
template <int K, typename T>
__device__ bool solve_refined(const T vals[K + 1][K], double out[K + 1]) {
  float A[K][K], LU[K][K], x[K];
  int perm[K];
  double Ad[K][K], bd[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
#pragma unroll
    for (int i = 0; i < K; ++i) {
      Ad[j][i] = (double)vals[i][j] - (double)vals[K][j];
      A[j][i] = (float)Ad[j][i];
    }
    bd[j] = -(double)vals[K][j];
    perm[j] = j;
  }
#pragma unroll
  for (int j = 0; j < K; ++j)
#pragma unroll
    for (int i = 0; i < K; ++i) LU[j][i] = A[j][i];
  // LU with partial pivoting in FP32
#pragma unroll
  for (int i = 0; i < K; ++i) {
    int p = i;
    float best = fabsf(LU[i][i]);
#pragma unroll
    for (int j = i + 1; j < K; ++j)
      if (fabsf(LU[j][i]) > best) {
        best = fabsf(LU[j][i]);
        p = j;
      }
#pragma unroll
    for (int r = i + 1; r < K; ++r)
      if (p == r) {
#pragma unroll
        for (int l = 0; l < K; ++l) {
          float t = LU[i][l];
          LU[i][l] = LU[r][l];
          LU[r][l] = t;
        }
        int t = perm[i];
        perm[i] = perm[r];
        perm[r] = t;
      }
    if (LU[i][i] == 0.0f) return false;
#pragma unroll
    for (int j = i + 1; j < K; ++j) {
      LU[j][i] = LU[j][i] / LU[i][i];
#pragma unroll
      for (int l = i + 1; l < K; ++l) LU[j][l] -= LU[j][i] * LU[i][l];
    }
  }
  auto lu_solve = [&](const double rhs[K], float sol[K]) {
    float y[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      float s = (float)rhs[perm[i]];
#pragma unroll
      for (int j = 0; j < i; ++j) s -= LU[i][j] * y[j];
      y[i] = s;
    }
#pragma unroll
    for (int i = K - 1; i >= 0; --i) {
      float s = y[i];
#pragma unroll
      for (int j = i + 1; j < K; ++j) s -= LU[i][j] * sol[j];
      sol[i] = s / LU[i][i];
    }
  };
  lu_solve(bd, x);
  // one refinement step: r = b - A x in FP64, correction in FP32, update in FP64
  double xd[K], r[K];
  float dx[K];
#pragma unroll
  for (int i = 0; i < K; ++i) xd[i] = (double)x[i];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double s = bd[j];
#pragma unroll
    for (int i = 0; i < K; ++i) s -= Ad[j][i] * xd[i];
    r[j] = s;
  }
  lu_solve(r, dx);
  double sum = 0.0;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    out[i] = xd[i] + (double)dx[i];
    sum += out[i];
  }
  out[K] = 1.0 - sum;
  return true;
}

}  // namespace ftk2b
