// Fused critical-point extraction over a regular spacetime mesh.
//
// Replaces the per-simplex loop of the reference's feed() phase 1 and the
// face re-extraction of phase 2 (engine.hpp:118-158, 161-180, 1342-1367) and
// the incumbent extraction_kernel (cuda_engine.hpp:366-493): every m-simplex
// of the Freudenthal/Kuhn triangulation of the local box is visited exactly
// once, as (corner vertex, chain type), with the corner ranging over every
// vertex so that the upper-boundary simplices phase 2 discovers are included.
//
// One thread block owns a spatial tile of corners and marches through time,
// keeping one 64-bit cull word per vertex of the previous and current time
// slice in shared memory.  A hypercube is rejected as a whole when the AND of
// its vertices' words proves that every simplex in it fails the barycentric
// solve (see vertex_word); only the rare surviving hypercubes are enumerated
// simplex by simplex, with the exact integer SoS test and the bit-exact solve.
#include "cp_device.cuh"
#include "cp_internal.h"

namespace ftk2b {

__constant__ ChainTable c_chains[2];  // [0]: d=3, m=2 (12 chains); [1]: d=4, m=3 (60)

// ---------------------------------------------------------------------------
// Per-vertex cull word.
//
//   bits 0..2   component j strongly positive:  v_j >  kappa' * b,  b = max_k |v_k|
//   bits 3..5   component j strongly negative:  v_j < -kappa' * b
//   bit  6      tiny: b < 4e-13
//   bits 8..63  magnitude-band mask {n-1, n, n+1}, n = (exponent(b) - E_LO) / B
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
// Vertices outside the mesh get ~0 (neutral under AND).
template <typename T> struct CullParams;
template <> struct CullParams<double> {
  static constexpr double kappa_prime = 1.0 / 4096.0;  // 2^-12
  static constexpr int band = 4;                       // exponents per band
};
template <> struct CullParams<float> {
  static constexpr float kappa_prime = 1.0f / 64.0f;   // 2^-6
  static constexpr int band = 2;
};
constexpr int kElo = -42;      // 2^-42 < 4e-13: smaller magnitudes are "tiny"
constexpr int kBands = 56;
constexpr unsigned long long kAbsent = ~0ull;

__device__ __forceinline__ int exponent_of(double b) {
  return (int)((__double_as_longlong(b) >> 52) & 0x7FF) - 1023;
}
__device__ __forceinline__ int exponent_of(float b) {
  return (int)((__float_as_int(b) >> 23) & 0xFF) - 127;
}

template <typename T, int M>
__device__ __forceinline__ unsigned long long vertex_word(const T v[M]) {
  bool nan = false;
  T b = T(0);
#pragma unroll
  for (int j = 0; j < M; ++j) {
    nan |= (v[j] != v[j]);
    b = fmax(b, fabs(v[j]));
  }
  if (nan) return 0ull;  // never culled
  const T thr = b * CullParams<T>::kappa_prime;  // exact power-of-two scaling
  unsigned long long w = 0;
#pragma unroll
  for (int j = 0; j < M; ++j) {
    w |= (unsigned long long)(v[j] > thr) << j;
    w |= (unsigned long long)(v[j] < -thr) << (3 + j);
  }
  w |= (unsigned long long)(b < T(4e-13)) << 6;
  const int e = exponent_of(b);
  const int rel = e - kElo;
  if (rel >= 0 && rel < kBands * CullParams<T>::band && b > T(0)) {
    const int n = rel / CullParams<T>::band;
    unsigned long long band = (7ull << n) >> 1;  // bits n-1, n, n+1
    band &= (1ull << kBands) - 1;
    w |= band << 8;
  }
  return w;
}

__device__ __forceinline__ bool word_culled(unsigned long long w) {
  return (((w & 0x3Full) != 0) && ((w >> 8) != 0)) || ((w & 0x40ull) != 0);
}

// ---------------------------------------------------------------------------
// field access

template <typename T>
__device__ __forceinline__ T field_at(const FieldAccess& fa, int j, const long long g[4], int d,
                                      unsigned long long vid) {
  const T* base = static_cast<const T*>(fa.comp[j]);
  if (fa.per_vertex) return base[vid];
  long long o = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < d) o += (g[k] - fa.shift[k]) * fa.estride[k];
  return base[o];
}

template <typename T>
__device__ __forceinline__ T scalar_at(const FieldAccess& fa, const long long g[4], int d,
                                       unsigned long long vid) {
  const T* base = static_cast<const T*>(fa.scalar);
  if (fa.scalar_per_vertex) return base[vid];
  long long o = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < d) o += g[k] * fa.sstride[k];
  return base[o];
}

// ---------------------------------------------------------------------------

template <int D> struct Tile;
template <> struct Tile<4> {
  static constexpr int TX = 32, TY = 4, TZ = 4;
};
template <> struct Tile<3> {
  static constexpr int TX = 32, TY = 16, TZ = 1;
};

constexpr int kThreads = 256;

template <typename T, int D>
__global__ void __launch_bounds__(kThreads, 4)
    extract_regular_kernel(RegularMesh mesh, FieldAccess fa, ExtractConfig cfg, FeatureSink sink) {
  constexpr int M = D - 1;
  constexpr int TX = Tile<D>::TX, TY = Tile<D>::TY, TZ = Tile<D>::TZ;
  constexpr int VX = TX + 1, VY = TY + 1, VZ = (D == 4) ? TZ + 1 : 1;
  constexpr int VS = VX * VY * VZ;
  constexpr int NC = TX * TY * TZ;
  constexpr int TBIT = 1 << (D - 1);  // mask bit of the time axis
  constexpr int NV = 1 << D;          // vertices per hypercube

  __shared__ unsigned long long W[2][VS];
  __shared__ unsigned short surv[NC];
  __shared__ int nsurv;

  const ChainTable& CT = c_chains[D - 3];
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;

  // tile origin (local coordinates)
  int tix = blockIdx.x;
  const int x0 = (tix % cfg.tiles[0]) * TX;
  tix /= cfg.tiles[0];
  const int y0 = (tix % cfg.tiles[1]) * TY;
  tix /= cfg.tiles[1];
  const int z0 = (D == 4) ? tix * TZ : 0;
  const long long lt = mesh.ld[D - 1];
  const long long t0 = (long long)blockIdx.y * cfg.tchunk;
  const long long t1 = min(t0 + (long long)cfg.tchunk, lt);

  auto load_slice = [&](unsigned long long* dst, long long ts) {
    for (int i = tid; i < VS; i += kThreads) {
      const int vx = i % VX;
      const int r = i / VX;
      const int vy = r % VY;
      const int vz = r / VY;
      long long l[4] = {x0 + vx, y0 + vy, (D == 4) ? z0 + vz : ts, ts};
      bool in = l[0] < mesh.ld[0] && l[1] < mesh.ld[1] && (D == 3 || l[2] < mesh.ld[2]);
      unsigned long long w = kAbsent;
      if (in) {
        long long g[4];
        unsigned long long vid = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
          g[k] = l[k] + mesh.off[k];
          vid += (unsigned long long)g[k] * mesh.gstride[k];
        }
        T v[M];
#pragma unroll
        for (int j = 0; j < M; ++j) v[j] = field_at<T>(fa, j, g, D, vid);
        w = vertex_word<T, M>(v);
      }
      dst[i] = w;
    }
  };

  int cur = 0;
  load_slice(W[0], t0);
  for (long long ct = t0; ct < t1; ++ct) {
    const int nxt = cur ^ 1;
    if (ct + 1 < lt) {
      load_slice(W[nxt], ct + 1);
    } else {
      for (int i = tid; i < VS; i += kThreads) W[nxt][i] = kAbsent;
    }
    if (tid == 0) nsurv = 0;
    __syncthreads();

    // ---- hypercube cull
    for (int c = tid; c < NC; c += kThreads) {
      const int cx = c % TX;
      const int cy = (c / TX) % TY;
      const int cz = c / (TX * TY);
      if (x0 + cx >= mesh.ld[0] || y0 + cy >= mesh.ld[1] || (D == 4 && z0 + cz >= mesh.ld[2])) continue;
      unsigned long long acc = kAbsent;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const int dx = v & 1, dy = (v >> 1) & 1, dz = (D == 4) ? (v >> 2) & 1 : 0;
        const int slot = ((cz + dz) * VY + (cy + dy)) * VX + (cx + dx);
        acc &= ((v & TBIT) ? W[nxt] : W[cur])[slot];
      }
      if (!word_culled(acc)) surv[atomicAdd(&nsurv, 1)] = (unsigned short)c;
    }
    __syncthreads();

    // ---- surviving hypercubes: enumerate chains, exact tests
    const int ns = nsurv;
    for (int s = warp; s < ns; s += kThreads / 32) {
      const int c = surv[s];
      const int cx = c % TX;
      const int cy = (c / TX) % TY;
      const int cz = c / (TX * TY);
      const long long l[4] = {x0 + cx, y0 + cy, (D == 4) ? z0 + cz : ct, ct};
      int valid = 0;  // axes along which the corner can step by +1
#pragma unroll
      for (int k = 0; k < D; ++k)
        if (l[k] + 1 < mesh.ld[k]) valid |= 1 << k;
      long long g0[4];
      unsigned long long vid0 = 0;
#pragma unroll
      for (int k = 0; k < D; ++k) {
        g0[k] = l[k] + mesh.off[k];
        vid0 += (unsigned long long)g0[k] * mesh.gstride[k];
      }
      for (int base = 0; base < CT.n; base += 32) {
        const int ch = base + lane;
        bool acc = false;
        double lam_out[4] = {0, 0, 0, 0};
        float bary_out[4] = {0.f, 0.f, 0.f, 0.f};
        float sc_out = 0.f;
        if (ch < CT.n) {
          int mk[M + 1];
          mk[0] = 0;
#pragma unroll
          for (int i = 0; i < M; ++i) mk[i + 1] = CT.mask[ch][i];
          if ((mk[M] & ~valid) == 0) {
            unsigned long long wacc = kAbsent;
#pragma unroll
            for (int i = 0; i <= M; ++i) {
              const int dx = mk[i] & 1, dy = (mk[i] >> 1) & 1, dz = (D == 4) ? (mk[i] >> 2) & 1 : 0;
              const int slot = ((cz + dz) * VY + (cy + dy)) * VX + (cx + dx);
              wacc &= ((mk[i] & TBIT) ? W[nxt] : W[cur])[slot];
            }
            if (!word_culled(wacc)) {
              T vals[M + 1][M];
              long long gv[M + 1][4];
              unsigned long long vid[M + 1];
#pragma unroll
              for (int i = 0; i <= M; ++i) {
                vid[i] = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                  gv[i][k] = (k < D) ? g0[k] + ((mk[i] >> k) & 1) : 0;
                  if (k < D) vid[i] += (unsigned long long)gv[i][k] * mesh.gstride[k];
                }
#pragma unroll
                for (int j = 0; j < M; ++j) vals[i][j] = field_at<T>(fa, j, gv[i], D, vid[i]);
              }
              bool inside;
              if constexpr (M == 2) inside = sos_inside2<T>(vals, cfg.Q);
              else inside = sos_inside3<T>(vals, cfg.Q);
              if (inside) {
                T lam[M + 1];
                if (solve_exact<M, T>(vals, lam)) {
                  acc = true;
#pragma unroll
                  for (int i = 0; i <= M; ++i) {
                    lam_out[i] = (double)lam[i];
                    bary_out[i] = (float)lam[i];
                  }
                  if (fa.has_scalar) {
                    using F = fp<T>;
                    T s = T(0);
#pragma unroll
                    for (int i = 0; i <= M; ++i) s = F::add(s, F::mul(lam[i], scalar_at<T>(fa, gv[i], D, vid[i])));
                    sc_out = (float)s;
                  }
                  if (cfg.refined) {
                    double r[M + 1];
                    if (solve_refined<M, T>(vals, r))
#pragma unroll
                      for (int i = 0; i <= M; ++i) lam_out[i] = r[i];
                  }
                }
              }
            }
          }
        }
        const unsigned ball = __ballot_sync(0xFFFFFFFFu, acc);
        if (ball) {
          unsigned int basei = 0;
          const int leader = __ffs(ball) - 1;
          if (lane == leader) basei = atomicAdd(sink.count, (unsigned)__popc(ball));
          basei = __shfl_sync(0xFFFFFFFFu, basei, leader);
          if (acc) {
            const unsigned idx = basei + __popc(ball & ((1u << lane) - 1));
            if (idx < sink.cap) {
              sink.key[idx] = vid0 * (unsigned long long)CT.n + (unsigned long long)ch;
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                sink.lam[4 * (size_t)idx + i] = lam_out[i];
                sink.bary4[4 * (size_t)idx + i] = bary_out[i];
              }
              sink.scalar[idx] = sc_out;
            }
          }
        }
      }
    }
    __syncthreads();
    cur = nxt;
  }
}

// ---------------------------------------------------------------------------

static void build_chains(ChainTable& t, int d, int m) {
  // strictly increasing non-empty masks m1 < ... < mm (each a superset of the
  // previous), enumerated in lexicographic order of the mask sequence; since
  // vertex ids grow with the mask value along every axis order, this is also
  // the Simplex order of the simplices at one corner (mesh.hpp:36-42)
  t.n = 0;
  const int full = (1 << d) - 1;
  int cur[5] = {0, 0, 0, 0, 0};
  int next[5] = {0, 0, 0, 0, 0};
  int depth = 1;
  while (depth > 0) {
    int prev = cur[depth - 1];
    int nx = next[depth] + 1;
    while (nx <= full && !(((nx & prev) == prev) && nx != prev)) ++nx;
    if (nx > full) {
      next[depth] = 0;
      --depth;
      continue;
    }
    next[depth] = nx;
    cur[depth] = nx;
    if (depth == m) {
      for (int k = 0; k < m; ++k) t.mask[t.n][k] = (unsigned char)cur[k + 1];
      t.n++;
    } else {
      ++depth;
      next[depth] = 0;
    }
  }
}

void upload_chain_tables() {
  ChainTable h[2];
  build_chains(h[0], 3, 2);
  build_chains(h[1], 4, 3);
  cudaMemcpyToSymbol(c_chains, h, sizeof(h));
}

cudaError_t launch_extract_regular(int f64, const RegularMesh& mesh, const FieldAccess& fa,
                                   const ExtractConfig& cfg, const FeatureSink& sink,
                                   cudaStream_t st) {
  const long long lt = mesh.ld[mesh.d - 1];
  const unsigned nchunks = (unsigned)((lt + cfg.tchunk - 1) / cfg.tchunk);
  const unsigned ntiles = (unsigned)cfg.tiles[0] * cfg.tiles[1] * cfg.tiles[2];
  dim3 grid(ntiles, nchunks);
  if (mesh.d == 4) {
    if (f64) extract_regular_kernel<double, 4><<<grid, kThreads, 0, st>>>(mesh, fa, cfg, sink);
    else extract_regular_kernel<float, 4><<<grid, kThreads, 0, st>>>(mesh, fa, cfg, sink);
  } else {
    if (f64) extract_regular_kernel<double, 3><<<grid, kThreads, 0, st>>>(mesh, fa, cfg, sink);
    else extract_regular_kernel<float, 3><<<grid, kThreads, 0, st>>>(mesh, fa, cfg, sink);
  }
  return cudaGetLastError();
}

}  // namespace ftk2b
