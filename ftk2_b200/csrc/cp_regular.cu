// Fused critical-point extraction over a regular spacetime mesh.
//
// Replaces the per-simplex loop of the reference's feed() phase 1 and the
// face re-extraction of phase 2 (engine.hpp:118-158, 161-180, 1342-1367) and
// the incumbent extraction_kernel (cuda_engine.hpp:366-493): every m-simplex
// of the Freudenthal/Kuhn triangulation of the local box is visited exactly
// once, as (corner vertex, chain type), with the corner ranging over every
// vertex so that the upper-boundary simplices phase 2 discovers are included.
//
// One thread block owns a spatial tile of corners (32 along x, one warp lane
// each) and marches through time.  Each time slice of the tile (plus a
// one-vertex halo) is brought into shared memory by one TMA tensor-tile copy
// per array, double-buffered so the next slice streams in while the current
// step is culled.  Every vertex gets a 64-bit cull word; a hypercube is
// rejected when the AND of its vertices' words proves that no simplex in it
// can pass the barycentric solve (see vertex_word).  Only the rare surviving
// hypercubes are enumerated simplex by simplex with the exact integer SoS test
// and the bit-exact solve, and accepted simplices are compacted by warp ballot.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>

#include "cp_cull.cuh"
#include "cp_device.cuh"
#include "cp_field.cuh"
#include "cp_internal.h"

namespace ftk2b {

__constant__ ChainTable c_chains[2];  // [0]: d=3, m=2 (12 chains); [1]: d=4, m=3 (60)
// chains whose vertices all stay inside the mesh, by the mask of axes along
// which a corner may step: [0][vmask] for d = 3, [1][vmask] for d = 4
__constant__ unsigned long long c_chains_by_vmask[2][16];
// chains whose last vertex steps along the time axis
__constant__ unsigned long long c_time_chains[2];

// ---------------------------------------------------------------------------
// TMA / mbarrier primitives (inline PTX)

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait for the phase of the given parity; false if it never completed.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  const unsigned a = smem_addr(bar);
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            int c3, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}

// ---------------------------------------------------------------------------

template <int D> struct Tile;
template <> struct Tile<4> {
  // warp w owns corner row cy = w % 8 and corner z levels 2 (w / 8) .. +1
  static constexpr int TX = 32, TY = 8, TZ = 4;
};
template <> struct Tile<3> {
  // warp w owns corner rows cy = 2w, 2w + 1
  static constexpr int TX = 32, TY = 32, TZ = 1;
};

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kRows = 2;  // corner rows a warp culls per step

// Compile-time geometry of one block's time slice in shared memory, as the
// TMA box lays it out: multicomponent [VZ][VY][VXBOX * M], separate arrays
// [M][VZ][VY][VXBOX] (each component padded to 128 bytes).  VXBOX >= TX + 1
// is padded so every box row is a multiple of 16 bytes.
__host__ __device__ constexpr int vxbox_of(bool multi, int m, int es) {
  return ((33 * (multi ? m : 1) * es) % 16 == 0)   ? 33
         : ((34 * (multi ? m : 1) * es) % 16 == 0) ? 34
         : ((35 * (multi ? m : 1) * es) % 16 == 0) ? 35
                                                     : 36;
}
__host__ __device__ constexpr int round128(int b) { return (b + 127) & ~127; }

template <typename T, int D, bool MULTI>
struct Geo {
  static constexpr int M = D - 1;
  static constexpr int TX = Tile<D>::TX, TY = Tile<D>::TY, TZ = Tile<D>::TZ;
  static constexpr int VX = TX + 1, VY = TY + 1, VZ = (D == 4) ? TZ + 1 : 1;
  static constexpr int VS = VX * VY * VZ;                     // vertex slots of a slice
  static constexpr int VPT = (VS + kThreads - 1) / kThreads;  // slots per thread
  static constexpr int VSP = VPT * kThreads;                  // padded slots
  static constexpr int VXBOX = vxbox_of(MULTI, M, (int)sizeof(T));
  static constexpr int COMP_RAW = VXBOX * VY * VZ * (int)sizeof(T);  // bytes of one component box
  static constexpr int COMP = round128(COMP_RAW);
  static constexpr int BYTES = MULTI ? round128(COMP_RAW * M) : COMP * M;  // one slice buffer
  static constexpr int TX_BYTES = COMP_RAW * M;                          // bytes TMA delivers
  static constexpr int COMP_ELEMS = COMP / (int)sizeof(T);
  static constexpr int WORDS = 2 * BYTES;                                // offset of the word slots
  static constexpr int SMEM = WORDS + 3 * VSP * 4;
};

__device__ __forceinline__ unsigned long long pack_corner(long long x, long long y, long long z,
                                                          long long t) {
  return (unsigned long long)x | ((unsigned long long)y << 16) | ((unsigned long long)z << 32) |
         ((unsigned long long)t << 48);
}

// Stage 1: stream the field through shared memory, cull hypercubes, queue
// the survivors with the chains whose own vertices survive the cull.
template <typename T, int D, bool MULTI, bool TMA>
__global__ void __launch_bounds__(kThreads, 2)
    extract_regular_kernel(const __grid_constant__ CUtensorMap map0,
                           const __grid_constant__ CUtensorMap map1,
                           const __grid_constant__ CUtensorMap map2, RegularMesh mesh, FieldAccess fa,
                           ExtractConfig cfg, CandidateQueue cq, unsigned* err) {
  using G = Geo<T, D, MULTI>;
  constexpr int M = D - 1;
  constexpr int TX = G::TX, TY = G::TY, TZ = G::TZ;
  constexpr int VX = G::VX, VY = G::VY, VZ = G::VZ, VS = G::VS, VPT = G::VPT, VSP = G::VSP;
  constexpr int TBIT = 1 << (D - 1);  // mask bit of the time axis
  constexpr int HW = sizeof(T) / 4;   // the high 32-bit word of an element is its last
  static_assert(D == 3 ? kWarps * kRows == TY : kWarps == TY * (TZ / kRows),
                "every corner row of the tile belongs to exactly one warp");

  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned long long bar[2];
  __shared__ unsigned band_tbl[kBandTable];
  unsigned* const Wb = reinterpret_cast<unsigned*>(smem + G::WORDS);

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;

  // tile origin (local coordinates)
  int tix = blockIdx.x;
  const int x0 = (tix % cfg.tiles[0]) * TX;
  tix /= cfg.tiles[0];
  const int y0 = (tix % cfg.tiles[1]) * TY;
  tix /= cfg.tiles[1];
  const int z0 = (D == 4) ? tix * TZ : 0;
  const int ldx = (int)mesh.ld[0], ldy = (int)mesh.ld[1], ldz = (D == 4) ? (int)mesh.ld[2] : 1;
  // time in int: local dims are below 2^16
  const int lt = (int)mesh.ld[D - 1];
  const int t0 = (int)blockIdx.y * cfg.tchunk;
  const int t1 = min(t0 + cfg.tchunk, lt);
  const int s_end = min(t1, lt - 1);  // last vertex slice this block reads
  // array coordinates of local (0,0,0,0): global for multicomponent arrays,
  // local for separate arrays
  int aoff[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) aoff[k] = (k < D) ? (int)(mesh.off[k] - fa.shift[k]) : 0;
  // array time coordinate of vertex slice s: (s + aoff) xor tflip (a stream's
  // two-slot ring stores timestep t in slot t & 1; tflip = 0 otherwise)
  auto tcoord = [&](int s) { return (s + aoff[D - 1]) ^ fa.tflip; };

  // per-thread vertex slots of a slice, fixed for the whole time march:
  // element offset of component 0 in a slice buffer and a validity bit
  int voff[VPT];
  unsigned vvalid = 0;
#pragma unroll
  for (int u = 0; u < VPT; ++u) {
    const int i = tid + u * kThreads;
    const int vx = i % VX, vy = (i / VX) % VY, vz = i / (VX * VY);
    const bool in = i < VS && x0 + vx < ldx && y0 + vy < ldy && (D == 3 || z0 + vz < ldz);
    voff[u] = in ? (MULTI ? ((vz * VY + vy) * G::VXBOX + vx) * M : (vz * VY + vy) * G::VXBOX + vx) : 0;
    vvalid |= (in ? 1u : 0u) << u;
  }
  fill_band_table<T>(band_tbl, tid, kThreads);  // visible after the first barrier below

  // ---- slice staging
  auto issue = [&](int s, int buf) {
    unsigned char* dst0 = smem + buf * G::BYTES;
    if constexpr (TMA) {
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bar[buf], G::TX_BYTES);
        const int cx = (x0 + aoff[0]) * (MULTI ? M : 1);
        const int cy = y0 + aoff[1];
        if constexpr (MULTI) {
          if constexpr (D == 4) tma_load_4d(dst0, &map0, cx, cy, z0 + aoff[2], tcoord(s), &bar[buf]);
          else tma_load_3d(dst0, &map0, cx, cy, tcoord(s), &bar[buf]);
        } else {
          const CUtensorMap* maps[3] = {&map0, &map1, &map2};
#pragma unroll
          for (int j = 0; j < M; ++j) {
            if constexpr (D == 4)
              tma_load_4d(dst0 + j * G::COMP, maps[j], cx, cy, z0 + aoff[2], tcoord(s), &bar[buf]);
            else
              tma_load_3d(dst0 + j * G::COMP, maps[j], cx, cy, tcoord(s), &bar[buf]);
          }
        }
      }
    } else {
      // plain cooperative loads into the same layout (zero outside the array)
      T* dst = reinterpret_cast<T*>(dst0);
      constexpr int NPER = G::VXBOX * VY * VZ;
      for (int e = tid; e < NPER * M; e += kThreads) {
        const int j = MULTI ? e % M : e / NPER;
        const int r = MULTI ? e / M : e % NPER;
        const int vx = r % G::VXBOX;
        const int vy = (r / G::VXBOX) % VY;
        const int vz = r / (G::VXBOX * VY);
        const long long l[4] = {x0 + vx, y0 + vy, (D == 4) ? z0 + vz : (long long)s, (long long)s};
        bool in = true;
        long long o = 0;
        if (fa.per_vertex) {
          // 1-D per-vertex arrays: index by vertex id, only inside the mesh
#pragma unroll
          for (int k = 0; k < D; ++k) {
            in &= l[k] < mesh.ld[k];
            o += (l[k] + mesh.off[k]) * (long long)mesh.gstride[k];
          }
        } else {
#pragma unroll
          for (int k = 0; k < D; ++k) {
            const long long a = (k == D - 1) ? (long long)tcoord(s) : l[k] + aoff[k];
            in &= a >= 0 && a < fa.adims[k];
            o += a * fa.estride[k];
          }
        }
        T v = T(0);
        if (in) v = static_cast<const T*>(fa.comp[j])[o];
        if (MULTI) dst[((vz * VY + vy) * G::VXBOX + vx) * M + j] = v;
        else dst[j * G::COMP_ELEMS + (vz * VY + vy) * G::VXBOX + vx] = v;
      }
    }
  };
  // every thread waits for the slice's TMA phase itself (try_wait suspends
  // in hardware); returns false when the bounded wait gave up
  auto wait = [&](int s, int buf) -> bool {
    if constexpr (TMA) return mbar_wait(&bar[buf], (unsigned)(((s - t0) >> 1) & 1));
    else return true;
  };
  auto words = [&](int buf, int slot) {
    const unsigned* r = reinterpret_cast<const unsigned*>(smem + buf * G::BYTES) + (HW - 1);
    unsigned* dst = Wb + slot * VSP;
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      unsigned h[M];
#pragma unroll
      for (int j = 0; j < M; ++j) h[j] = r[HW * (MULTI ? voff[u] + j : voff[u] + j * G::COMP_ELEMS)];
      const unsigned w = vertex_word_hi<T, M>(h, band_tbl);
      dst[tid + u * kThreads] = ((vvalid >> u) & 1u) ? w : kAbsent;
    }
  };

  if constexpr (TMA) {
    if (tid == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    issue(t0, 0);
    if (t0 + 1 <= s_end) issue(t0 + 1, 1);
  } else {
    __syncthreads();
    issue(t0, 0);
    __syncthreads();
  }
  int slot_a = 0;  // word slot of slice ct
  {
    const bool ok = wait(t0, 0);
    if (ok) words(0, slot_a);
    if (__syncthreads_or(!ok)) {
      // give the other copy in flight a bounded chance to land before leaving
      if (TMA && t0 + 1 <= s_end) mbar_wait(&bar[1], 0);
      if (tid == 0) atomicOr(err, 2u);
      return;
    }
  }
  if (TMA && t0 + 2 <= s_end) issue(t0 + 2, 0);

  // corner validity per (lane, row) does not change along time
  const int cyw = (D == 4) ? warp % TY : warp * kRows;
  const int czw = (D == 4) ? (warp / TY) * kRows : 0;
  unsigned row_valid = 0;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    const int cy = (D == 4) ? cyw : cyw + q;
    const int cz = (D == 4) ? czw + q : 0;
    if (x0 + lane < ldx && y0 + cy < ldy && (D == 3 || z0 + cz < ldz)) row_valid |= 1u << q;
  }

  for (int ct = t0; ct < t1; ++ct) {
    const int s = ct + 1;
    const int slot_b = slot_a == 2 ? 0 : slot_a + 1;  // word slot of slice s
    unsigned* B = Wb + slot_b * VSP;
    bool ok = true;
    if (s <= s_end) {
      const int buf = (s - t0) & 1;
      if (!TMA) {
        issue(s, buf);
        __syncthreads();
      }
      ok = wait(s, buf);
      if (ok) words(buf, slot_b);
    } else {
      for (int i = tid; i < VS; i += kThreads) B[i] = kAbsent;
    }
    // the one block barrier of the step: words of slice s are visible, its
    // raw buffer is free, and every warp has finished culling step ct - 1
    if (__syncthreads_or(!ok)) {
      if (TMA && s + 1 <= s_end) mbar_wait(&bar[((s - t0) & 1) ^ 1], (unsigned)(((s + 1 - t0) >> 1) & 1));
      if (tid == 0) atomicOr(err, 2u);
      return;
    }
    if (TMA && s + 2 <= s_end) issue(s + 2, (s - t0) & 1);

    // ---- hypercube cull: lanes along x, kRows corner rows per warp
    const unsigned* A = Wb + slot_a * VSP;
    unsigned R[kRows + 1];
#pragma unroll
    for (int q = 0; q <= kRows; ++q) {
      unsigned r, e;
      if constexpr (D == 4) {
        const int i0 = ((czw + q) * VY + cyw) * VX + lane, i1 = i0 + VX;
        r = A[i0] & A[i1] & B[i0] & B[i1];
        e = (lane == 31) ? (A[i0 + 1] & A[i1 + 1] & B[i0 + 1] & B[i1 + 1]) : kAbsent;
      } else {
        const int i0 = (cyw + q) * VX + lane;
        r = A[i0] & B[i0];
        e = (lane == 31) ? (A[i0 + 1] & B[i0 + 1]) : kAbsent;
      }
      const unsigned nb = __shfl_down_sync(0xFFFFFFFFu, r, 1);
      R[q] = r & (lane == 31 ? e : nb);
    }
#pragma unroll
    for (int q = 0; q < kRows; ++q) {
      const int cy = (D == 4) ? cyw : cyw + q;
      const int cz = (D == 4) ? czw + q : 0;
      const bool keep = ((row_valid >> q) & 1u) && !word_culled(R[q] & R[q + 1]);
      const unsigned ball = __ballot_sync(0xFFFFFFFFu, keep);
      if (ball) {
        // surviving hypercubes are queued with every chain that fits in the
        // mesh; the exact-test kernel applies the per-simplex word test
        unsigned basei = 0;
        if (lane == 0) basei = atomicAdd(cq.count, (unsigned)__popc(ball));
        basei = __shfl_sync(0xFFFFFFFFu, basei, 0);
        if (keep) {
          const unsigned idx = basei + __popc(ball & ((1u << lane) - 1));
          if (idx < cq.cap) {
            const int l0 = x0 + lane, l1 = y0 + cy, l2 = (D == 4) ? z0 + cz : ct;
            int vmask = 0;  // axes along which the corner can step by +1
            if (l0 + 1 < ldx) vmask |= 1;
            if (l1 + 1 < ldy) vmask |= 2;
            if (D == 4 && l2 + 1 < ldz) vmask |= 4;
            if (ct + 1 < lt) vmask |= TBIT;
            cq.corner[idx] = pack_corner(l0, l1, (D == 4) ? l2 : 0, ct);
            unsigned long long ch = c_chains_by_vmask[D - 3][vmask];
            // a stream's window starts one slice before the new timestep: the
            // purely spatial simplices of that slice were counted already
            if (cfg.skip_first_spatial && ct == 0) ch &= c_time_chains[D - 3];
            cq.chains[idx] = ch;
          }
        }
      }
    }
    slot_a = slot_b;
  }
}

// Stage 2: exact SoS test and bit-exact solve of the queued chains.  One warp
// per candidate hypercube: its 2^D vertices' values are gathered once into
// shared memory, then each lane tests one chain; accepted simplices are
// compacted by warp ballot.
constexpr int kRefineWarps = 8;

template <typename T, int D>
__global__ void __launch_bounds__(kRefineWarps * 32, 2)
    refine_regular_kernel(RegularMesh mesh, FieldAccess fa, ExtractConfig cfg, CandidateQueue cq,
                          FeatureSink sink) {
  constexpr int M = D - 1;
  constexpr int NV = 1 << D;
  __shared__ T cube[kRefineWarps][NV][M];
  __shared__ unsigned band_tbl[kBandTable];
  fill_band_table<T>(band_tbl, threadIdx.x, blockDim.x);
  __syncthreads();
  const ChainTable& CT = c_chains[D - 3];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const unsigned n = min(*cq.count, cq.cap);
  const unsigned gw = blockIdx.x * kRefineWarps + wib;
  const unsigned nw = gridDim.x * kRefineWarps;
  for (unsigned c = gw; c < n; c += nw) {
    const unsigned long long pc = cq.corner[c];
    const unsigned long long chains = cq.chains[c];
    const long long l[4] = {(long long)(pc & 0xFFFF), (long long)((pc >> 16) & 0xFFFF),
                            (long long)((pc >> 32) & 0xFFFF), (long long)(pc >> 48)};
    long long g0[4];
    unsigned long long vid0 = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      // D = 3: the time coordinate is the third axis
      const long long lk = (D == 4) ? l[k] : (k < 2 ? l[k] : (k == 2 ? l[3] : 0));
      g0[k] = (k < D) ? lk + mesh.off[k] : 0;
      if (k < D) vid0 += (unsigned long long)g0[k] * mesh.gstride[k];
    }
    // gather the hypercube's vertex values (only vertices inside the mesh)
    for (int e = lane; e < NV * M; e += 32) {
      const int v = e / M, j = e % M;
      long long g[4];
      unsigned long long vid = 0;
      bool in = true;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        g[k] = (k < D) ? g0[k] + ((v >> k) & 1) : 0;
        if (k < D) {
          in &= g[k] - mesh.off[k] < mesh.ld[k];
          vid += (unsigned long long)g[k] * mesh.gstride[k];
        }
      }
      cube[wib][v][j] = in ? field_at<T>(fa, j, g, D, vid) : T(0);
    }
    __syncwarp();
    // cull words of the hypercube's vertices (absent outside the mesh)
    unsigned vw = kAbsent;
    if (lane < NV) {
      unsigned h[M];
#pragma unroll
      for (int j = 0; j < M; ++j) h[j] = hi_word<T>(cube[wib][lane][j]);
      bool in = true;
#pragma unroll
      for (int k = 0; k < D; ++k) in &= g0[k] + ((lane >> k) & 1) - mesh.off[k] < mesh.ld[k];
      vw = in ? vertex_word_hi<T, M>(h, band_tbl) : kAbsent;
    }
    for (int base = 0; base < CT.n; base += 32) {
      const int ch = base + lane;
      bool acc = false;
      double lam_out[4] = {0, 0, 0, 0};
      float bary_out[4] = {0.f, 0.f, 0.f, 0.f};
      float sc_out = 0.f;
      int mk[M + 1];
      mk[0] = 0;
      bool live = ch < CT.n && ((chains >> ch) & 1ull);
#pragma unroll
      for (int i = 0; i < M; ++i) mk[i + 1] = live ? CT.mask[ch][i] : 0;
      {
        unsigned wacc = kAbsent;
#pragma unroll
        for (int i = 0; i <= M; ++i) wacc &= __shfl_sync(0xFFFFFFFFu, vw, mk[i]);
        live = live && !word_culled(wacc);
      }
      if (live) {
        T vals[M + 1][M];
#pragma unroll
        for (int i = 0; i <= M; ++i)
#pragma unroll
          for (int j = 0; j < M; ++j) vals[i][j] = cube[wib][mk[i]][j];
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
              T sc = T(0);
#pragma unroll
              for (int i = 0; i <= M; ++i) {
                long long gv[4];
                unsigned long long vid = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                  gv[k] = (k < D) ? g0[k] + ((mk[i] >> k) & 1) : 0;
                  if (k < D) vid += (unsigned long long)gv[k] * mesh.gstride[k];
                }
                sc = F::add(sc, F::mul(lam[i], scalar_at<T>(fa, gv, D, vid)));
              }
              sc_out = (float)sc;
            }
            if (cfg.refined) {
              double rr[M + 1];
              if (solve_refined<M, T>(vals, rr))
#pragma unroll
                for (int i = 0; i <= M; ++i) lam_out[i] = rr[i];
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
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// host side

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
  unsigned long long byv[2][16];
  for (int t = 0; t < 2; ++t)
    for (int vm = 0; vm < 16; ++vm) {
      unsigned long long m = 0;
      for (int c = 0; c < h[t].n; ++c)
        if ((h[t].mask[c][t + 1] & ~vm) == 0) m |= 1ull << c;  // last vertex mask is index m-1 = t+1
      byv[t][vm] = m;
    }
  cudaMemcpyToSymbol(c_chains_by_vmask, byv, sizeof(byv));
  unsigned long long tc[2] = {0, 0};
  for (int t = 0; t < 2; ++t) {
    const int tbit = 1 << (t + 2);  // time axis: bit d - 1
    for (int c = 0; c < h[t].n; ++c)
      if (h[t].mask[c][t + 1] & tbit) tc[t] |= 1ull << c;
  }
  cudaMemcpyToSymbol(c_time_chains, tc, sizeof(tc));
}


// cuTensorMapEncodeTiled is a driver API entry point; it is resolved through
// the runtime so that the library carries no link-time libcuda dependency.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  });
  return fn;
}

static bool encode_map(CUtensorMap* map, bool f64, const void* base, int rank, const uint64_t* dims,
                       const uint64_t* strides_bytes, const uint32_t* box) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return false;
  cuuint64_t gd[5], gs[4];
  cuuint32_t bx[5], es[5];
  for (int i = 0; i < rank; ++i) {
    gd[i] = dims[i];
    bx[i] = box[i];
    es[i] = 1;
    if (i) gs[i - 1] = strides_bytes[i - 1];
  }
  CUresult r = encode(
      map, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank,
      const_cast<void*>(base), gd, gs, bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename T, int D, bool MULTI>
static cudaError_t launch_t(const RegularMesh& mesh, const FieldAccess& fa, const ExtractConfig& cfg,
                            const CandidateQueue& cq, unsigned* err, cudaStream_t st, bool allow_tma,
                            int* used_tma) {
  using G = Geo<T, D, MULTI>;
  constexpr int M = D - 1;
  const size_t es = sizeof(T);

  // TMA applies when every box starts on a 16-byte boundary and the array
  // strides are multiples of 16 bytes: inner coordinate = array x * (M or 1)
  CUtensorMap maps[3];
  memset(maps, 0, sizeof(maps));
  bool tma = allow_tma && !fa.per_vertex;
  const long long ax0 = mesh.off[0] - fa.shift[0];
  const size_t inner_es = (MULTI ? M : 1) * es;
  if (tma) {
    if (((size_t)ax0 * inner_es) % 16 != 0) tma = false;
    if (((size_t)fa.adims[0] * inner_es) % 16 != 0) tma = false;
    for (int j = 0; j < (MULTI ? 1 : M); ++j)
      if (((uintptr_t)fa.comp[j]) % 16 != 0) tma = false;
    for (int k = 0; k < D; ++k)
      if (fa.adims[k] * (k == 0 ? (MULTI ? M : 1) : 1) > 0x7FFFFFFFll) tma = false;
  }
  if (tma) {
    uint64_t dims[4], strides[3];
    uint32_t box[4];
    dims[0] = (uint64_t)fa.adims[0] * (MULTI ? M : 1);
    box[0] = (uint32_t)(G::VXBOX * (MULTI ? M : 1));
    uint64_t s = dims[0] * es;
    for (int k = 1; k < D; ++k) {
      dims[k] = (uint64_t)fa.adims[k];
      strides[k - 1] = s;
      s *= dims[k];
    }
    box[1] = G::VY;
    if (D == 4) {
      box[2] = G::VZ;
      box[3] = 1;
    } else {
      box[2] = 1;
    }
    for (int j = 0; j < (MULTI ? 1 : M) && tma; ++j)
      tma = encode_map(&maps[j], sizeof(T) == 8, fa.comp[j], D, dims, strides, box);
  }
  if (used_tma) *used_tma = tma ? 1 : 0;
  const size_t shm = G::SMEM;
  const long long lt = mesh.ld[D - 1];
  const unsigned nchunks = (unsigned)((lt + cfg.tchunk - 1) / cfg.tchunk);
  const unsigned ntiles = (unsigned)cfg.tiles[0] * cfg.tiles[1] * cfg.tiles[2];
  dim3 grid(ntiles, nchunks);
  cudaError_t e;
  if (tma) {
    auto k = extract_regular_kernel<T, D, MULTI, true>;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e) return e;
    k<<<grid, kThreads, shm, st>>>(maps[0], maps[1], maps[2], mesh, fa, cfg, cq, err);
  } else {
    auto k = extract_regular_kernel<T, D, MULTI, false>;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e) return e;
    k<<<grid, kThreads, shm, st>>>(maps[0], maps[1], maps[2], mesh, fa, cfg, cq, err);
  }
  return cudaGetLastError();
}

template <typename T, int D>
static cudaError_t launch_td(const RegularMesh& mesh, const FieldAccess& fa, const ExtractConfig& cfg,
                             const CandidateQueue& cq, unsigned* err, cudaStream_t st, bool allow_tma,
                             int* used_tma) {
  const bool multi = !fa.per_vertex && fa.estride[0] == D - 1;  // interleaved components
  return multi ? launch_t<T, D, true>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma)
               : launch_t<T, D, false>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma);
}

void regular_tile(int d, int* tx, int* ty, int* tz) {
  if (d == 4) {
    *tx = Tile<4>::TX;
    *ty = Tile<4>::TY;
    *tz = Tile<4>::TZ;
  } else {
    *tx = Tile<3>::TX;
    *ty = Tile<3>::TY;
    *tz = Tile<3>::TZ;
  }
}

cudaError_t launch_extract_regular(int f64, const RegularMesh& mesh, const FieldAccess& fa,
                                   const ExtractConfig& cfg, const CandidateQueue& cq, unsigned* err,
                                   cudaStream_t st, bool allow_tma, int* used_tma) {
  if (mesh.d == 4)
    return f64 ? launch_td<double, 4>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma)
               : launch_td<float, 4>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma);
  return f64 ? launch_td<double, 3>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma)
             : launch_td<float, 3>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma);
}

cudaError_t launch_refine_regular(int f64, const RegularMesh& mesh, const FieldAccess& fa,
                                  const ExtractConfig& cfg, const CandidateQueue& cq,
                                  const FeatureSink& sink, int num_sms, cudaStream_t st) {
  const int blocks = num_sms * 8;
  const int thr = kRefineWarps * 32;
  if (mesh.d == 4) {
    if (f64) refine_regular_kernel<double, 4><<<blocks, thr, 0, st>>>(mesh, fa, cfg, cq, sink);
    else refine_regular_kernel<float, 4><<<blocks, thr, 0, st>>>(mesh, fa, cfg, cq, sink);
  } else {
    if (f64) refine_regular_kernel<double, 3><<<blocks, thr, 0, st>>>(mesh, fa, cfg, cq, sink);
    else refine_regular_kernel<float, 3><<<blocks, thr, 0, st>>>(mesh, fa, cfg, cq, sink);
  }
  return cudaGetLastError();
}

}  // namespace ftk2b
