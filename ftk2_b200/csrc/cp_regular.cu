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

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "cp_batch.h"
#include "cp_cull.cuh"
#include "cp_device.cuh"
#include "cp_field.cuh"
#include "cp_internal.h"
#include "cp_pdl.cuh"

namespace ftk2b {

__constant__ ChainTable c_chains[2];  // [0]: d=3, m=2 (12 chains); [1]: d=4, m=3 (60)
// chains whose vertices all stay inside the mesh, by the mask of axes along
// which a corner may step: [0][vmask] for d = 3, [1][vmask] for d = 4
__constant__ unsigned long long c_chains_by_vmask[2][16];
// chains whose last vertex steps along the time axis
__constant__ unsigned long long c_time_chains[2];
// masks of vertices 1..m of every chain, a byte each (m1 | m2 << 8 | m3 << 16),
// 0 past the table: read with lane-dependent chain indices, which the
// constant bank would serialise, so it lives in global memory
__device__ unsigned g_chain_pk[2][kMaxChains];

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

// Bounded wait for the phase of the given parity (at most `limit` polls);
// false if it never completed.
constexpr int kWaitPolls = 1 << 22;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit = kWaitPolls) {
  const unsigned a = smem_addr(bar);
  for (int it = 0; it < limit; ++it) {
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

// The mbarrier receives one arrival when every cp.async this thread issued
// before has landed (.noinc: the barrier's expected count covers it).
__device__ __forceinline__ void cp_async_mbar_arrive(unsigned long long* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
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

// Per-thread asynchronous global -> shared copies (each thread later reads
// back only what it copied itself, after cp.async.wait_group).
__device__ __forceinline__ void cp_async_16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_small(void* dst, const void* src) {
  static_assert(N == 4 || N == 8, "cp.async.ca copies 4, 8 or 16 bytes");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src), "n"(N)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// element copy with zero fill: src_bytes = 0 writes zeros without reading
template <int N>
__device__ __forceinline__ void cp_async_zfill(void* dst, const void* src, unsigned src_bytes) {
  static_assert(N == 4 || N == 8, "element copies of 4 or 8 bytes");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src), "n"(N), "r"(src_bytes)
               : "memory");
}

// ---------------------------------------------------------------------------

template <int D> struct Tile;
template <> struct Tile<4> {
  // warp w owns corner row cy = w % 8 and corner z levels 2 (w / 8) .. +1
  static constexpr int TX = 32, TY = 8, TZ = 4;
};
template <> struct Tile<3> {
  // warp w < 15 owns corner rows cy = 2w, 2w + 1 (warp 15 none): 31 x 33
  // vertex slots fit the block's 512 threads twice (32 rows would take 1089
  // slots, a third pass over mostly empty slots)
  static constexpr int TX = 32, TY = 30, TZ = 1;
};

constexpr int kThreads = 512;
// surviving hypercubes a block collects in shared memory before it reserves
// queue space for all of them with one atomic (more go to the queue directly)
constexpr int kCandBuf = 256;
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
  static constexpr int BOX_BYTES = MULTI ? round128(COMP_RAW * M) : COMP * M;
  // row staging (arrays a TMA tensor map cannot describe): box row r of
  // a slice goes to bytes [r * ROWB, (r + 1) * ROWB) of the buffer, its data
  // starting at the row's source address mod 16 (rows component-major for
  // separate arrays)
  static constexpr int ROWS = VY * VZ * (MULTI ? 1 : M);
  static constexpr int ROWB = ((VX * (MULTI ? M : 1) * (int)sizeof(T) + 15) & ~15) + 32;
  static constexpr int BULK_BYTES = round128(ROWS * ROWB);
  static constexpr int BYTES = BOX_BYTES > BULK_BYTES ? BOX_BYTES : BULK_BYTES;  // one slice buffer
  static constexpr int TX_BYTES = COMP_RAW * M;                          // bytes TMA delivers
  static constexpr int COMP_ELEMS = COMP / (int)sizeof(T);
  static constexpr int WORDS = 2 * BYTES;                                // offset of the word slots
  // the block's candidate buffer (corner, chains) and its count, after the word slots
  static constexpr int CAND = WORDS + 2 * VSP * 4;
  // chunk staging: the source address of every box row
  static constexpr int ROWSRC = CAND + 16 * kCandBuf + 16;
  static constexpr int SMEM = ROWSRC + 8 * ROWS;
};

__device__ __forceinline__ unsigned long long pack_corner(long long x, long long y, long long z,
                                                          long long t) {
  return (unsigned long long)x | ((unsigned long long)y << 16) | ((unsigned long long)z << 32) |
         ((unsigned long long)t << 48);
}

// The block's buffered candidates into the queue with one reservation:
// ccount[0] holds how many the block found (those past kCandBuf went to the
// queue directly), cbuf their (corner, chains) pairs.  Every thread calls
// it after a block barrier that follows the last candidate writes; it
// leaves ccount[0] = 0, and the buffer may take new candidates after the
// next block barrier.
__device__ __forceinline__ void flush_candidates(const unsigned long long* cbuf, unsigned* ccount,
                                                 const CandidateQueue& cq, unsigned field_id) {
  const unsigned nc = min(ccount[0], (unsigned)kCandBuf);
  if (threadIdx.x == 0) ccount[1] = nc ? atomicAdd(cq.count, nc) : 0u;
  __syncthreads();
  if (threadIdx.x == 0) ccount[0] = 0;
  const unsigned cbase = ccount[1];
  for (unsigned i = threadIdx.x; i < nc; i += kThreads) {
    const unsigned gi = cbase + i;
    if (gi < cq.cap) {
      cq.corner[gi] = cbuf[2 * i];
      cq.chains[gi] = cbuf[2 * i + 1];
      if (cq.field) cq.field[gi] = field_id;
    }
  }
}

// Stage 1: stream the field through shared memory, cull hypercubes, queue
// the survivors with the chains whose own vertices survive the cull.
//
// cull_tile marches one tile over the corner time steps of one chunk.  The
// block's two slice buffers, word slots, mbarriers and band table are the
// caller's: bar[0..1] take TMA tensor copies (one arrival each), bar[2] is
// the failure-path barrier that nothing completes, bar[3..4] take the chunk
// copies of the block's threads (kThreads arrivals each).  Bit b of ph is
// the parity of the phases barrier b (b = 0, 1) or 3 + b - 2 (b = 2, 3) has
// completed before this call (so that a persistent block can march many
// tiles); it is advanced past the copies this call waits for.  Surviving
// hypercubes go to the candidate buffer cbuf / ccount (flush_candidates);
// with defer, the call first flushes what the block's previous tile left
// there (as candidates of field pend_field) and leaves its own for the
// next call, else it flushes its own at the end.  Returns false when a
// bounded wait gave up (the error flag is set).
template <typename T, int D, bool MULTI, bool TMA>
__device__ __forceinline__ bool cull_tile(const CUtensorMap* map0, const CUtensorMap* map1,
                                          const CUtensorMap* map2, const RegularMesh& mesh, const FieldAccess& fa,
                                          const ExtractConfig& cfg, const CandidateQueue& cq, unsigned* err,
                                          int tile, int chunk, unsigned char* smem, unsigned long long* bar,
                                          const unsigned* band_tbl, unsigned& ph,
                                          unsigned long long* cbuf, unsigned* ccount, bool defer,
                                          unsigned pend_field) {
  using G = Geo<T, D, MULTI>;
  constexpr int M = D - 1;
  constexpr int TX = G::TX, TY = G::TY, TZ = G::TZ;
  constexpr int VX = G::VX, VY = G::VY, VZ = G::VZ, VS = G::VS, VPT = G::VPT, VSP = G::VSP;
  constexpr int TBIT = 1 << (D - 1);  // mask bit of the time axis
  constexpr int HW = sizeof(T) / 4;   // the high 32-bit word of an element is its last
  static_assert(D == 3 ? kWarps * kRows >= TY : kWarps == TY * (TZ / kRows),
                "every corner row of the tile belongs to exactly one warp");
  unsigned* const Wb = reinterpret_cast<unsigned*>(smem + G::WORDS);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;

  // tile origin (local coordinates)
  int tix = tile;
  const int x0 = (tix % cfg.tiles[0]) * TX;
  tix /= cfg.tiles[0];
  const int y0 = (tix % cfg.tiles[1]) * TY;
  tix /= cfg.tiles[1];
  const int z0 = (D == 4) ? tix * TZ : 0;
  const int ldx = (int)mesh.ld[0], ldy = (int)mesh.ld[1], ldz = (D == 4) ? (int)mesh.ld[2] : 1;
  // time in int: local dims are below 2^16
  const int lt = (int)mesh.ld[D - 1];
  const int t0 = chunk * cfg.tchunk;
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

  // 16-byte chunk copies of the box rows stage arrays that TMA cannot
  // describe (rows not 16-byte multiples, misaligned offsets); per-vertex
  // arrays keep element copies
  const bool bulk = !TMA && !fa.per_vertex;
  const bool mbar = TMA || bulk;

  // per-thread vertex slots of a slice, fixed for the whole time march:
  // element offset of component 0 in a slice buffer (bulk staging: byte
  // offset from the row's slot, and the row's source offset mod 16 without
  // the time term, 4 bits per slot) and an absence mask; set once the first
  // slices' copies are in flight
  int voff[VPT];
  unsigned vshift = 0;
  unsigned vinv[VPT];  // ~0 for slots outside the mesh (absent under AND), else 0
  auto set_slots = [&]() {
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      const int i = tid + u * kThreads;
      const int vx = i % VX, vy = (i / VX) % VY, vz = i / (VX * VY);
      const bool in = i < VS && x0 + vx < ldx && y0 + vy < ldy && (D == 3 || z0 + vz < ldz);
      if (bulk) {
        voff[u] = in ? (vz * VY + vy) * G::ROWB + vx * (MULTI ? M : 1) * (int)sizeof(T) : 0;
        long long e = (long long)(x0 + aoff[0]) * fa.estride[0] + (long long)(y0 + vy + aoff[1]) * fa.estride[1];
        if (D == 4) e += (long long)(z0 + vz + aoff[2]) * fa.estride[2];
        vshift |= (unsigned)((e * (long long)sizeof(T)) & 15) << (4 * u);
      } else {
        voff[u] = in ? (MULTI ? ((vz * VY + vy) * G::VXBOX + vx) * M : (vz * VY + vy) * G::VXBOX + vx) : 0;
      }
      vinv[u] = in ? 0u : kAbsent;
    }
  };
  // source address mod 16 of each array, and the time axis' element stride
  unsigned pbase = 0;
#pragma unroll
  for (int j = 0; j < (MULTI ? 1 : M); ++j)
    pbase |= (unsigned)(reinterpret_cast<uintptr_t>(fa.comp[j]) & 15) << (4 * j);
  const long long tstride = fa.estride[D - 1];
  // chunk staging: the source address of every box row at array time 0 (0
  // for rows outside the mesh) in shared memory, and the bytes of a row's
  // local vertices; the block's threads copy the rows in 16-byte blocks
  unsigned long long* const rsrc = reinterpret_cast<unsigned long long*>(smem + G::ROWSRC);
  const int rbytes = min(VX, ldx - x0) * (MULTI ? M : 1) * (int)sizeof(T);
  if (bulk) {
    for (int r = tid; r < G::ROWS; r += kThreads) {
      const int rr = MULTI ? r : r % (VY * VZ);
      const int j = MULTI ? 0 : r / (VY * VZ);
      const int vy = rr % VY, vz = rr / VY;
      unsigned long long a = 0;
      if (y0 + vy < ldy && (D == 3 || z0 + vz < ldz)) {
        long long e = (long long)(x0 + aoff[0]) * fa.estride[0] + (long long)(y0 + vy + aoff[1]) * fa.estride[1];
        if (D == 4) e += (long long)(z0 + vz + aoff[2]) * fa.estride[2];
        a = (unsigned long long)(reinterpret_cast<uintptr_t>(j == 0 ? fa.comp[0] : (j == 1 ? fa.comp[1] : fa.comp[2])) +
                                 (uintptr_t)(e * (long long)sizeof(T)));
      }
      rsrc[r] = a;
    }
  }
  // chunk copies and TMA copies complete on separate barriers (different
  // arrival counts); bits 2..3 of ph hold the phase parities of the chunk
  // barriers
  unsigned long long* const sb = bulk ? bar + 3 : bar;
  const int sp = bulk ? 2 : 0;

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
          if constexpr (D == 4) tma_load_4d(dst0, map0, cx, cy, z0 + aoff[2], tcoord(s), &bar[buf]);
          else tma_load_3d(dst0, map0, cx, cy, tcoord(s), &bar[buf]);
        } else {
          const CUtensorMap* maps[3] = {map0, map1, map2};
#pragma unroll
          for (int j = 0; j < M; ++j) {
            if constexpr (D == 4)
              tma_load_4d(dst0 + j * G::COMP, maps[j], cx, cy, z0 + aoff[2], tcoord(s), &bar[buf]);
            else
              tma_load_3d(dst0 + j * G::COMP, maps[j], cx, cy, tcoord(s), &bar[buf]);
          }
        }
      }
    } else if (bulk) {
      // every thread: 16-byte blocks c = tid + k * kThreads of the box rows
      // (CPR blocks per row slot), each row from the 16-byte block of its
      // first element to the block of its last (an aligned 16-byte block
      // never crosses a page, so the bytes read around the row lie in pages
      // the row occupies); then one arrival on the slice's barrier once the
      // thread's copies have landed
      constexpr int CPR = G::ROWB / 16;
      constexpr int CPT = (G::ROWS * CPR + kThreads - 1) / kThreads;
      const uintptr_t tb = (uintptr_t)((long long)tcoord(s) * tstride * (long long)sizeof(T));
#pragma unroll
      for (int k = 0; k < CPT; ++k) {
        const int c = tid + k * kThreads;
        if (c < G::ROWS * CPR) {
          const int r = c / CPR, q = c - r * CPR;
          const unsigned long long b = rsrc[r];
          const uintptr_t src = (uintptr_t)b + tb;
          const uintptr_t lo = (src & ~(uintptr_t)15) + 16 * (uintptr_t)q;
          if (b && lo < src + (uintptr_t)rbytes && FTK2B_CHECK(r * G::ROWB + 16 * q + 16 <= G::BYTES, err))
            cp_async_16(dst0 + r * G::ROWB + 16 * q, reinterpret_cast<const void*>(lo));
        }
      }
      cp_async_mbar_arrive(&sb[buf]);
    } else {
      // per-thread asynchronous element copies into the same layout (zeros
      // outside the array), one commit group per slice
      T* dst = reinterpret_cast<T*>(dst0);
      constexpr int NPER = G::VXBOX * VY * VZ;
      if (!fa.per_vertex) {
        // one box row per warp at a time: (vz, vy) rows of VXBOX * M
        // interleaved elements, or (j, vz, vy) rows of VXBOX elements
        constexpr int RW = MULTI ? G::VXBOX * M : G::VXBOX;
        constexpr int NROWS = VY * VZ * (MULTI ? 1 : M);
        const long long ax = (long long)x0 + aoff[0];  // array x of the box's first vertex
        const long long at = (long long)tcoord(s);
        for (int row = warp; row < NROWS; row += kWarps) {
          const int j = MULTI ? 0 : row / (VY * VZ);
          const int rr = MULTI ? row : row % (VY * VZ);
          const int vy = rr % VY, vz = rr / VY;
          const long long a1 = (long long)y0 + vy + aoff[1];
          const long long a2 = (D == 4) ? (long long)z0 + vz + aoff[2] : at;
          bool row_in = a1 >= 0 && a1 < fa.adims[1] && a2 >= 0 && a2 < fa.adims[2];
          long long ob = a1 * fa.estride[1] + a2 * fa.estride[2];
          if (D == 4) {
            row_in = row_in && at >= 0 && at < fa.adims[3];
            ob += at * fa.estride[3];
          }
          // elements of the row inside the array along x
          const long long xin = fa.adims[0] - ax;
          const long long xe = xin * (MULTI ? M : 1);
          const int nin = !row_in || xin <= 0 ? 0 : (xe < RW ? (int)xe : RW);
          const T* src = static_cast<const T*>(fa.comp[j]) + ob + ax * fa.estride[0];
          T* d = MULTI ? dst + (vz * VY + vy) * RW : dst + j * G::COMP_ELEMS + (vz * VY + vy) * G::VXBOX;
          for (int q = lane; q < RW; q += 32) {
            const bool in = q < nin && ax >= 0;
            // separate arrays step by estride[0] along x; interleaved rows are contiguous
            const long long so = MULTI ? q : (long long)q * fa.estride[0];
            cp_async_zfill<sizeof(T)>(d + q, in ? src + so : static_cast<const T*>(fa.comp[j]),
                                      in ? (unsigned)sizeof(T) : 0u);
          }
        }
      } else {
        for (int e = tid; e < NPER * M; e += kThreads) {
          const int j = MULTI ? e % M : e / NPER;
          const int r = MULTI ? e / M : e % NPER;
          const int vx = r % G::VXBOX;
          const int vy = (r / G::VXBOX) % VY;
          const int vz = r / (G::VXBOX * VY);
          const long long l[4] = {x0 + vx, y0 + vy, (D == 4) ? z0 + vz : (long long)s, (long long)s};
          // 1-D per-vertex arrays: index by vertex id, only inside the mesh
          bool in = true;
          long long o = 0;
#pragma unroll
          for (int k = 0; k < D; ++k) {
            in &= l[k] < mesh.ld[k];
            o += (l[k] + mesh.off[k]) * (long long)mesh.gstride[k];
          }
          const T* src = static_cast<const T*>(fa.comp[j]) + (in ? o : 0);
          T* d = MULTI ? &dst[((vz * VY + vy) * G::VXBOX + vx) * M + j]
                       : &dst[j * G::COMP_ELEMS + (vz * VY + vy) * G::VXBOX + vx];
          cp_async_zfill<sizeof(T)>(d, src, in ? (unsigned)sizeof(T) : 0u);
        }
      }
      cp_async_commit();
    }
  };
  // every thread waits for the slice's TMA phase itself (try_wait suspends
  // in hardware); returns false when the bounded wait gave up
  auto wait = [&](int s, int buf) -> bool {
    if (mbar) {
      return mbar_wait(&sb[buf], ((ph >> (sp + buf)) + (unsigned)((s - t0) >> 1)) & 1u);
    } else {
      // slice s + 1 (when it exists) was issued after s: one group may stay
      // in flight; then every thread's copies of slice s are visible
      if (s + 1 <= s_end) cp_async_wait<1>();
      else cp_async_wait<0>();
      __syncthreads();
      return true;
    }
  };
  // cull words of slice s into w[] (the thread's slots; absent outside the mesh)
  auto words = [&](int buf, int s, unsigned (&w)[VPT]) {
    const unsigned* r = reinterpret_cast<const unsigned*>(smem + buf * G::BYTES) + (HW - 1);
    if (bulk) {
      const unsigned char* rb = smem + buf * G::BYTES + 4 * (HW - 1);
      const unsigned ts = (unsigned)(((long long)tcoord(s) * tstride * (long long)sizeof(T)) & 15);
#pragma unroll
      for (int u = 0; u < VPT; ++u) {
        if (u == VPT - 1 && VS < VSP && tid + u * kThreads >= VS) {  // a padding slot: no vertex
          w[u] = kAbsent;
          continue;
        }
        unsigned h[M];
        const unsigned su = (vshift >> (4 * u)) + ts;
#pragma unroll
        for (int j = 0; j < M; ++j) {
          const unsigned sh = (su + (pbase >> (4 * (MULTI ? 0 : j)))) & 15u;
          const int o = voff[u] + (MULTI ? j * (int)sizeof(T) : j * VY * VZ * G::ROWB) + (int)sh;
          h[j] = FTK2B_CHECK(o >= 0 && o + 4 * HW <= G::BYTES, err) ? *reinterpret_cast<const unsigned*>(rb + o) : 0u;
        }
        const unsigned x = vertex_word_hi<T, M>(h, band_tbl);
        w[u] = x | vinv[u];
      }
      return;
    }
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      if (u == VPT - 1 && VS < VSP && tid + u * kThreads >= VS) {  // a padding slot: no vertex
        w[u] = kAbsent;
        continue;
      }
      unsigned h[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const int ix = HW * (MULTI ? voff[u] + j : voff[u] + j * G::COMP_ELEMS);
        h[j] = FTK2B_CHECK(ix >= 0 && 4 * (ix + HW) <= G::BYTES, err) ? r[ix] : 0u;
      }
      const unsigned x = vertex_word_hi<T, M>(h, band_tbl);
      w[u] = x | vinv[u];
    }
  };
  // Each thread keeps its slots' words of the previous slice in registers
  // and stores, per time step, the AND of the two slices' words: a
  // hypercube's 2^D vertices then take 2^(D-1) shared-memory words.
  unsigned prev[VPT];

  if (!defer && tid == 0) ccount[0] = 0;
  // the previous tile of a persistent block is done with every buffer
  __syncthreads();
  issue(t0, 0);
  if (t0 + 1 <= s_end) issue(t0 + 1, 1);
  set_slots();
  // a persistent block's previous tile left its candidates in the buffer:
  // reserve their queue space while this tile's first slices are in flight
  if (defer) flush_candidates(cbuf, ccount, cq, pend_field);
  {
    bool ok = wait(t0, 0);
    // failure-path check (host option): after the first slice has landed,
    // wait on bar[2], which nothing ever completes, with the caller's short
    // poll bound; the block then leaves through the bounded-wait error path
    if (ok && mbar && cfg.stall_polls > 0) ok = mbar_wait(&bar[2], 0u, cfg.stall_polls);
    if (ok) words(0, t0, prev);
    if (__syncthreads_or(!ok)) {
      // give the other copy in flight a bounded chance to land before leaving
      if (mbar && t0 + 1 <= s_end) mbar_wait(&sb[1], (ph >> (sp + 1)) & 1u);
      if (tid == 0) atomicOr(err, 2u);
      return false;
    }
  }
  if (t0 + 2 <= s_end) issue(t0 + 2, 0);

  // corner validity per (lane, row) does not change along time
  const int cyw = (D == 4) ? warp % TY : warp * kRows;
  const int czw = (D == 4) ? (warp / TY) * kRows : 0;
  unsigned row_valid = 0;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    const int cy = (D == 4) ? cyw : cyw + q;
    const int cz = (D == 4) ? czw + q : 0;
    if (x0 + lane < ldx && cy < TY && y0 + cy < ldy && (D == 3 || z0 + cz < ldz)) row_valid |= 1u << q;
  }
  const bool has_rows = D == 4 || cyw < TY;  // warp-uniform: the warp owns corner rows of the tile

  for (int ct = t0; ct < t1; ++ct) {
    const int s = ct + 1;
    // time-pair words of step ct (slices ct and s; slots alternate by step)
    unsigned* const A = Wb + ((ct - t0) & 1) * VSP;
    bool ok = true;
    if (s <= s_end) {
      const int buf = (s - t0) & 1;
      ok = wait(s, buf);
      if (ok) {
        unsigned cur[VPT];
        words(buf, s, cur);
#pragma unroll
        for (int u = 0; u < VPT; ++u) {
          A[tid + u * kThreads] = prev[u] & cur[u];
          prev[u] = cur[u];
        }
      }
    } else {  // no slice after the last one: the step's words are slice ct's
#pragma unroll
      for (int u = 0; u < VPT; ++u) A[tid + u * kThreads] = prev[u];
    }
    // the one block barrier of the step: words of step ct are visible, slice
    // s's raw buffer is free, and every warp has finished culling step ct - 1
    if (__syncthreads_or(!ok)) {
      const int ob = ((s - t0) & 1) ^ 1;
      if (mbar && s + 1 <= s_end) mbar_wait(&sb[ob], ((ph >> (sp + ob)) + (unsigned)((s + 1 - t0) >> 1)) & 1u);
      if (tid == 0) atomicOr(err, 2u);
      return false;
    }
    if (s + 2 <= s_end) issue(s + 2, (s - t0) & 1);
    if (!has_rows) continue;

    // ---- hypercube cull: lanes along x, kRows corner rows per warp
    unsigned R[kRows + 1];
#pragma unroll
    for (int q = 0; q <= kRows; ++q) {
      unsigned r, e;
      if constexpr (D == 4) {
        const int i0 = ((czw + q) * VY + cyw) * VX + lane, i1 = i0 + VX;
        const bool okA = FTK2B_CHECK(i1 + 1 < VSP, err);
        r = okA ? A[i0] & A[i1] : kAbsent;
        e = (lane == 31 && okA) ? (A[i0 + 1] & A[i1 + 1]) : kAbsent;
      } else {
        const int i0 = (cyw + q) * VX + lane;
        const bool okA = FTK2B_CHECK(i0 + 1 < VSP, err);
        r = okA ? A[i0] : kAbsent;
        e = (lane == 31 && okA) ? A[i0 + 1] : kAbsent;
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
        // mesh (the exact-test kernel applies the per-simplex word test),
        // first into the block's buffer
        unsigned basei = 0;
        if (lane == 0) basei = atomicAdd(ccount, (unsigned)__popc(ball));
        basei = __shfl_sync(0xFFFFFFFFu, basei, 0);
        if (keep) {
          const unsigned idx = basei + __popc(ball & ((1u << lane) - 1));
          const int l0 = x0 + lane, l1 = y0 + cy, l2 = (D == 4) ? z0 + cz : ct;
          int vmask = 0;  // axes along which the corner can step by +1
          if (l0 + 1 < ldx) vmask |= 1;
          if (l1 + 1 < ldy) vmask |= 2;
          if (D == 4 && l2 + 1 < ldz) vmask |= 4;
          if (ct + 1 < lt) vmask |= TBIT;
          const unsigned long long corner = pack_corner(l0, l1, (D == 4) ? l2 : 0, ct);
          unsigned long long ch = c_chains_by_vmask[D - 3][vmask];
          // a stream's window starts one slice before the new timestep: the
          // purely spatial simplices of that slice were counted already
          if (cfg.skip_first_spatial && ct == 0) ch &= c_time_chains[D - 3];
          if (idx < kCandBuf) {
            cbuf[2 * idx] = corner;
            cbuf[2 * idx + 1] = ch;
          } else {
            const unsigned gi = atomicAdd(cq.count, 1u);
            if (gi < cq.cap) {
              cq.corner[gi] = corner;
              cq.chains[gi] = ch;
              if (cq.field) cq.field[gi] = cq.field_id;
            }
          }
        }
      }
    }
  }
  // the block's buffered candidates into the queue (deferred: by the
  // block's next tile, or after its last)
  if (!defer) {
    __syncthreads();
    flush_candidates(cbuf, ccount, cq, cq.field_id);
  }
  if (mbar) {
    // slices t0 .. s_end alternate buffers 0, 1, 0, ...
    const unsigned nsl = (unsigned)(s_end - t0 + 1);
    ph ^= ((((nsl + 1) >> 1) & 1u) << sp) | (((nsl >> 1) & 1u) << (sp + 1));
  }
  return true;
}

template <typename T, int D, bool MULTI, bool TMA>
__global__ void __launch_bounds__(kThreads, 2)
    extract_regular_kernel(const __grid_constant__ CUtensorMap map0,
                           const __grid_constant__ CUtensorMap map1,
                           const __grid_constant__ CUtensorMap map2, RegularMesh mesh, FieldAccess fa,
                           ExtractConfig cfg, CandidateQueue cq, unsigned* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned long long bar[5];
  __shared__ unsigned band_tbl[kBandTable];
  fill_band_table<T>(band_tbl, threadIdx.x, kThreads);  // visible after the tile's first barrier
  // TMA tensor copies complete on bar[0..1], the threads' chunk copies on
  // bar[3..4]; bar[2] only serves the failure-path check and never completes
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    mbar_init(&bar[3], kThreads);
    mbar_init(&bar[4], kThreads);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  unsigned ph = 0;  // phase parities of bar[0], bar[1], bar[3], bar[4]
  using G = Geo<T, D, MULTI>;
  cull_tile<T, D, MULTI, TMA>(&map0, &map1, &map2, mesh, fa, cfg, cq, err, (int)blockIdx.x, (int)blockIdx.y, smem,
                              bar, band_tbl, ph, reinterpret_cast<unsigned long long*>(smem + G::CAND),
                              reinterpret_cast<unsigned*>(smem + G::CAND + 16 * kCandBuf), false, 0u);
}

// ---------------------------------------------------------------------------
// Stage 1, tile-statistics form (cull mode 1), in three launches.
//
// 1. plane_stats_kernel: per (slice, z plane, y-tile, x-tile), the minimum
//    and maximum of every component over the tile's TX + 1 by TY + 1 vertices
//    of that plane, kept as order-preserving integer keys of the high 32-bit
//    words; every vertex row is read once with coalesced loads.
// 2. tile_runs_kernel: one thread per tile merges the TZ + 1 planes of its
//    box per slice, decides every tile-step (the hypercubes between slices c
//    and c+1) and lists the runs of consecutive steps that survive.  A step is dropped when
//      * every magnitude is below 4e-13 (the first pivot of every solve is
//        below 1e-12, zero_crossing.hpp:72), or
//      * some component is strictly positive above kappa * M on every vertex,
//        or strictly negative below -kappa * M (M = the step's largest
//        magnitude; kappa = 2^-24 for double, 2^-12 for float): the argument
//        of the per-vertex cull words applied to the whole tile-step.
//    The bounds are conservative: minima of high words are lower bounds of
//    positive values and maxima upper bounds of negative ones, M is rounded up.
// 3. run_cull_kernel: persistent CTAs walk the runs; thread 0 streams each
//    run's slices, in order and across run boundaries, through a ring of
//    kNbuf TMA buffers, and the block computes the per-vertex words and the
//    per-hypercube cull of every step of the run, as extract_regular_kernel
//    does for a whole tile.
constexpr int kNbuf = 4;

template <typename T, int D, bool MULTI>
struct Geo2 {
  using G = Geo<T, D, MULTI>;
  static constexpr int WORDS = kNbuf * G::BYTES;     // offset of the word slots
  // word slots: one per raw buffer (the words of stream slice q in slot
  // q % kNbuf) and one that stays all-absent (the missing next slice of a
  // run's last corner slice)
  static constexpr int SMEM = WORDS + (kNbuf + 1) * G::VSP * 4;
};

__device__ __forceinline__ int ord_key(unsigned h) {
  // signed-integer order of IEEE sign-magnitude words
  return (int)(h ^ ((unsigned)((int)h >> 31) >> 1));
}

constexpr int kStatsWarps = 8;

// One warp per (chunk of XT x-tiles, y-tile, z plane, slice) of separate
// component arrays: it streams the TY + 1 vertex rows of its y-tile (the next
// tile's first row included) over the chunk's XT * TX + 1 vertices, lane l
// loading vertex 32 g + l of every component (g: 32-vertex group), and writes
// per x-tile the minimum and maximum order key of every component over the
// tile's TX + 1 x-vertices and TY + 1 rows of this plane.  Group XT holds the
// chunk's halo vertex (the next tile's first vertex), which belongs to the
// last tile of the chunk as well.  The z planes of a tile are merged when the
// tile-steps are decided, so no plane is read twice.
template <typename T, int D, int XT>
__global__ void __launch_bounds__(kStatsWarps * 32, 2)
    plane_stats_kernel(RegularMesh mesh, FieldAccess fa, ExtractConfig cfg) {
  constexpr int M = D - 1;
  constexpr int TX = Tile<D>::TX, TY = Tile<D>::TY;
  constexpr int NG = XT + 1;
  static_assert(TX == 32, "a 32-vertex group is one x-tile");
  const int lane = threadIdx.x & 31;
  const int nxc = (cfg.tiles[0] + XT - 1) / XT;
  const int ldz = (D == 4) ? (int)mesh.ld[2] : 1;
  const int lt = (int)mesh.ld[D - 1];
  long long task = (long long)blockIdx.x * kStatsWarps + (threadIdx.x >> 5);
  const int xc = (int)(task % nxc);
  task /= nxc;
  const int yt = (int)(task % cfg.tiles[1]);
  task /= cfg.tiles[1];
  const int z = (int)(task % ldz);
  const int s = (int)(task / ldz);
  if (s >= lt) return;  // whole warp
  const int xt0 = xc * XT;
  const int x0 = xt0 * TX, y0 = yt * TY;
  const int nvy = min(TY + 1, (int)mesh.ld[1] - y0);
  const int nx = min(XT * TX + 1, (int)mesh.ld[0] - x0);  // chunk vertices, halo included
  const long long at = ((long long)s + mesh.off[D - 1] - fa.shift[D - 1]) ^ fa.tflip;
  long long obase = at * fa.estride[D - 1] + (x0 + mesh.off[0] - fa.shift[0]) * fa.estride[0];
  if (D == 4) obase += (z + mesh.off[2] - fa.shift[2]) * fa.estride[2];
  int kmn[NG][M], kmx[NG][M];
#pragma unroll
  for (int g = 0; g < NG; ++g)
#pragma unroll
    for (int r = 0; r < M; ++r) {
      kmn[g][r] = 0x7FFFFFFF;
      kmx[g][r] = (int)0x80000000;
    }
  for (int vy = 0; vy < nvy; ++vy) {
    const long long orow = obase + (y0 + vy + mesh.off[1] - fa.shift[1]) * fa.estride[1];
    T v[NG][M];
#pragma unroll
    for (int g = 0; g < NG; ++g)
#pragma unroll
      for (int r = 0; r < M; ++r) {
        const int x = 32 * g + lane;
        v[g][r] = (x < nx) ? __ldcs(static_cast<const T*>(fa.comp[r]) + orow + x * fa.estride[0]) : T(0);
      }
#pragma unroll
    for (int g = 0; g < NG; ++g)
#pragma unroll
      for (int r = 0; r < M; ++r)
        if (32 * g + lane < nx) {
          const int key = ord_key(hi_word<T>(v[g][r]));
          kmn[g][r] = min(kmn[g][r], key);
          kmx[g][r] = max(kmx[g][r], key);
        }
  }
  const size_t row_entry = (((size_t)s * ldz + z) * cfg.tiles[1] + yt) * cfg.tiles[0];
#pragma unroll
  for (int t = 0; t < XT; ++t) {
    if (xt0 + t >= cfg.tiles[0]) break;  // whole warp
    int rmn[M], rmx[M];
#pragma unroll
    for (int c = 0; c < M; ++c) {
      rmn[c] = kmn[t][c];
      rmx[c] = kmx[t][c];
      if (lane == 0) {  // the halo vertex: lane 0 of group t + 1
        rmn[c] = min(rmn[c], kmn[t + 1][c]);
        rmx[c] = max(rmx[c], kmx[t + 1][c]);
      }
      rmn[c] = __reduce_min_sync(0xFFFFFFFFu, rmn[c]);
      rmx[c] = __reduce_max_sync(0xFFFFFFFFu, rmx[c]);
    }
    if (lane == 0) {
      int4 lo, hi;
      lo.x = rmn[0];
      lo.y = M > 1 ? rmn[M > 1 ? 1 : 0] : 0x7FFFFFFF;
      lo.z = M > 2 ? rmn[M > 2 ? 2 : 0] : 0x7FFFFFFF;
      lo.w = rmx[0];
      hi.x = M > 1 ? rmx[M > 1 ? 1 : 0] : (int)0x80000000;
      hi.y = M > 2 ? rmx[M > 2 ? 2 : 0] : (int)0x80000000;
      hi.z = 0;
      hi.w = 0;
      int4* dst = reinterpret_cast<int4*>(cfg.tstats + 8 * (row_entry + xt0 + t));
      dst[0] = lo;
      dst[1] = hi;
    }
  }
}

// high 32-bit word of element u of a 16-byte vector (little-endian)
template <typename T>
__device__ __forceinline__ unsigned vec_hi_word(const uint4& w, int u) {
  if (sizeof(T) == 8) return u == 0 ? w.y : w.w;
  return u == 0 ? w.x : u == 1 ? w.y : u == 2 ? w.z : w.w;
}
// The same statistics for interleaved components whose rows start on 16-byte
// boundaries, streamed: persistent warps walk the tasks (warp w takes tasks
// w, w + W, ... for W warps in the grid) as one continuous sequence of rows,
// and every thread keeps S - 1 rows of its own 16-byte copies in flight
// through a private S-stage ring in shared memory, across task boundaries.
//   Lane l serves tile t = l / LPT of the chunk (LPT = 32 / XT lanes per
//   tile) as its q = l % LPT-th part: its vector j covers tile elements
//   LPT V j + V q .. + V - 1 (V elements per 16 bytes), so every copy
//   instruction of the warp reads XT runs of LPT V consecutive elements.  The
//   component of element e is e mod M = (a + V q) mod M with a = (LPT V j + u)
//   mod M known at compile time: each lane keeps one accumulator per slot a
//   and rotates them by V q when the task ends.  Lane q = LPT - 1 also copies
//   the tile's halo vertex (the next tile's first).
template <typename T, int D, int XT, int S>
struct StatsStream {
  static constexpr int M = D - 1;
  static constexpr int V = 16 / (int)sizeof(T);
  static constexpr int LPT = 32 / XT;
  static constexpr int NV = 32 * M / (LPT * V);
  static constexpr int THREADS = kStatsWarps * 32;
  static constexpr int HALO = S * THREADS * NV;              // uint4 offset of the halo slots
  static constexpr int SMEM = 16 * (HALO + S * kStatsWarps * XT);
  static_assert(NV * LPT * V == 32 * M, "a tile row splits evenly over its lanes");
};

template <typename T, int D, int XT, int S>
__global__ void __launch_bounds__(kStatsWarps * 32, 2)
    plane_stats_stream_kernel(RegularMesh mesh, FieldAccess fa, ExtractConfig cfg, int ntasks) {
  using SS = StatsStream<T, D, XT, S>;
  constexpr int M = SS::M, V = SS::V, LPT = SS::LPT, NV = SS::NV;
  constexpr int TX = Tile<D>::TX, TY = Tile<D>::TY;
  extern __shared__ __align__(128) unsigned char smem[];
  uint4* const ring = reinterpret_cast<uint4*>(smem);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t = lane / LPT, q = lane % LPT;
  const int tb = 32 * M * t;  // the lane's tile, first element of the chunk row
  const int nxc = (cfg.tiles[0] + XT - 1) / XT;
  const int ldz = (D == 4) ? (int)mesh.ld[2] : 1;
  const int nw = (int)gridDim.x * kStatsWarps;

  struct Task {
    int task, vy, nvy, ne, y0, xt0, yt, z, s;
    const T* base;
  };
  auto decode = [&](int task, Task& g) {
    g.task = task;
    g.vy = 0;
    if (task >= ntasks) return;
    int r = task;
    const int xc = r % nxc;
    r /= nxc;
    g.yt = r % cfg.tiles[1];
    r /= cfg.tiles[1];
    g.z = r % ldz;
    g.s = r / ldz;
    g.xt0 = xc * XT;
    const int x0 = g.xt0 * TX;
    g.y0 = g.yt * TY;
    g.nvy = min(TY + 1, (int)mesh.ld[1] - g.y0);
    g.ne = min(XT * TX + 1, (int)mesh.ld[0] - x0) * M;
    const long long at = ((long long)g.s + mesh.off[D - 1] - fa.shift[D - 1]) ^ fa.tflip;
    long long o = at * fa.estride[D - 1] + (x0 + mesh.off[0] - fa.shift[0]) * fa.estride[0] +
                  (long long)(g.y0 + mesh.off[1] - fa.shift[1]) * fa.estride[1];
    if (D == 4) o += (g.z + mesh.off[2] - fa.shift[2]) * fa.estride[2];
    g.base = static_cast<const T*>(fa.comp[0]) + o;
  };
  auto vslot = [&](int stage, int j) { return ring + (stage * NV + j) * SS::THREADS + tid; };
  auto hslot = [&](int stage) { return ring + SS::HALO + (stage * kStatsWarps + warp) * XT + t; };

  Task gi, gc;  // the issuing and the consuming side of the row sequence
  decode(blockIdx.x * kStatsWarps + warp, gi);
  gc = gi;
  auto issue = [&](int stage) {
    if (gi.task < ntasks) {
      const T* row = gi.base + (long long)gi.vy * fa.estride[1];
#pragma unroll
      for (int j = 0; j < NV; ++j) {
        const int e = tb + LPT * V * j + V * q;
        if (e + V <= gi.ne) {
          cp_async_16(vslot(stage, j), row + e);
        } else {
#pragma unroll
          for (int u = 0; u < V; ++u)
            if (e + u < gi.ne) cp_async_small<sizeof(T)>(reinterpret_cast<T*>(vslot(stage, j)) + u, row + e + u);
        }
      }
      if (q == LPT - 1) {
#pragma unroll
        for (int u = 0; u < M; ++u)
          if (tb + 32 * M + u < gi.ne)
            cp_async_small<sizeof(T)>(reinterpret_cast<T*>(hslot(stage)) + u, row + tb + 32 * M + u);
      }
      if (++gi.vy == gi.nvy) decode(gi.task + nw, gi);
    }
    cp_async_commit();  // empty groups keep the count uniform
  };

  // two accumulator sets, by the parity of the vector index, halve the
  // dependent min / max chains of a row
  int kmn[2][M], kmx[2][M], hmn[M], hmx[M];
  auto reset = [&]() {
#pragma unroll
    for (int a = 0; a < M; ++a) {
      kmn[0][a] = kmn[1][a] = hmn[a] = 0x7FFFFFFF;
      kmx[0][a] = kmx[1][a] = hmx[a] = (int)0x80000000;
    }
  };
  reset();
#pragma unroll
  for (int p = 0; p < S - 1; ++p) issue(p);
  int stage = 0;
  while (gc.task < ntasks) {
    issue(stage == 0 ? S - 1 : stage - 1);  // the slot consumed one row ago
    cp_async_wait<S - 1>();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      const uint4 w = *vslot(stage, j);
      const int e0 = tb + LPT * V * j + V * q;
      const bool full = e0 + V <= gc.ne;  // the whole vector lies in the row
#pragma unroll
      for (int u = 0; u < V; ++u) {
        const int a = (LPT * V * j + u) % M;
        if (full || e0 + u < gc.ne) {
          const int key = ord_key(vec_hi_word<T>(w, u));
          kmn[j & 1][a] = min(kmn[j & 1][a], key);
          kmx[j & 1][a] = max(kmx[j & 1][a], key);
        }
      }
    }
    if (q == LPT - 1) {
      const uint4 w = *hslot(stage);
#pragma unroll
      for (int u = 0; u < M; ++u)
        if (tb + 32 * M + u < gc.ne) {
          const int key = ord_key(vec_hi_word<T>(w, u));
          hmn[u] = min(hmn[u], key);
          hmx[u] = max(hmx[u], key);
        }
    }
    stage = (stage + 1 == S) ? 0 : stage + 1;
    if (++gc.vy < gc.nvy) continue;
    // task complete: slot a holds component (a + V q) mod M
    int rmn[M], rmx[M];
    const int rot = (V * q) % M;
#pragma unroll
    for (int c = 0; c < M; ++c) {
      rmn[c] = hmn[c];
      rmx[c] = hmx[c];
#pragma unroll
      for (int a = 0; a < M; ++a)
        if ((a + rot) % M == c) {
          rmn[c] = min(rmn[c], min(kmn[0][a], kmn[1][a]));
          rmx[c] = max(rmx[c], max(kmx[0][a], kmx[1][a]));
        }
#pragma unroll
      for (int o = 1; o < LPT; o <<= 1) {
        rmn[c] = min(rmn[c], __shfl_xor_sync(0xFFFFFFFFu, rmn[c], o));
        rmx[c] = max(rmx[c], __shfl_xor_sync(0xFFFFFFFFu, rmx[c], o));
      }
    }
    if (q == 0 && gc.xt0 + t < cfg.tiles[0]) {
      int4 lo, hi;
      lo.x = rmn[0];
      lo.y = M > 1 ? rmn[M > 1 ? 1 : 0] : 0x7FFFFFFF;
      lo.z = M > 2 ? rmn[M > 2 ? 2 : 0] : 0x7FFFFFFF;
      lo.w = rmx[0];
      hi.x = M > 1 ? rmx[M > 1 ? 1 : 0] : (int)0x80000000;
      hi.y = M > 2 ? rmx[M > 2 ? 2 : 0] : (int)0x80000000;
      hi.z = 0;
      hi.w = 0;
      const size_t entry = (((size_t)gc.s * ldz + gc.z) * cfg.tiles[1] + gc.yt) * cfg.tiles[0] + gc.xt0 + t;
      int4* dst = reinterpret_cast<int4*>(cfg.tstats + 8 * entry);
      dst[0] = lo;
      dst[1] = hi;
    }
    reset();
    decode(gc.task + nw, gc);
  }
  cp_async_wait<0>();
}

// largest high-word magnitude of a set of values, from the order keys of its
// per-component extremes (|v| <= max(|min|, |max|)); a NaN or infinity, whose
// key lies beyond every finite one, gives a magnitude >= the exponent mask
__device__ __forceinline__ unsigned key_mag(int k) {
  return k >= 0 ? (unsigned)k : (~(unsigned)k & 0x7FFFFFFFu);
}

// whether the tile-step between slices c and c+1 (c+1 absent for the last
// corner slice) can hold no accepted simplex
template <typename T, int M>
__device__ __forceinline__ bool tile_step_culled(const int* st_c, const int* st_s) {
  using P = CullParams<T>;
  constexpr int kKappaTile = P::kappa_exp + 3 * P::band;  // kappa = 2^-kKappaTile
  unsigned am = (unsigned)st_c[6];
  int kmn[3] = {st_c[0], st_c[1], st_c[2]}, kmx[3] = {st_c[3], st_c[4], st_c[5]};
  if (st_s) {
    am = max(am, (unsigned)st_s[6]);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      kmn[j] = min(kmn[j], st_s[j]);
      kmx[j] = max(kmx[j], st_s[3 + j]);
    }
  }
  if (am >= P::expmask) return false;  // an infinite or NaN value: never dropped
  if (am < P::tiny_hi) return true;
  const unsigned mup = am + 1u;  // upper bound of M in high-word space
  const unsigned kexp = (unsigned)kKappaTile << P::mant;
  if ((mup & P::expmask) <= kexp) return false;
  const unsigned thr = mup - kexp;  // kappa * M_up, exact
  const int kpos = (int)thr, kneg = ord_key(thr | 0x80000000u);
  bool culled = false;
#pragma unroll
  for (int j = 0; j < M; ++j) culled |= (kmn[j] > kpos) || (kmx[j] < kneg);
  return culled;
}

// The statistics of one tile over slice c: the plane entries of its z
// planes z0 .. z0 + TZ (clipped to the mesh) merged, and the magnitude bound
// in word 6.
template <int D>
__device__ __forceinline__ void tile_slice_stats(const RegularMesh& mesh, const ExtractConfig& cfg, int xt, int yt,
                                                 int zt, int c, int out[8]) {
  constexpr int TZ = Tile<D>::TZ;
  const int ldz = (D == 4) ? (int)mesh.ld[2] : 1;
  const int z0 = (D == 4) ? zt * TZ : 0;
  const int nz = (D == 4) ? min(TZ + 1, ldz - z0) : 1;
  int4 a[TZ + 1], b[TZ + 1];
#pragma unroll
  for (int k = 0; k <= TZ; ++k)
    if (k < nz) {
      const int4* e = reinterpret_cast<const int4*>(
          cfg.tstats + 8 * ((((size_t)c * ldz + z0 + k) * cfg.tiles[1] + yt) * cfg.tiles[0] + xt));
      a[k] = e[0];
      b[k] = e[1];
    }
  int4 p = a[0], q = b[0];
#pragma unroll
  for (int k = 1; k <= TZ; ++k)
    if (k < nz) {
      p.x = min(p.x, a[k].x);
      p.y = min(p.y, a[k].y);
      p.z = min(p.z, a[k].z);
      p.w = max(p.w, a[k].w);
      q.x = max(q.x, b[k].x);
      q.y = max(q.y, b[k].y);
    }
  out[0] = p.x;
  out[1] = p.y;
  out[2] = p.z;
  out[3] = p.w;
  out[4] = q.x;
  out[5] = q.y;
  unsigned am = 0;
#pragma unroll
  for (int j = 0; j < D - 1; ++j) am = max(am, max(key_mag(out[j]), key_mag(out[3 + j])));
  out[6] = (int)am;
  out[7] = 0;
}

template <typename T, int D>
__global__ void tile_runs_kernel(RegularMesh mesh, ExtractConfig cfg) {
  constexpr int M = D - 1;
  const int ntiles = cfg.tiles[0] * cfg.tiles[1] * cfg.tiles[2];
  const int lt = (int)mesh.ld[D - 1];
  for (int tile = blockIdx.x * blockDim.x + threadIdx.x; tile < ntiles; tile += gridDim.x * blockDim.x) {
    const int xt = tile % cfg.tiles[0], yt = (tile / cfg.tiles[0]) % cfg.tiles[1];
    const int zt = tile / (cfg.tiles[0] * cfg.tiles[1]);
    int sc[8], ss[8];
    tile_slice_stats<D>(mesh, cfg, xt, yt, zt, 0, ss);
    int start = -1;
    for (int c = 0; c <= lt; ++c) {
      bool keep = false;
      if (c < lt) {
#pragma unroll
        for (int f = 0; f < 8; ++f) sc[f] = ss[f];
        if (c + 1 < lt) tile_slice_stats<D>(mesh, cfg, xt, yt, zt, c + 1, ss);
        keep = !tile_step_culled<T, M>(sc, c + 1 < lt ? ss : nullptr);
      }
      if (keep && start < 0) start = c;
      if (!keep && start >= 0) {
        const unsigned r = atomicAdd(cfg.n_runs, 1u);
        if (r < cfg.runs_cap) {
          uint4 run;
          run.x = (unsigned)tile;
          run.y = (unsigned)start;
          run.z = (unsigned)c;
          run.w = 0;
          reinterpret_cast<uint4*>(cfg.runs)[r] = run;
        }
        start = -1;
      }
    }
  }
}

template <typename T, int D, bool MULTI, bool TMA>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 2 : 1)
    run_cull_kernel(const __grid_constant__ CUtensorMap map0, const __grid_constant__ CUtensorMap map1,
                    const __grid_constant__ CUtensorMap map2, RegularMesh mesh, FieldAccess fa, ExtractConfig cfg,
                    CandidateQueue cq, unsigned* err) {
  using G = Geo<T, D, MULTI>;
  using G2 = Geo2<T, D, MULTI>;
  constexpr int M = D - 1;
  constexpr int TX = G::TX, TY = G::TY, TZ = G::TZ;
  constexpr int VX = G::VX, VY = G::VY, VZ = G::VZ, VS = G::VS, VPT = G::VPT, VSP = G::VSP;
  constexpr int TBIT = 1 << (D - 1);
  constexpr int HW = sizeof(T) / 4;
  static_assert(D == 3 ? kWarps * kRows >= TY : kWarps == TY * (TZ / kRows),
                "every corner row of the tile belongs to exactly one warp");

  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned long long bar[kNbuf];
  __shared__ unsigned band_tbl[kBandTable];
  unsigned* const W0 = reinterpret_cast<unsigned*>(smem + G2::WORDS);
  auto wslot = [&](int w) { return W0 + w * VSP; };

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int ldx = (int)mesh.ld[0], ldy = (int)mesh.ld[1], ldz = (D == 4) ? (int)mesh.ld[2] : 1;
  const int lt = (int)mesh.ld[D - 1];
  const int n_items = (int)min(*cfg.n_runs, cfg.runs_cap);
  const uint4* runs = reinterpret_cast<const uint4*>(cfg.runs);
  int aoff[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) aoff[k] = (k < D) ? (int)(mesh.off[k] - fa.shift[k]) : 0;
  auto tcoord = [&](int s) { return (s + aoff[D - 1]) ^ fa.tflip; };
  auto item_geom = [&](int item, int& x0, int& y0, int& z0, int& t0, int& t1, int& s_end) {
    const uint4 run = runs[item];
    int tix = (int)run.x;
    x0 = (tix % cfg.tiles[0]) * TX;
    tix /= cfg.tiles[0];
    y0 = (tix % cfg.tiles[1]) * TY;
    tix /= cfg.tiles[1];
    z0 = (D == 4) ? tix * TZ : 0;
    t0 = (int)run.y;
    t1 = (int)run.z;
    s_end = min(t1, lt - 1);
  };
  fill_band_table<T>(band_tbl, tid, kThreads);

  // ---- producer (thread 0): the CTA's slice stream over its runs
  int p_item = blockIdx.x, p_s = 0, p_send = -1, px0 = 0, py0 = 0, pz0 = 0;
  int pq = 0;  // stream index of the next slice to issue
  auto p_begin = [&]() {
    if (p_item < n_items) {
      int t0, t1;
      item_geom(p_item, px0, py0, pz0, t0, t1, p_send);
      p_s = t0;
    }
  };
  auto issue_next = [&]() {
    const int buf = pq % kNbuf;
    unsigned char* dst0 = smem + buf * G::BYTES;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar[buf], G::TX_BYTES);
    const int cx = (px0 + aoff[0]) * (MULTI ? M : 1);
    const int cy = py0 + aoff[1];
    if constexpr (MULTI) {
      if constexpr (D == 4) tma_load_4d(dst0, &map0, cx, cy, pz0 + aoff[2], tcoord(p_s), &bar[buf]);
      else tma_load_3d(dst0, &map0, cx, cy, tcoord(p_s), &bar[buf]);
    } else {
      const CUtensorMap* maps[3] = {&map0, &map1, &map2};
#pragma unroll
      for (int j = 0; j < M; ++j) {
        if constexpr (D == 4)
          tma_load_4d(dst0 + j * G::COMP, maps[j], cx, cy, pz0 + aoff[2], tcoord(p_s), &bar[buf]);
        else
          tma_load_3d(dst0 + j * G::COMP, maps[j], cx, cy, tcoord(p_s), &bar[buf]);
      }
    }
    ++pq;
    if (++p_s > p_send) {
      p_item += gridDim.x;
      p_begin();
    }
  };
  auto produce_until = [&](int qmax) {
    while (pq <= qmax && p_item < n_items) issue_next();
  };

  int x0 = 0, y0 = 0, z0 = 0, t0 = 0, t1 = 0, s_end = 0;
  int voff[VPT];
#pragma unroll
  for (int u = 0; u < VPT; ++u) voff[u] = 0;
  unsigned vvalid = 0, row_valid = 0;
  const int cyw = (D == 4) ? warp % TY : warp * kRows;
  const int czw = (D == 4) ? (warp / TY) * kRows : 0;
  auto load_plain = [&](int s, int buf) {
    T* dst = reinterpret_cast<T*>(smem + buf * G::BYTES);
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
  };
  int cq_idx = 0;  // stream index of slice t0 of the current run
  auto arrive = [&](int s) -> bool {
    const int q = cq_idx + (s - t0);
    if constexpr (TMA) return mbar_wait(&bar[q % kNbuf], (unsigned)((q / kNbuf) & 1));
    load_plain(s, q % kNbuf);
    __syncthreads();
    return true;
  };
  auto words = [&](int s, unsigned* dst) {
    const unsigned* r =
        reinterpret_cast<const unsigned*>(smem + ((cq_idx + (s - t0)) % kNbuf) * G::BYTES) + (HW - 1);
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      unsigned h[M];
#pragma unroll
      for (int j = 0; j < M; ++j) h[j] = r[HW * (MULTI ? voff[u] + j : voff[u] + j * G::COMP_ELEMS)];
      const unsigned w = vertex_word_hi<T, M>(h, band_tbl);
      dst[tid + u * kThreads] = ((vvalid >> u) & 1u) ? w : kAbsent;
    }
  };

  if (TMA && tid == 0)
    for (int b = 0; b < kNbuf; ++b) mbar_init(&bar[b], 1);
  if (TMA && tid == 0) asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  for (int i = tid; i < VSP; i += kThreads) wslot(kNbuf)[i] = kAbsent;
  __syncthreads();
  if (TMA && tid == 0) {
    p_begin();
    produce_until(kNbuf - 1);
  }
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    item_geom(item, x0, y0, z0, t0, t1, s_end);
    vvalid = 0;
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      const int i = tid + u * kThreads;
      const int vx = i % VX, vy = (i / VX) % VY, vz = i / (VX * VY);
      const bool in = i < VS && x0 + vx < ldx && y0 + vy < ldy && (D == 3 || z0 + vz < ldz);
      voff[u] = in ? (MULTI ? ((vz * VY + vy) * G::VXBOX + vx) * M : (vz * VY + vy) * G::VXBOX + vx) : 0;
      vvalid |= (in ? 1u : 0u) << u;
    }
    row_valid = 0;
#pragma unroll
    for (int q = 0; q < kRows; ++q) {
      const int cy = (D == 4) ? cyw : cyw + q;
      const int cz = (D == 4) ? czw + q : 0;
      if (x0 + lane < ldx && cy < TY && y0 + cy < ldy && (D == 3 || z0 + cz < ldz)) row_valid |= 1u << q;
    }
    for (int c = t0; c < t1; ++c) {
      const int s = c + 1;
      const bool has_s = s <= s_end;
      bool ok = true;
      // words of stream slice q live in slot q % kNbuf: the slots written
      // here were last read two or more steps ago, before the previous
      // step's barrier
      const int q_c = cq_idx + (c - t0);
      if (c == t0) {
        ok = arrive(c);
        if (ok) words(c, wslot(q_c % kNbuf));
      }
      if (ok && has_s) {
        ok = arrive(s);
        if (ok) words(s, wslot((q_c + 1) % kNbuf));
      }
      // the one barrier of the step: words of both slices visible, every
      // read of the raw buffer that the next issued slice reuses done
      if (__syncthreads_or(!ok)) {
        if (TMA && tid == 0)
          for (int q = cq_idx + (c - t0); q < pq; ++q) mbar_wait(&bar[q % kNbuf], (unsigned)((q / kNbuf) & 1));
        if (tid == 0) atomicOr(err, 2u);
        return;
      }
      if (TMA && tid == 0) produce_until(q_c + kNbuf - 1);
      if (D == 3 && cyw >= TY) continue;  // warp-uniform: no corner rows of the tile
      const unsigned* A = wslot(q_c % kNbuf);
      const unsigned* B = has_s ? wslot((q_c + 1) % kNbuf) : wslot(kNbuf);
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
          unsigned basei = 0;
          if (lane == 0) basei = atomicAdd(cq.count, (unsigned)__popc(ball));
          basei = __shfl_sync(0xFFFFFFFFu, basei, 0);
          if (keep) {
            const unsigned idx = basei + __popc(ball & ((1u << lane) - 1));
            if (idx < cq.cap) {
              const int l0 = x0 + lane, l1 = y0 + cy, l2 = (D == 4) ? z0 + cz : c;
              int vmask = 0;
              if (l0 + 1 < ldx) vmask |= 1;
              if (l1 + 1 < ldy) vmask |= 2;
              if (D == 4 && l2 + 1 < ldz) vmask |= 4;
              if (c + 1 < lt) vmask |= TBIT;
              unsigned long long ch = c_chains_by_vmask[D - 3][vmask];
              if (cfg.skip_first_spatial && c == 0) ch &= c_time_chains[D - 3];
              cq.corner[idx] = pack_corner(l0, l1, (D == 4) ? l2 : 0, c);
              if (cq.field) cq.field[idx] = cq.field_id;
              cq.chains[idx] = ch;
            }
          }
        }
      }
    }
    cq_idx += s_end - t0 + 1;
  }
}

// Stage 2: exact SoS test and bit-exact solve of the queued chains.  One warp
// per candidate hypercube: its 2^D vertices' values are gathered once into
// shared memory, then each lane tests one chain; accepted simplices are
// compacted by warp ballot.
constexpr int kRefineWarps = 8;

// One candidate hypercube (packed local corner pc, chains to test) of a
// regular mesh, by one warp; cube is the warp's 2^D * M staging slots.
// Accepted simplices get key key_base + corner vertex id * chains + rank.
template <typename T, int D>
__device__ __forceinline__ void refine_candidate(const RegularMesh& mesh, const FieldAccess& fa,
                                                 const ExtractConfig& cfg, unsigned long long pc,
                                                 unsigned long long chains, const FeatureSink& sink,
                                                 unsigned long long key_base, T* cube, const unsigned* band_tbl,
                                                 int lane) {
  constexpr int M = D - 1;
  constexpr int NV = 1 << D;
  const ChainTable& CT = c_chains[D - 3];
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
    T val = in ? field_at<T>(fa, j, g, D, vid) : T(0);
    if (cfg.fiber) val = fp<T>::sub(val, (T)(j ? cfg.fthr[1] : cfg.fthr[0]));  // values[i][j] - thresholds[j]
    cube[v * M + j] = val;
  }
  __syncwarp();
  // cull words of the hypercube's vertices (absent outside the mesh)
  unsigned vw = kAbsent;
  if (lane < NV) {
    unsigned h[M];
#pragma unroll
    for (int j = 0; j < M; ++j) h[j] = hi_word<T>(cube[lane * M + j]);
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
      live = live && (cfg.fiber || !word_culled(wacc));
    }
    if (live) {
      T vals[M + 1][M];
#pragma unroll
      for (int i = 0; i <= M; ++i)
#pragma unroll
        for (int j = 0; j < M; ++j) vals[i][j] = cube[mk[i] * M + j];
      bool inside;
      if constexpr (M == 2) inside = sos_inside2<T>(vals, cfg.Q);
      else inside = sos_inside3<T>(vals, cfg.Q);
      if (inside) {
        T lam[M + 1];
        bool solved = solve_exact<M, T>(vals, lam);
        if (!solved && cfg.fiber) {
          // FiberPredicate keeps the simplex at the centroid: (T)1.0 / 3.0
#pragma unroll
          for (int i = 0; i <= M; ++i) lam[i] = (T)((double)(T)1.0 / 3.0);
          solved = true;
        }
        if (solved) {
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
          sink.key[idx] = key_base + vid0 * (unsigned long long)CT.n + (unsigned long long)ch;
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

template <typename T, int D>
__global__ void __launch_bounds__(kRefineWarps * 32, 2)
    refine_regular_kernel(RegularMesh mesh, FieldAccess fa, ExtractConfig cfg, CandidateQueue cq,
                          FeatureSink sink) {
  constexpr int M = D - 1;
  constexpr int NV = 1 << D;
  __shared__ T cube[kRefineWarps][NV * M];
  __shared__ unsigned band_tbl[kBandTable];
  fill_band_table<T>(band_tbl, threadIdx.x, blockDim.x);
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const unsigned n = min(*cq.count, cq.cap);
  const unsigned gw = blockIdx.x * kRefineWarps + wib;
  const unsigned nw = gridDim.x * kRefineWarps;
  for (unsigned c = gw; c < n; c += nw)
    refine_candidate<T, D>(mesh, fa, cfg, cq.corner[c], cq.chains[c], sink, 0ull, cube[wib], band_tbl, lane);
}

// ---------------------------------------------------------------------------
// The exact test of the surviving hypercubes.
//   single field, two launches:
//     refine_test_kernel    32 candidates per block: one thread per vertex
//                           gathers values, quantises them for the inside
//                           tests and computes the cull words; the chains
//                           that survive them are laid out as (candidate,
//                           chain) pairs by a prefix count in shared memory
//                           and each pair gets one thread for the fast-path
//                           inside test; the accepted ones go to a list
//     refine_accept_kernel  the solve of every listed simplex (one thread
//                           each, values read from the field), and the whole
//                           test with the 128-bit path for candidates holding
//                           a quantised value past 2^31
//   batches, three launches: batch_test_kernel (refine_test_kernel with 16
//   lanes per candidate and each candidate's field record), the solve, and
//   the 128-bit path, the last two reading values from the fields
// The only atomics are the lists' and the sink's.

// Masks of vertices 1..M of chain ch, a byte each (m1 | m2 << 8 | m3 << 16);
// 0 past the table.
template <int D>
__device__ __forceinline__ unsigned chain_packed(int ch) {
  return g_chain_pk[D - 3][ch];
}

constexpr int kStageVals = 48;  // 2^D * M values per candidate, D <= 4

// The fast-path inside test of listed simplex (candidate, chain ch) from the
// candidate's quantised values qsrc; chain_pk: chain_packed of every chain of
// the mesh's dimension.
template <int D>
__device__ __forceinline__ bool inside_pair_q(int ch, const int* qsrc, const unsigned* chain_pk) {
  constexpr int M = D - 1;
  int mk[M + 1];
  mk[0] = 0;
  const unsigned pk = chain_pk[ch];
#pragma unroll
  for (int k = 0; k < M; ++k) mk[k + 1] = (pk >> (8 * k)) & 0xFF;
  int q[M + 1][M];
#pragma unroll
  for (int k = 0; k <= M; ++k)
#pragma unroll
    for (int j = 0; j < M; ++j) q[k][j] = qsrc[mk[k] * M + j];
  if constexpr (M == 2) return sos_inside2_q(q);
  else return sos_inside3_q(q);
}

// Listed simplex (candidate, chain ch) by one thread: BIG = true, the whole
// exact test (inside test from the field values, 128-bit quantisation);
// BIG = false, a simplex the fast-path inside test accepted.  Then the solve
// and, when accepted, its canonical key and reported values.  src: the
// candidate's staged values, or null to read the simplex's values from the
// field.
template <typename T, int D, bool BIG>
__device__ __forceinline__ bool test_pair(const RegularMesh& mesh, const FieldAccess& fa, const ExtractConfig& cfg,
                                          unsigned long long pc, int ch, const T* src, const unsigned* chain_pk,
                                          unsigned long long key_base, unsigned long long& key, double lam_out[4],
                                          float bary_out[4], float& sc_out) {
  constexpr int M = D - 1;
  const ChainTable& CT = c_chains[D - 3];
  int mk[M + 1];
  mk[0] = 0;
  const unsigned pk = chain_pk[ch];
#pragma unroll
  for (int k = 0; k < M; ++k) mk[k + 1] = (pk >> (8 * k)) & 0xFF;
  const long long l[4] = {(long long)(pc & 0xFFFF), (long long)((pc >> 16) & 0xFFFF),
                          (long long)((pc >> 32) & 0xFFFF), (long long)(pc >> 48)};
  long long g0[4];
  unsigned long long vid0 = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const long long lk = (D == 4) ? l[k] : (k < 2 ? l[k] : (k == 2 ? l[3] : 0));
    g0[k] = (k < D) ? lk + mesh.off[k] : 0;
    if (k < D) vid0 += (unsigned long long)g0[k] * mesh.gstride[k];
  }
  T vals[M + 1][M];
  if (src) {
#pragma unroll
    for (int k = 0; k <= M; ++k)
#pragma unroll
      for (int j = 0; j < M; ++j) vals[k][j] = src[mk[k] * M + j];
  } else {
    // a chain that survives lies inside the mesh
#pragma unroll
    for (int k = 0; k <= M; ++k) {
      long long gv[4];
      unsigned long long vid = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        gv[q] = (q < D) ? g0[q] + ((mk[k] >> q) & 1) : 0;
        if (q < D) vid += (unsigned long long)gv[q] * mesh.gstride[q];
      }
#pragma unroll
      for (int j = 0; j < M; ++j) {
        T x = field_at<T>(fa, j, gv, D, vid);
        if (cfg.fiber) x = fp<T>::sub(x, (T)(j ? cfg.fthr[1] : cfg.fthr[0]));  // values[i][j] - thresholds[j]
        vals[k][j] = x;
      }
    }
  }
  if constexpr (BIG) {
    bool inside;
    if constexpr (M == 2) inside = sos_inside2<T>(vals, cfg.Q);
    else inside = sos_inside3<T>(vals, cfg.Q);
    if (!inside) return false;
  }
  T lam[M + 1];
  bool solved = solve_exact<M, T>(vals, lam);
  if (!solved && cfg.fiber) {
    // FiberPredicate keeps the simplex at the centroid: (T)1.0 / 3.0
#pragma unroll
    for (int k = 0; k <= M; ++k) lam[k] = (T)((double)(T)1.0 / 3.0);
    solved = true;
  }
  if (!solved) return false;
  key = key_base + vid0 * (unsigned long long)CT.n + (unsigned long long)ch;
#pragma unroll
  for (int k = 0; k <= M; ++k) {
    lam_out[k] = (double)lam[k];
    bary_out[k] = (float)lam[k];
  }
  if (fa.has_scalar) {
    using F = fp<T>;
    T sc = T(0);
#pragma unroll
    for (int k = 0; k <= M; ++k) {
      long long gv[4];
      unsigned long long vid = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        gv[q] = (q < D) ? g0[q] + ((mk[k] >> q) & 1) : 0;
        if (q < D) vid += (unsigned long long)gv[q] * mesh.gstride[q];
      }
      sc = F::add(sc, F::mul(lam[k], scalar_at<T>(fa, gv, D, vid)));
    }
    sc_out = (float)sc;
  }
  if (cfg.refined) {
    double rr[M + 1];
    if (solve_refined<M, T>(vals, rr))
#pragma unroll
      for (int k = 0; k <= M; ++k) lam_out[k] = rr[k];
  }
  return true;
}

// warp-ballot compaction of the accepted simplices of one pass into the sink
__device__ __forceinline__ void sink_write(const FeatureSink& sink, bool acc, unsigned long long key,
                                           const double lam_out[4], const float bary_out[4], float sc_out, int lane) {
  const unsigned ball = __ballot_sync(0xFFFFFFFFu, acc);
  if (!ball) return;
  unsigned b0 = 0;
  const int leader = __ffs(ball) - 1;
  if (lane == leader) b0 = atomicAdd(sink.count, (unsigned)__popc(ball));
  b0 = __shfl_sync(0xFFFFFFFFu, b0, leader);
  if (!acc) return;
  const unsigned idx = b0 + __popc(ball & ((1u << lane) - 1u));
  if (idx < sink.cap) {
    sink.key[idx] = key;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      sink.lam[4 * (size_t)idx + k] = lam_out[k];
      sink.bary4[4 * (size_t)idx + k] = bary_out[k];
    }
    sink.scalar[idx] = sc_out;
  }
}

constexpr int kPairCands = 64;  // candidates a block of the exact-test launch takes at a time
// candidates a block of the single-field test takes at a time: small groups
// balance the launch's few blocks across the SMs
constexpr int kTestCands = 32;

// The block's next kPairCands entries of `live` from `first` laid out as a
// list of (slot, chain) pairs in shared memory (slot << 6 | chain), by a
// prefix count of the masks' set bits; returns the number of simplices.
// Shared: msk[kPairCands], off[kPairCands + 1], plist[kPairCands * 64].
__device__ __forceinline__ unsigned pairs_layout_smem(const unsigned long long* msk, unsigned* off,
                                                      unsigned short* plist);
__device__ __forceinline__ unsigned pairs_layout(const unsigned long long* live, unsigned first, unsigned n,
                                                 unsigned long long* msk, unsigned* off, unsigned short* plist) {
  const int t = threadIdx.x;
  if (t < kPairCands) {
    const unsigned c = first + t;
    msk[t] = c < n ? live[c] : 0ull;
  }
  __syncthreads();
  return pairs_layout_smem(msk, off, plist);
}

// The same from masks already in shared memory (visible to the block).
__device__ __forceinline__ unsigned pairs_layout_smem(const unsigned long long* msk, unsigned* off,
                                                      unsigned short* plist) {
  const int t = threadIdx.x;
  if (t < 32) {
    // two candidates per lane, a warp-wide inclusive scan of their counts
    const unsigned a = __popcll(msk[2 * t]), b = __popcll(msk[2 * t + 1]);
    unsigned incl = a + b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (t >= o) incl += y;
    }
    off[2 * t] = incl - a - b;
    off[2 * t + 1] = incl - b;
    if (t == 31) off[kPairCands] = incl;
  }
  __syncthreads();
  if (t < kPairCands) {
    unsigned o = off[t];
    for (unsigned long long m = msk[t]; m; m &= m - 1) plist[o++] = (unsigned short)((t << 6) | (__ffsll(m) - 1));
  }
  __syncthreads();
  return off[kPairCands];
}

// warp-aggregated append of (candidate << 8 | chain) to the inside list
__device__ __forceinline__ void acc_append(const RefineStage& rs, bool in, unsigned c, int ch, int lane) {
  const unsigned ball = __ballot_sync(0xFFFFFFFFu, in);
  if (!ball) return;
  const int leader = __ffs(ball) - 1;
  unsigned b0 = 0;
  if (lane == leader) b0 = atomicAdd(rs.acc_count, (unsigned)__popc(ball));
  b0 = __shfl_sync(0xFFFFFFFFu, b0, leader);
  if (!in) return;
  const unsigned idx = b0 + __popc(ball & ((1u << lane) - 1u));
  if (idx < rs.acc_cap) rs.acc[idx] = ((unsigned long long)c << 8) | (unsigned)ch;
}

// The single-field exact test, part 1: each block takes kTestCands
// candidates at a time, gathers them with one thread per hypercube vertex (each loading its
// vertex's M components at once, computing its cull word and quantised values
// in registers; the chain test shuffles within the candidate's 2^D lanes),
// keeps the quantised values and chain masks in shared memory, lays the
// surviving (candidate, chain) pairs out, and runs the fast-path inside test
// with one thread per pair, listing the accepted simplices.  Candidates with
// a quantised value past 2^31 go to the 128-bit list instead.
template <typename T, int D>
__global__ void __launch_bounds__(kRefineWarps * 32, 4) refine_test_kernel(RegularMesh mesh, FieldAccess fa,
                                                                          ExtractConfig cfg, CandidateQueue cq,
                                                                          RefineStage rs) {
  constexpr int M = D - 1;
  constexpr int NV = 1 << D;                 // threads per candidate
  constexpr int kThr = kRefineWarps * 32;
  constexpr int PER_PASS = kThr / NV;        // candidates per gather pass
  constexpr int PASSES = kTestCands / PER_PASS;
  constexpr int R = (D == 4) ? 4 : 2;        // chain rounds: ceil(chains / NV), 60 / 16 and 12 / 8
  static_assert(PASSES * PER_PASS == kTestCands, "the gather passes cover the block's candidates");
  __shared__ unsigned band_tbl[kBandTable];
  __shared__ unsigned chain_pk[kMaxChains];
  __shared__ unsigned long long msk[kPairCands];
  __shared__ unsigned off[kPairCands + 1];
  __shared__ unsigned short plist[kTestCands * 64];
  __shared__ __align__(16) int sq[kTestCands * kStageVals];
  fill_band_table<T>(band_tbl, threadIdx.x, blockDim.x);
  for (int i = threadIdx.x; i < kMaxChains; i += blockDim.x) chain_pk[i] = chain_packed<D>(i);
  // the layout scans kPairCands masks; slots past the block's kTestCands stay empty
  if (threadIdx.x >= kTestCands && threadIdx.x < kPairCands) msk[threadIdx.x] = 0ull;
  const int lane = threadIdx.x & 31;
  const int v = threadIdx.x & (NV - 1), grp = lane / NV, slot = threadIdx.x / NV;
  unsigned pkr[R];  // chain_packed of chains r * NV + v
#pragma unroll
  for (int r = 0; r < R; ++r) pkr[r] = r * NV + v < kMaxChains ? chain_packed<D>(r * NV + v) : 0u;
  const int nch = c_chains[D - 3].n;
  const unsigned lowmask = NV == 32 ? 0xFFFFFFFFu : ((1u << NV) - 1u);
  pdl_enter();
  __syncthreads();
  const unsigned n = min(*cq.count, cq.cap);
  for (unsigned first = blockIdx.x * kTestCands; first < n; first += gridDim.x * kTestCands) {
    // every pass's loads first (corners, then the vertices' components, as
    // read-only global loads), so that the passes' memory latencies overlap
    unsigned long long chains_p[PASSES];
    bool in_p[PASSES];
    T x_p[PASSES][M];
#pragma unroll
    for (int pass = 0; pass < PASSES; ++pass) {
      const unsigned c = first + pass * PER_PASS + slot;
      const bool has = c < n;
      const unsigned long long pc = has ? __ldg(&cq.corner[c]) : 0ull;
      chains_p[pass] = has ? __ldg(&cq.chains[c]) : 0ull;
      const long long l[4] = {(long long)(pc & 0xFFFF), (long long)((pc >> 16) & 0xFFFF),
                              (long long)((pc >> 32) & 0xFFFF), (long long)(pc >> 48)};
      long long g[4];
      bool in = has;
      unsigned long long vid = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const long long lq = (D == 4) ? l[q] : (q < 2 ? l[q] : (q == 2 ? l[3] : 0));
        g[q] = (q < D) ? lq + mesh.off[q] + ((v >> q) & 1) : 0;
        if (q < D) {
          in &= g[q] - mesh.off[q] < mesh.ld[q];
          vid += (unsigned long long)g[q] * mesh.gstride[q];
        }
      }
      // the vertex's components: one array offset for all of them
      long long o = 0;
      if (!fa.per_vertex) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (q < D) {
            long long a = g[q] - fa.shift[q];
            if (q == D - 1) a ^= fa.tflip;
            o += a * fa.estride[q];
          }
      } else {
        o = (long long)vid;
      }
      in_p[pass] = in;
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const T* src = static_cast<const T*>(j == 0 ? fa.comp[0] : (j == 1 ? fa.comp[1] : fa.comp[2]));
        x_p[pass][j] = in ? __ldg(src + o) : T(0);
      }
    }
#pragma unroll
    for (int pass = 0; pass < PASSES; ++pass) {
      const int k = pass * PER_PASS + slot;
      const unsigned c = first + k;
      const bool has = c < n, in = in_p[pass];
      const unsigned long long chains = chains_p[pass];
      unsigned h[M];
      bool big = false;
#pragma unroll
      for (int j = 0; j < M; ++j) {
        T x = x_p[pass][j];
        if (cfg.fiber) x = fp<T>::sub(x, (T)(j ? cfg.fthr[1] : cfg.fthr[0]));  // values[i][j] - thresholds[j]
        h[j] = hi_word<T>(x);
        const int qv = quant_small_p(quant_p((double)x, cfg.Q));
        big |= qv == kQBig;
        if (FTK2B_CHECK(k * kStageVals + v * M + j < kTestCands * kStageVals, rs.err)) sq[k * kStageVals + v * M + j] = qv;
      }
      const unsigned vw = in ? vertex_word_hi<T, M>(h, band_tbl) : kAbsent;  // absent: neutral under AND
      const bool gbig = ((__ballot_sync(0xFFFFFFFFu, big) >> (grp * NV)) & lowmask) != 0;
      const unsigned w0 = __shfl_sync(0xFFFFFFFFu, vw, 0, NV);
      unsigned long long mask = 0;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int ch = r * NV + v;
        bool live = ch < nch && ((chains >> ch) & 1ull);
        unsigned wacc = w0;
#pragma unroll
        for (int i = 0; i < M; ++i) wacc &= __shfl_sync(0xFFFFFFFFu, vw, (pkr[r] >> (8 * i)) & 0xFF, NV);
        live = live && (cfg.fiber || !word_culled(wacc));
        mask |= (unsigned long long)((__ballot_sync(0xFFFFFFFFu, live) >> (grp * NV)) & lowmask) << (r * NV);
      }
      if (v == 0) {
        // a candidate holding a value off the fast path: every chain on the
        // 128-bit path (at most one list entry per candidate)
        unsigned long long fast = mask;
        if (has && gbig && mask) {
          const unsigned s2 = atomicAdd(rs.big_count, 1u);
          rs.big_list[s2] = c;
          rs.big_live[s2] = mask;
          fast = 0;
        }
        msk[k] = fast;
      }
    }
    __syncthreads();
    const unsigned P = pairs_layout_smem(msk, off, plist);
    if (threadIdx.x == 0) atomicAdd(rs.count, P);
    for (unsigned base = 0; base < P; base += blockDim.x) {
      const unsigned p = base + threadIdx.x;
      const unsigned e = p < P ? plist[p] : 0u;
      const int k = (int)(e >> 6), ch = (int)(e & 63);
      const bool ins = p < P && inside_pair_q<D>(ch, sq + k * kStageVals, chain_pk);
      acc_append(rs, ins, first + k, ch, lane);
    }
    __syncthreads();  // shared memory is rebuilt for the next candidates
  }
}

// The single-field exact test, part 2: blocks below solve_blocks solve the
// simplices on the inside list (one thread each; a list longer than its
// capacity raises the sink count past the sink's capacity, so that the call
// reports overflow and runs again with larger buffers); the others run the
// whole test on the candidates listed for the 128-bit path.  Values are read
// from the field.
template <typename T, int D>
__global__ void __launch_bounds__(kRefineWarps * 32, 2) refine_accept_kernel(RegularMesh mesh, FieldAccess fa,
                                                                            ExtractConfig cfg, CandidateQueue cq,
                                                                            RefineStage rs, FeatureSink sink,
                                                                            int solve_blocks) {
  __shared__ unsigned long long msk[kPairCands];
  __shared__ unsigned off[kPairCands + 1];
  __shared__ unsigned chain_pk[kMaxChains];
  __shared__ unsigned short plist[kPairCands * 64];
  for (int i = threadIdx.x; i < kMaxChains; i += blockDim.x) chain_pk[i] = chain_packed<D>(i);
  pdl_enter();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  if ((int)blockIdx.x < solve_blocks) {
    const unsigned na = *rs.acc_count;
    if (blockIdx.x == 0 && threadIdx.x == 0 && na > rs.acc_cap) atomicMax(sink.count, na);
    const unsigned n = min(na, rs.acc_cap);
    const unsigned stride = solve_blocks * blockDim.x;
    for (unsigned base = blockIdx.x * blockDim.x; base < n; base += stride) {
      const unsigned i = base + threadIdx.x;
      bool acc = false;
      double lam_out[4] = {0, 0, 0, 0};
      float bary_out[4] = {0.f, 0.f, 0.f, 0.f};
      float sc_out = 0.f;
      unsigned long long key = 0;
      if (i < n) {
        const unsigned long long e = rs.acc[i];
        const unsigned c = (unsigned)(e >> 8);
        if (FTK2B_CHECK(c < min(*cq.count, cq.cap) && (e & 255) < kMaxChains, rs.err))
          acc = test_pair<T, D, false>(mesh, fa, cfg, cq.corner[c], (int)(e & 255), (const T*)nullptr, chain_pk, 0ull,
                                       key, lam_out, bary_out, sc_out);
      }
      sink_write(sink, acc, key, lam_out, bary_out, sc_out, lane);
    }
    return;
  }
  const unsigned nb = *rs.big_count;
  const unsigned bb = blockIdx.x - solve_blocks, nbb = gridDim.x - solve_blocks;
  for (unsigned first = bb * kPairCands; first < nb; first += nbb * kPairCands) {
    const unsigned P = pairs_layout(rs.big_live, first, nb, msk, off, plist);
    if (threadIdx.x == 0) atomicAdd(rs.count, P);
    for (unsigned base = 0; base < P; base += blockDim.x) {
      const unsigned p = base + threadIdx.x;
      const unsigned e = p < P ? plist[p] : 0u;
      const int k = (int)(e >> 6), ch = (int)(e & 63);
      bool acc = false;
      double lam_out[4] = {0, 0, 0, 0};
      float bary_out[4] = {0.f, 0.f, 0.f, 0.f};
      float sc_out = 0.f;
      unsigned long long key = 0;
      if (p < P) {
        const unsigned c = rs.big_list[first + k];
        acc = test_pair<T, D, true>(mesh, fa, cfg, cq.corner[c], ch, (const T*)nullptr, chain_pk, 0ull, key, lam_out,
                                    bary_out, sc_out);
      }
      sink_write(sink, acc, key, lam_out, bary_out, sc_out, lane);
    }
    __syncthreads();
  }
}

// One candidate of a batch by a group of 16 lanes, one per hypercube vertex
// (lanes 8-15 idle for a 2D+t field): the quantised form of its values into
// qout (the vertex's M values at qout[v * M]), the vertices' cull words, and
// the mask of the chains that survive them into *live_out (or, with a
// quantised value past 2^31, the candidate onto the 128-bit list and 0 into
// *live_out).  gmask: the group's lanes; gshift: its first lane.
template <typename T, int D>
__device__ __forceinline__ void gather_group(const RegularMesh& mesh, const FieldAccess& fa, const ExtractConfig& cfg,
                                             unsigned c, unsigned long long pc, unsigned long long chains, int v,
                                             unsigned gmask, int gshift, const unsigned* band_tbl,
                                             const unsigned* chain_pk, const RefineStage& rs, int* qout,
                                             unsigned long long* live_out) {
  constexpr int M = D - 1;
  constexpr int NV = 1 << D;
  constexpr int R = (D == 4) ? 4 : 1;  // chain rounds of 16: 60 and 12 chains
  const int nch = c_chains[D - 3].n;
  const long long l[4] = {(long long)(pc & 0xFFFF), (long long)((pc >> 16) & 0xFFFF),
                          (long long)((pc >> 32) & 0xFFFF), (long long)(pc >> 48)};
  long long g[4];
  bool in = v < NV;
  unsigned long long vid = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long lq = (D == 4) ? l[q] : (q < 2 ? l[q] : (q == 2 ? l[3] : 0));
    g[q] = (q < D) ? lq + mesh.off[q] + ((v >> q) & 1) : 0;
    if (q < D) {
      in &= g[q] - mesh.off[q] < mesh.ld[q];
      vid += (unsigned long long)g[q] * mesh.gstride[q];
    }
  }
  long long o = 0;
  if (!fa.per_vertex) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (q < D) {
        long long a = g[q] - fa.shift[q];
        if (q == D - 1) a ^= fa.tflip;
        o += a * fa.estride[q];
      }
  } else {
    o = (long long)vid;
  }
  unsigned h[M];
  bool big = false;
  T x[M];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const T* src = static_cast<const T*>(j == 0 ? fa.comp[0] : (j == 1 ? fa.comp[1] : fa.comp[2]));
    x[j] = in ? __ldg(src + o) : T(0);
  }
#pragma unroll
  for (int j = 0; j < M; ++j) {
    if (cfg.fiber) x[j] = fp<T>::sub(x[j], (T)(j ? cfg.fthr[1] : cfg.fthr[0]));  // values[i][j] - thresholds[j]
    h[j] = hi_word<T>(x[j]);
    const int qv = quant_small_p(quant_p((double)x[j], cfg.Q));
    big |= v < NV && qv == kQBig;
    if (v < NV) qout[v * M + j] = qv;
  }
  const unsigned vw = in ? vertex_word_hi<T, M>(h, band_tbl) : kAbsent;  // absent: neutral under AND
  const bool gbig = ((__ballot_sync(gmask, big) >> gshift) & 0xFFFFu) != 0;
  const unsigned w0 = __shfl_sync(gmask, vw, 0, 16);
  unsigned long long mask = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int ch = r * 16 + v;
    bool live = ch < nch && ((chains >> ch) & 1ull);
    const unsigned pk = chain_pk[ch];
    unsigned wacc = w0;
#pragma unroll
    for (int i = 0; i < M; ++i) wacc &= __shfl_sync(gmask, vw, (pk >> (8 * i)) & 0xFF, 16);
    live = live && (cfg.fiber || !word_culled(wacc));
    mask |= (unsigned long long)((__ballot_sync(gmask, live) >> gshift) & 0xFFFFu) << (r * 16);
  }
  if (v == 0) {
    unsigned long long fast = mask;
    if (gbig && mask) {
      const unsigned slot = atomicAdd(rs.big_count, 1u);
      rs.big_list[slot] = c;
      rs.big_live[slot] = mask;
      fast = 0;
    }
    *live_out = fast;
  }
}

// Batches, exact test part 1: refine_test_kernel with every candidate's own
// field record.  A block takes kTestCands candidates at a time, 16 lanes per
// candidate (two per warp), quantises their values into shared memory, lays
// out the (candidate, chain) pairs that survive the cull words and runs the
// fast-path inside test with one thread per pair, listing the accepted
// simplices; candidates holding a quantised value past 2^31 go to the
// 128-bit list.
template <typename T>
__global__ void __launch_bounds__(kRefineWarps * 32, 4) batch_test_kernel(const BatchField* __restrict__ fields,
                                                                         CandidateQueue cq, RefineStage rs) {
  constexpr int PER_PASS = kRefineWarps * 2;  // candidates per gather pass
  constexpr int PASSES = kTestCands / PER_PASS;
  static_assert(PASSES * PER_PASS == kTestCands, "the gather passes cover the block's candidates");
  __shared__ unsigned band_tbl[kBandTable];
  __shared__ unsigned chain_pk[2][kMaxChains];
  __shared__ unsigned long long msk[kPairCands];
  __shared__ unsigned off[kPairCands + 1];
  __shared__ unsigned short plist[kTestCands * 64];
  __shared__ __align__(16) int sq[kTestCands * kStageVals];
  __shared__ int sd[kTestCands];  // the dimension of each candidate's mesh
  fill_band_table<T>(band_tbl, threadIdx.x, blockDim.x);
  for (int i = threadIdx.x; i < kMaxChains; i += blockDim.x) {
    chain_pk[0][i] = chain_packed<3>(i);
    chain_pk[1][i] = chain_packed<4>(i);
  }
  // the layout scans kPairCands masks; slots past the block's kTestCands stay empty
  if (threadIdx.x >= kTestCands && threadIdx.x < kPairCands) msk[threadIdx.x] = 0ull;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int v = lane & 15, grp = lane >> 4;
  const unsigned gmask = 0xFFFFu << (16 * grp);
  pdl_enter();
  __syncthreads();
  const unsigned n = min(*cq.count, cq.cap);
  for (unsigned first = blockIdx.x * kTestCands; first < n; first += gridDim.x * kTestCands) {
#pragma unroll
    for (int pass = 0; pass < PASSES; ++pass) {
      const int k = pass * PER_PASS + wib * 2 + grp;
      const unsigned c = first + k;
      if (c >= n) {  // the whole group
        if (v == 0) msk[k] = 0ull;
        continue;
      }
      const BatchField& F = fields[cq.field[c]];
      const unsigned long long pc = __ldg(&cq.corner[c]), chains = __ldg(&cq.chains[c]);
      const int d = F.mesh.d;
      if (v == 0) sd[k] = d;
      if (d == 4)
        gather_group<T, 4>(F.mesh, F.fa, F.cfg, c, pc, chains, v, gmask, 16 * grp, band_tbl, chain_pk[1], rs,
                           sq + k * kStageVals, &msk[k]);
      else
        gather_group<T, 3>(F.mesh, F.fa, F.cfg, c, pc, chains, v, gmask, 16 * grp, band_tbl, chain_pk[0], rs,
                           sq + k * kStageVals, &msk[k]);
    }
    __syncthreads();
    const unsigned P = pairs_layout_smem(msk, off, plist);
    if (threadIdx.x == 0) atomicAdd(rs.count, P);
    for (unsigned base = 0; base < P; base += blockDim.x) {
      const unsigned p = base + threadIdx.x;
      const unsigned e = p < P ? plist[p] : 0u;
      const int k = (int)(e >> 6), ch = (int)(e & 63);
      bool ins = false;
      if (p < P && FTK2B_CHECK(k < kTestCands, rs.err))
        ins = sd[k] == 4 ? inside_pair_q<4>(ch, sq + k * kStageVals, chain_pk[1])
                         : inside_pair_q<3>(ch, sq + k * kStageVals, chain_pk[0]);
      acc_append(rs, ins, first + k, ch, lane);
    }
    __syncthreads();  // shared memory is rebuilt for the next candidates
  }
}

// Batches, the whole test with the 128-bit path of the candidates on that
// list, values read from each candidate's field.
template <typename T>
__global__ void __launch_bounds__(kRefineWarps * 32, 2) batch_big_kernel(const BatchField* __restrict__ fields,
                                                                        CandidateQueue cq, RefineStage rs,
                                                                        FeatureSink sink) {
  __shared__ unsigned long long msk[kPairCands];
  __shared__ unsigned off[kPairCands + 1];
  __shared__ unsigned chain_pk[2][kMaxChains];
  __shared__ unsigned short plist[kPairCands * 64];
  for (int i = threadIdx.x; i < kMaxChains; i += blockDim.x) {
    chain_pk[0][i] = chain_packed<3>(i);
    chain_pk[1][i] = chain_packed<4>(i);
  }
  pdl_enter();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned n = *rs.big_count;
  for (unsigned first = blockIdx.x * kPairCands; first < n; first += gridDim.x * kPairCands) {
    const unsigned P = pairs_layout(rs.big_live, first, n, msk, off, plist);
    if (threadIdx.x == 0) atomicAdd(rs.count, P);
    for (unsigned base = 0; base < P; base += blockDim.x) {
      const unsigned p = base + threadIdx.x;
      const unsigned e = p < P ? plist[p] : 0u;
      const int k = (int)(e >> 6), ch = (int)(e & 63);
      bool acc = false;
      double lam_out[4] = {0, 0, 0, 0};
      float bary_out[4] = {0.f, 0.f, 0.f, 0.f};
      float sc_out = 0.f;
      unsigned long long key = 0;
      if (p < P) {
        const unsigned c = rs.big_list[first + k];
        const BatchField& F = fields[cq.field[c]];
        if (F.mesh.d == 4)
          acc = test_pair<T, 4, true>(F.mesh, F.fa, F.cfg, cq.corner[c], ch, (const T*)nullptr, chain_pk[1],
                                      F.key_base, key, lam_out, bary_out, sc_out);
        else
          acc = test_pair<T, 3, true>(F.mesh, F.fa, F.cfg, cq.corner[c], ch, (const T*)nullptr, chain_pk[0],
                                      F.key_base, key, lam_out, bary_out, sc_out);
      }
      sink_write(sink, acc, key, lam_out, bary_out, sc_out, lane);
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(kRefineWarps * 32) batch_solve_kernel(const BatchField* __restrict__ fields,
                                                                        CandidateQueue cq, RefineStage rs,
                                                                        FeatureSink sink) {
  __shared__ unsigned chain_pk[2][kMaxChains];
  for (int i = threadIdx.x; i < kMaxChains; i += blockDim.x) {
    chain_pk[0][i] = chain_packed<3>(i);
    chain_pk[1][i] = chain_packed<4>(i);
  }
  pdl_enter();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned na = *rs.acc_count;
  if (blockIdx.x == 0 && threadIdx.x == 0 && na > rs.acc_cap) atomicMax(sink.count, na);
  const unsigned n = min(na, rs.acc_cap);
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const unsigned i = base + threadIdx.x;
    bool acc = false;
    double lam_out[4] = {0, 0, 0, 0};
    float bary_out[4] = {0.f, 0.f, 0.f, 0.f};
    float sc_out = 0.f;
    unsigned long long key = 0;
    if (i < n) {
      const unsigned long long e = rs.acc[i];
      const unsigned c = (unsigned)(e >> 8);
      const int ch = (int)(e & 255);
      const BatchField& F = fields[cq.field[c]];
      if (F.mesh.d == 4)
        acc = test_pair<T, 4, false>(F.mesh, F.fa, F.cfg, cq.corner[c], ch, (const T*)nullptr, chain_pk[1],
                                     F.key_base, key, lam_out, bary_out, sc_out);
      else
        acc = test_pair<T, 3, false>(F.mesh, F.fa, F.cfg, cq.corner[c], ch, (const T*)nullptr, chain_pk[0],
                                     F.key_base, key, lam_out, bary_out, sc_out);
    }
    sink_write(sink, acc, key, lam_out, bary_out, sc_out, lane);
  }
}

// ---------------------------------------------------------------------------
// Batches: every field's tiles in one persistent launch, every candidate of
// the batch in one exact-test launch.  Each item runs the single-field code
// (cull_tile, refine_candidate) with its field's record, so a field's
// candidates and features are those of its own extraction.

constexpr int kBatchSmemFields = 2048;  // item bases kept in shared memory up to this many fields

template <typename T, bool MULTI>
__global__ void __launch_bounds__(kThreads, 2)
    batch_cull_kernel(const BatchField* __restrict__ fields, const unsigned* __restrict__ item_base, int nf,
                      unsigned n_items, unsigned* item_next, CandidateQueue cq, unsigned* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned long long bar[5];
  __shared__ unsigned band_tbl[kBandTable];
  __shared__ unsigned s_item, s_field;
  __shared__ unsigned s_ib[kBatchSmemFields];
  // candidate buffer shared by the items of every dimension: an item's
  // candidates are flushed by the block's next item
  __shared__ unsigned long long s_cbuf[2 * kCandBuf];
  __shared__ unsigned s_ccount[2];
  __shared__ RegularMesh s_mesh;
  __shared__ FieldAccess s_fa;
  __shared__ ExtractConfig s_cfg;
  __shared__ int s_tma;
  __shared__ unsigned s_ibase;
  static_assert(sizeof(RegularMesh) % 4 == 0 && sizeof(FieldAccess) % 4 == 0 && sizeof(ExtractConfig) % 4 == 0 &&
                    (sizeof(RegularMesh) + sizeof(FieldAccess) + sizeof(ExtractConfig)) / 4 <= kThreads,
                "one thread per word of a field record");
  const bool ib_smem = nf <= kBatchSmemFields;
  if (ib_smem)
    for (int i = threadIdx.x; i < nf; i += kThreads) s_ib[i] = item_base[i];
  const unsigned* ib = ib_smem ? s_ib : item_base;
  fill_band_table<T>(band_tbl, threadIdx.x, kThreads);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    mbar_init(&bar[3], kThreads);
    mbar_init(&bar[4], kThreads);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  unsigned ph = 0;  // phase parities of bar[0], bar[1], bar[3], bar[4]
  // thread 0 takes the next item while the block works on the current one
  unsigned next = threadIdx.x == 0 ? atomicAdd(item_next, 1u) : 0u;
  unsigned cur_field = 0xFFFFFFFFu;  // field whose record is in shared memory
  unsigned last_field = 0;           // field of the candidates in the buffer
  if (threadIdx.x == 0) s_ccount[0] = 0;
  for (;;) {
    __syncthreads();  // s_item of the previous item has been read by every thread
    if (threadIdx.x == 0) {
      const unsigned it = next;
      if (it < n_items) next = atomicAdd(item_next, 1u);
      unsigned f = 0;
      if (it < n_items) {
        // the last field whose first item is <= it
        unsigned lo = 0, hi = (unsigned)nf;
        while (hi - lo > 1) {
          const unsigned mid = (lo + hi) >> 1;
          if (ib[mid] <= it) lo = mid;
          else hi = mid;
        }
        f = lo;
      }
      s_item = it;
      s_field = f;
    }
    __syncthreads();
    const unsigned it = s_item;
    if (it >= n_items) break;
    const unsigned f = s_field;
    const BatchField& F = fields[f];
    // the field's mesh, access and configuration into shared memory when the
    // item belongs to another field than the previous one (the tensor maps
    // stay in global memory, where TMA reads them)
    if (f != cur_field) {
      cur_field = f;
      constexpr int kMw = sizeof(RegularMesh) / 4, kFw = sizeof(FieldAccess) / 4, kCw = sizeof(ExtractConfig) / 4;
      const unsigned* src_m = reinterpret_cast<const unsigned*>(&F.mesh);
      const unsigned* src_f = reinterpret_cast<const unsigned*>(&F.fa);
      const unsigned* src_c = reinterpret_cast<const unsigned*>(&F.cfg);
      const int t = threadIdx.x;
      if (t < kMw) reinterpret_cast<unsigned*>(&s_mesh)[t] = src_m[t];
      else if (t < kMw + kFw) reinterpret_cast<unsigned*>(&s_fa)[t - kMw] = src_f[t - kMw];
      else if (t < kMw + kFw + kCw) reinterpret_cast<unsigned*>(&s_cfg)[t - kMw - kFw] = src_c[t - kMw - kFw];
      if (t == 0) {
        s_tma = F.tma;
        s_ibase = F.item_base;
      }
      __syncthreads();
    }
    const unsigned local = it - s_ibase;
    const unsigned ntiles = (unsigned)s_cfg.tiles[0] * s_cfg.tiles[1] * s_cfg.tiles[2];
    CandidateQueue q = cq;
    q.field_id = f;
    bool ok;
    if (s_mesh.d == 4) {
      ok = s_tma ? cull_tile<T, 4, MULTI, true>(&F.maps[0], &F.maps[1], &F.maps[2], s_mesh, s_fa, s_cfg, q, err,
                                                (int)(local % ntiles), (int)(local / ntiles), smem, bar, band_tbl,
                                                ph, s_cbuf, s_ccount, true, last_field)
                 : cull_tile<T, 4, MULTI, false>(&F.maps[0], &F.maps[1], &F.maps[2], s_mesh, s_fa, s_cfg, q, err,
                                                 (int)(local % ntiles), (int)(local / ntiles), smem, bar, band_tbl,
                                                 ph, s_cbuf, s_ccount, true, last_field);
    } else {
      ok = s_tma ? cull_tile<T, 3, MULTI, true>(&F.maps[0], &F.maps[1], &F.maps[2], s_mesh, s_fa, s_cfg, q, err,
                                                (int)(local % ntiles), (int)(local / ntiles), smem, bar, band_tbl,
                                                ph, s_cbuf, s_ccount, true, last_field)
                 : cull_tile<T, 3, MULTI, false>(&F.maps[0], &F.maps[1], &F.maps[2], s_mesh, s_fa, s_cfg, q, err,
                                                 (int)(local % ntiles), (int)(local / ntiles), smem, bar, band_tbl,
                                                 ph, s_cbuf, s_ccount, true, last_field);
    }
    last_field = f;
    if (!ok) break;  // the whole block saw the failed wait
  }
  // the last item's candidates
  __syncthreads();
  flush_candidates(s_cbuf, s_ccount, cq, last_field);
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
  unsigned pk[2][kMaxChains] = {};
  for (int t = 0; t < 2; ++t)
    for (int c = 0; c < h[t].n; ++c)
      for (int k = 0; k < t + 2; ++k) pk[t][c] |= (unsigned)h[t].mask[c][k] << (8 * k);
  cudaMemcpyToSymbol(g_chain_pk, pk, sizeof(pk));
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

// TMA applies when every box starts on a 16-byte boundary and the array
// strides are multiples of 16 bytes: inner coordinate = array x * (M or 1)
template <typename T, int D, bool MULTI>
static bool build_tma_maps(const RegularMesh& mesh, const FieldAccess& fa, bool allow_tma, CUtensorMap maps[3]) {
  using G = Geo<T, D, MULTI>;
  constexpr int M = D - 1;
  const size_t es = sizeof(T);
  memset(maps, 0, 3 * sizeof(CUtensorMap));
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
  return tma;
}

bool regular_tma_maps(int f64, const RegularMesh& mesh, const FieldAccess& fa, bool allow, CUtensorMap maps[3]) {
  const bool multi = !fa.per_vertex && fa.estride[0] == mesh.d - 1;
  if (mesh.d == 4) {
    if (f64) return multi ? build_tma_maps<double, 4, true>(mesh, fa, allow, maps)
                          : build_tma_maps<double, 4, false>(mesh, fa, allow, maps);
    return multi ? build_tma_maps<float, 4, true>(mesh, fa, allow, maps)
                 : build_tma_maps<float, 4, false>(mesh, fa, allow, maps);
  }
  if (f64) return multi ? build_tma_maps<double, 3, true>(mesh, fa, allow, maps)
                        : build_tma_maps<double, 3, false>(mesh, fa, allow, maps);
  return multi ? build_tma_maps<float, 3, true>(mesh, fa, allow, maps)
               : build_tma_maps<float, 3, false>(mesh, fa, allow, maps);
}

constexpr int kStatsStages = 4;

template <typename T, int D, int XT>
cudaError_t launch_stats_stream(const RegularMesh& mesh, const FieldAccess& fa, const ExtractConfig& cfg,
                                int ntasks, cudaStream_t st) {
  using SS = StatsStream<T, D, XT, kStatsStages>;
  auto k = plane_stats_stream_kernel<T, D, XT, kStatsStages>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SS::SMEM);
  if (e) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, SS::THREADS, SS::SMEM) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  const long long want = (long long)sms * per_sm;
  const long long need = (ntasks + kStatsWarps - 1) / kStatsWarps;
  k<<<(unsigned)std::max<long long>(1, std::min(want, need)), SS::THREADS, SS::SMEM, st>>>(mesh, fa, cfg, ntasks);
  return cudaGetLastError();
}

template <typename T, int D, bool MULTI>
static cudaError_t launch_t(const RegularMesh& mesh, const FieldAccess& fa, const ExtractConfig& cfg,
                            const CandidateQueue& cq, unsigned* err, cudaStream_t st, bool allow_tma,
                            int* used_tma, int* launches) {
  using G = Geo<T, D, MULTI>;
  constexpr int M = D - 1;

  CUtensorMap maps[3];
  const bool tma = build_tma_maps<T, D, MULTI>(mesh, fa, allow_tma, maps);
  if (used_tma) *used_tma = tma ? 1 : 0;
  const size_t shm = G::SMEM;
  const long long lt = mesh.ld[D - 1];
  const unsigned nchunks = (unsigned)((lt + cfg.tchunk - 1) / cfg.tchunk);
  const unsigned ntiles = (unsigned)cfg.tiles[0] * cfg.tiles[1] * cfg.tiles[2];
  dim3 grid(ntiles, nchunks);
  cudaError_t e;
  // cull mode 1: arrays the TMA kernels can stage, with the caller's scratch
  const bool vec_ok = tma && cfg.tstats && cfg.runs && cfg.n_runs && cfg.runs_cap;
  bool sep = false, stats_ok = false;
  if (cfg.cull_mode == 1 && vec_ok) {
    bool ilv = MULTI && fa.estride[0] == M;
    for (int j = 1; j < M && ilv; ++j)
      ilv = static_cast<const char*>(fa.comp[j]) == static_cast<const char*>(fa.comp[0]) + j * sizeof(T);
    // interleaved rows are read with 16-byte vectors, which needs every row
    // of a chunk to start on a 16-byte boundary (as the TMA boxes do)
    bool vec = ilv && (reinterpret_cast<uintptr_t>(fa.comp[0]) % 16 == 0) &&
               ((mesh.off[0] - fa.shift[0]) * M * (long long)sizeof(T)) % 16 == 0;
    for (int k = 1; k < D && vec; ++k) vec = (fa.estride[k] * (long long)sizeof(T)) % 16 == 0;
    sep = !ilv;
    stats_ok = vec || sep;
  }
  if (cfg.cull_mode == 1 && vec_ok && stats_ok) {
    // chunks of 8 x-tiles (256 vertices) for interleaved float rows, else 4
    const int xt = (cfg.tiles[0] <= 4 || sep || sizeof(T) == 8) ? 4 : 8;
    const long long ldz = (D == 4) ? mesh.ld[2] : 1;
    const long long tasks = (long long)((cfg.tiles[0] + xt - 1) / xt) * cfg.tiles[1] * ldz * lt;
    if (sep) {
      const unsigned sblocks = (unsigned)((tasks + kStatsWarps - 1) / kStatsWarps);
      plane_stats_kernel<T, D, 4><<<sblocks, kStatsWarps * 32, 0, st>>>(mesh, fa, cfg);
    } else {
      if (tasks >= 0x7FFFFFFF) return cudaErrorInvalidValue;
      if (xt == 4) e = launch_stats_stream<T, D, 4>(mesh, fa, cfg, (int)tasks, st);
      else e = launch_stats_stream<T, D, 8>(mesh, fa, cfg, (int)tasks, st);
      if (e) return e;
    }
    if ((e = cudaMemsetAsync(cfg.n_runs, 0, sizeof(unsigned), st))) return e;
    tile_runs_kernel<T, D><<<(unsigned)std::max<long long>(1, (ntiles + 255) / 256), 256, 0, st>>>(mesh, cfg);
    const size_t shm2 = Geo2<T, D, MULTI>::SMEM;
    auto k = run_cull_kernel<T, D, MULTI, true>;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm2);
    if (e) return e;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, shm2) != cudaSuccess || per_sm < 1) {
      cudaGetLastError();
      per_sm = 1;
    }
    // persistent CTAs; each reads the device-side run count itself
    k<<<(unsigned)(sms * per_sm), kThreads, shm2, st>>>(maps[0], maps[1], maps[2], mesh, fa, cfg, cq, err);
    if (launches) *launches = 3;
    return cudaGetLastError();
  }
  if (launches) *launches = 1;
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
                             int* used_tma, int* launches) {
  const bool multi = !fa.per_vertex && fa.estride[0] == D - 1;  // interleaved components
  return multi ? launch_t<T, D, true>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma, launches)
               : launch_t<T, D, false>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma, launches);
}

void tile_scratch_size(const RegularMesh& mesh, size_t* stats_bytes, unsigned* runs_cap) {
  int TX, TY, TZ;
  regular_tile(mesh.d, &TX, &TY, &TZ);
  const long long tiles = ((mesh.ld[0] + TX - 1) / TX) * ((mesh.ld[1] + TY - 1) / TY) *
                          (mesh.d == 4 ? (mesh.ld[2] + TZ - 1) / TZ : 1);
  const long long lt = mesh.ld[mesh.d - 1];
  // one 32-byte entry per (slice, z plane, y-tile, x-tile)
  const long long planes = (mesh.d == 4) ? mesh.ld[2] : 1;
  const long long ptiles = ((mesh.ld[0] + TX - 1) / TX) * ((mesh.ld[1] + TY - 1) / TY);
  *stats_bytes = (size_t)(32 * ptiles * planes * lt);
  // runs of surviving steps are separated by dropped ones: at most
  // ceil(lt / 2) per tile
  *runs_cap = (unsigned)std::min<long long>(tiles * ((lt + 1) / 2), 0x7FFFFFFF);
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
                                   cudaStream_t st, bool allow_tma, int* used_tma, int* launches) {
  if (mesh.d == 4)
    return f64 ? launch_td<double, 4>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma, launches)
               : launch_td<float, 4>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma, launches);
  return f64 ? launch_td<double, 3>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma, launches)
             : launch_td<float, 3>(mesh, fa, cfg, cq, err, st, allow_tma, used_tma, launches);
}

// FiberPredicate candidates: every local vertex is a hypercube corner whose
// chains inside the mesh all need the exact test (a chain is inside when its
// last vertex, the union of its steps, is).
__global__ void fiber_candidates_kernel(RegularMesh mesh, CandidateQueue cq) {
  const int D = mesh.d;
  const ChainTable& CT = c_chains[D - 3];
  unsigned long long nv = 1;
  for (int k = 0; k < D; ++k) nv *= (unsigned long long)mesh.ld[k];
  const unsigned long long n = nv < cq.cap ? nv : cq.cap;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long r = i, l[4] = {0, 0, 0, 0};
    unsigned inb = 0;
    for (int k = 0; k < D; ++k) {
      l[k] = r % (unsigned long long)mesh.ld[k];
      r /= (unsigned long long)mesh.ld[k];
      if (l[k] + 1 < (unsigned long long)mesh.ld[k]) inb |= 1u << k;
    }
    unsigned long long chains = 0;
    for (int ch = 0; ch < CT.n; ++ch)
      if ((CT.mask[ch][D - 2] & ~inb) == 0) chains |= 1ull << ch;
    // corner layout of the candidate queue: x | y << 16 | z << 32 | t << 48
    const unsigned long long t = l[D - 1];
    cq.corner[i] = l[0] | (l[1] << 16) | (D == 4 ? l[2] << 32 : 0ull) | (t << 48);
    cq.chains[i] = chains;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *cq.count = (unsigned)(nv < 0xFFFFFFFFull ? nv : 0xFFFFFFFFull);
}

cudaError_t launch_fiber_candidates(const RegularMesh& mesh, const CandidateQueue& cq, int num_sms,
                                    cudaStream_t st) {
  fiber_candidates_kernel<<<num_sms * 8, 256, 0, st>>>(mesh, cq);
  return cudaGetLastError();
}

template <typename T, int D>
static cudaError_t launch_refine_staged_t(const RegularMesh& mesh, const FieldAccess& fa, const ExtractConfig& cfg,
                                          const CandidateQueue& cq, const RefineStage& rs, const FeatureSink& sink,
                                          int num_sms, cudaStream_t st) {
  const int thr = kRefineWarps * 32;
  // programmatic dependent launches: each kernel waits for its predecessor
  // at its start (pdl_enter), so its launch overlaps the predecessor's tail
  // more blocks than fit at once: each takes one group while the candidates
  // last, and a block that finishes early makes room for the next
  cudaError_t e = launch_pdl(refine_test_kernel<T, D>, num_sms * 16, thr, 0, st, mesh, fa, cfg, cq, rs);
  // solve blocks, then blocks for the (usually short or empty) 128-bit list
  if (!e) e = launch_pdl(refine_accept_kernel<T, D>, num_sms * 2, thr, 0, st, mesh, fa, cfg, cq, rs, sink, num_sms);
  return e ? e : cudaGetLastError();
}

cudaError_t launch_refine_staged(int f64, const RegularMesh& mesh, const FieldAccess& fa, const ExtractConfig& cfg,
                                 const CandidateQueue& cq, const RefineStage& rs, const FeatureSink& sink, int num_sms,
                                 cudaStream_t st) {
  if (mesh.d == 4)
    return f64 ? launch_refine_staged_t<double, 4>(mesh, fa, cfg, cq, rs, sink, num_sms, st)
               : launch_refine_staged_t<float, 4>(mesh, fa, cfg, cq, rs, sink, num_sms, st);
  return f64 ? launch_refine_staged_t<double, 3>(mesh, fa, cfg, cq, rs, sink, num_sms, st)
             : launch_refine_staged_t<float, 3>(mesh, fa, cfg, cq, rs, sink, num_sms, st);
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


template <typename T, bool MULTI>
static cudaError_t launch_batch_cull_t(const BatchField* fields, const unsigned* item_base, int nf, unsigned n_items,
                                       unsigned* item_next, const CandidateQueue& cq, unsigned* err,
                                       cudaStream_t st) {
  constexpr int shm = Geo<T, 4, MULTI>::SMEM > Geo<T, 3, MULTI>::SMEM ? Geo<T, 4, MULTI>::SMEM
                                                                      : Geo<T, 3, MULTI>::SMEM;
  auto k = batch_cull_kernel<T, MULTI>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, shm);
  if (e) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, shm) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  const long long want = (long long)sms * per_sm;
  k<<<(unsigned)std::max<long long>(1, std::min<long long>(want, n_items)), kThreads, shm, st>>>(
      fields, item_base, nf, n_items, item_next, cq, err);
  return cudaGetLastError();
}

cudaError_t launch_batch_cull(int f64, int multi, const BatchField* fields, const unsigned* item_base, int nf,
                              unsigned n_items, unsigned* item_next, const CandidateQueue& cq, unsigned* err,
                              cudaStream_t st) {
  if (f64) return multi ? launch_batch_cull_t<double, true>(fields, item_base, nf, n_items, item_next, cq, err, st)
                        : launch_batch_cull_t<double, false>(fields, item_base, nf, n_items, item_next, cq, err, st);
  return multi ? launch_batch_cull_t<float, true>(fields, item_base, nf, n_items, item_next, cq, err, st)
               : launch_batch_cull_t<float, false>(fields, item_base, nf, n_items, item_next, cq, err, st);
}

template <typename T>
static cudaError_t launch_batch_refine_t(const BatchField* fields, const CandidateQueue& cq, const RefineStage& rs,
                                         const FeatureSink& sink, int num_sms, cudaStream_t st) {
  const int thr = kRefineWarps * 32;
  // programmatic dependent launches, as on the single-field path
  cudaError_t e = launch_pdl(batch_test_kernel<T>, num_sms * 16, thr, 0, st, fields, cq, rs);
  if (!e) e = launch_pdl(batch_solve_kernel<T>, num_sms * 2, thr, 0, st, fields, cq, rs, sink);
  if (!e) e = launch_pdl(batch_big_kernel<T>, num_sms, thr, 0, st, fields, cq, rs, sink);
  return e ? e : cudaGetLastError();
}

cudaError_t launch_batch_refine_staged(int f64, const BatchField* fields, const CandidateQueue& cq,
                                       const RefineStage& rs, const FeatureSink& sink, int num_sms, cudaStream_t st) {
  return f64 ? launch_batch_refine_t<double>(fields, cq, rs, sink, num_sms, st)
             : launch_batch_refine_t<float>(fields, cq, rs, sink, num_sms, st);
}

int batch_time_chunk(long long lt, int pick) {
  // pick 0: the whole time range per item; otherwise that many steps
  if (pick <= 0 || pick >= lt) return (int)std::max<long long>(1, lt);
  return pick;
}
}  // namespace ftk2b
