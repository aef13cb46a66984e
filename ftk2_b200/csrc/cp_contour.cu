// Level sets of a scalar field on a regular spacetime mesh: the
// SimplicialEngine<T, ContourPredicate<T>> path (execute + get_complex,
// engine.hpp:95-215 and 822-996; ContourPredicate predicate.hpp:135-183;
// marching_pentatope / marching_tetrahedron engine.hpp:1210-1339) as one
// device pipeline:
//
//   ct_sign    one pass over the field: the simulation-of-simplicity sign of
//              value - threshold at every vertex (sos.hpp:12-20), one byte
//   ct_mask    per vertex c, the directions e in {0,1}^d \ 0 whose edge to
//              c + e crosses (the signs differ, origin_inside<1>,
//              sos.hpp:211-220), and per-block counts
//   scan       block offsets.  Every Freudenthal edge joins some c to c + e,
//              so the edges in simplex order are the (c, e) pairs in vertex
//              order with e read as a binary number, x lowest: a feature's
//              rank is its block offset plus a prefix count, no sort needed
//   ct_emit    vertex ids and barycentrics of every feature at its rank
//   ct_first   (2D+t) the position at which the reference's sequential
//              patching first meets each node whose edge starts on an upper
//              boundary face (those are numbered in meeting order, after the
//              first pass's nodes, and 2D+t quads are cut along the diagonal
//              from their smallest-numbered node)
//   ct_cells   marching tetrahedra / pentatopes over every Kuhn simplex of
//              every hypercube: manifold cells, union-find hooks
//   sort       cells into lexicographic order (two stable radix passes)
//   ct_gather  sorted cells, duplicates flagged
//   label      track id = the component's smallest feature index
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>

#include "../../include/ftk2b.h"
#include "cp_api_internal.h"
#include "cp_device.cuh"
#include "cp_post.h"
#include "cp_uf.cuh"

using namespace ftk2b;

namespace {

constexpr int kCtThreads = 256;

struct CtGeom {
  int d;                        // mesh dims: 3 (2D+t) or 4 (3D+t)
  int per_vertex;               // field indexed by global vertex id
  unsigned long long L[4];      // local dims
  unsigned long long as[4];     // array strides of the local coordinates
  unsigned long long gs[4];     // global id strides
  unsigned long long g0;        // global id of the local origin
  unsigned long long nv;        // local vertices
  unsigned long long ncube;     // local hypercubes
  unsigned long long loff[16];  // local linear step to corner e
  unsigned long long goff[16];  // global id step to corner e
  unsigned long long aoff[16];  // array step to corner e
};

__device__ __forceinline__ void ct_coords(const CtGeom& g, unsigned long long i, unsigned long long* c) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k < g.d) {
      c[k] = i % g.L[k];
      i /= g.L[k];
    } else {
      c[k] = 0;
    }
  }
}

__device__ __forceinline__ unsigned long long ct_gid(const CtGeom& g, const unsigned long long* c) {
  unsigned long long v = g.g0;
  for (int k = 0; k < g.d; ++k) v += c[k] * g.gs[k];
  return v;
}

__device__ __forceinline__ unsigned long long ct_aidx(const CtGeom& g, const unsigned long long* c) {
  unsigned long long v = 0;
  for (int k = 0; k < g.d; ++k) v += c[k] * g.as[k];
  return v;
}

template <typename T>
__device__ __forceinline__ T ct_adj(const CtGeom& g, const T* __restrict__ a, unsigned long long aidx,
                                    unsigned long long gid, T thr) {
  const T v = g.per_vertex ? __ldg(a + gid) : __ldg(a + aidx);
  return fp<T>::sub(v, thr);
}

// sos::sign(v, id, Q) > 0: (int)(double(v) * Q + (v > 0 ? 0.5 : -0.5)) is
// positive exactly when the rounded sum is >= 1, negative when <= -1; zero
// goes by the parity of the vertex id.  Multiply and add rounded separately.
template <typename T>
__device__ __forceinline__ bool ct_positive(T adj, unsigned long long gid, double q) {
  const double x = __dadd_rn(__dmul_rn((double)adj, q), adj > T(0) ? 0.5 : -0.5);
  if (x >= 1.0) return true;
  if (x <= -1.0) return false;
  return (gid & 1ull) == 0;
}

template <typename T>
__global__ void ct_sign_kernel(CtGeom g, const T* __restrict__ a, T thr, double q,
                               unsigned char* __restrict__ pos) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < g.nv;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long c[4];
    ct_coords(g, i, c);
    const unsigned long long gid = ct_gid(g, c);
    pos[i] = ct_positive(ct_adj(g, a, ct_aidx(g, c), gid, thr), gid, q) ? 1 : 0;
  }
}

// block-wide exclusive scan of one count per thread; returns the thread's
// prefix, *total the block's sum
__device__ __forceinline__ unsigned ct_block_scan(unsigned v, unsigned* total) {
  __shared__ unsigned wsum[kCtThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    unsigned w = lane < kCtThreads / 32 ? wsum[lane] : 0;
    unsigned wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < kCtThreads / 32) wsum[lane] = wi - w;
    if (lane == kCtThreads / 32 - 1) *total = wi;
  }
  __syncthreads();
  return wsum[warp] + incl - v;
}

__device__ __forceinline__ unsigned ct_inbounds(const CtGeom& g, const unsigned long long* c) {
  unsigned inb = 0;
  for (int k = 0; k < g.d; ++k)
    if (c[k] + 1 < g.L[k]) inb |= 1u << k;
  return inb;
}

__global__ void ct_mask_kernel(CtGeom g, const unsigned char* __restrict__ pos, unsigned short* __restrict__ mask,
                               unsigned* __restrict__ blk, unsigned long long* __restrict__ total64) {
  __shared__ unsigned tot;
  const unsigned long long i = blockIdx.x * (unsigned long long)kCtThreads + threadIdx.x;
  unsigned m = 0;
  if (i < g.nv) {
    unsigned long long c[4];
    ct_coords(g, i, c);
    const unsigned inb = ct_inbounds(g, c);
    const unsigned char p = pos[i];
    const int ne = 1 << g.d;
    for (int e = 1; e < ne; ++e)
      if ((e & ~inb) == 0 && pos[i + g.loff[e]] != p) m |= 1u << (e - 1);
    mask[i] = (unsigned short)m;
  }
  ct_block_scan(__popc(m), &tot);
  if (threadIdx.x == 0) {
    blk[blockIdx.x] = tot;
    atomicAdd(total64, (unsigned long long)tot);  // exact count: the offsets are 32-bit
  }
}

// ZeroCrossingSolver<1,T>::solve (zero_crossing.hpp:93-104) with the
// predicate's fallback to the midpoint (predicate.hpp:149), in T, each
// operation rounded on its own
template <typename T>
__device__ __forceinline__ void ct_solve(T a0, T a1, T* l0, T* l1) {
  using F = fp<T>;
  const T dd = F::sub(a0, a1);
  bool ok = !(F::abs(dd) < T(1e-12));
  T x0 = T(0.5), x1 = T(0.5);
  if (ok) {
    x0 = F::div(-a1, dd);
    x1 = F::sub(T(1.0), x0);
    const T eps = T(1e-9);
    ok = x0 >= -eps && x0 <= F::add(T(1.0), eps);
  }
  *l0 = ok ? x0 : T(0.5);
  *l1 = ok ? x1 : T(0.5);
}

template <typename T>
__global__ void ct_emit_kernel(CtGeom g, const T* __restrict__ a, T thr, const unsigned short* __restrict__ mask,
                               const unsigned* __restrict__ blk_off, unsigned* __restrict__ voff,
                               unsigned long long* __restrict__ simp, double* __restrict__ lam,
                               float* __restrict__ bary) {
  __shared__ unsigned tot;
  const unsigned long long i = blockIdx.x * (unsigned long long)kCtThreads + threadIdx.x;
  const unsigned m = i < g.nv ? mask[i] : 0u;
  const unsigned base = blk_off[blockIdx.x] + ct_block_scan(__popc(m), &tot);
  if (i >= g.nv) return;
  voff[i] = base;
  if (!m) return;
  unsigned long long c[4];
  ct_coords(g, i, c);
  const unsigned long long gid = ct_gid(g, c), ai = ct_aidx(g, c);
  const T a0 = ct_adj(g, a, ai, gid, thr);
  unsigned r = base;
  const int ne = 1 << g.d;
  for (int e = 1; e < ne; ++e) {
    if (!((m >> (e - 1)) & 1u)) continue;
    const T a1 = ct_adj(g, a, ai + g.aoff[e], gid + g.goff[e], thr);
    T l0, l1;
    ct_solve(a0, a1, &l0, &l1);
    simp[2 * (size_t)r] = gid;
    simp[2 * (size_t)r + 1] = gid + g.goff[e];
    lam[2 * (size_t)r] = (double)l0;
    lam[2 * (size_t)r + 1] = (double)l1;
    bary[2 * (size_t)r] = (float)l0;
    bary[2 * (size_t)r + 1] = (float)l1;
    ++r;
  }
}

// Axis order of the p-th Kuhn simplex as the CPU mesh decodes it
// (mesh.hpp:407-409): successive swaps p[i] <-> p[i + j], j = p % (d - i).
__device__ __forceinline__ void ct_perm(int p_idx, int d, int* ax) {
  for (int i = 0; i < 4; ++i) ax[i] = i;
  int t = p_idx;
  for (int i = 0; i < d; ++i) {
    const int j = t % (d - i);
    const int x = ax[i];
    ax[i] = ax[i + j];
    ax[i + j] = x;
    t /= d - i;
  }
}

struct CtCube {
  unsigned long long base;  // local linear index of the hypercube's base vertex
  unsigned long long c[4];
  unsigned sgn;             // bit e: corner e is positive
};

__device__ __forceinline__ bool ct_load_cube(const CtGeom& g, unsigned long long q, const unsigned char* pos,
                                             CtCube* cb) {
  unsigned long long base = 0, r = q, ls = 1;
  for (int k = 0; k < g.d; ++k) {
    const unsigned long long n = g.L[k] - 1;
    cb->c[k] = r % n;
    r /= n;
    base += cb->c[k] * ls;
    ls *= g.L[k];
  }
  cb->base = base;
  unsigned s = 0;
  const int ne = 1 << g.d;
  for (int e = 0; e < ne; ++e) s |= (unsigned)pos[base + g.loff[e]] << e;
  cb->sgn = s;
  return s != 0 && s != (1u << ne) - 1u;  // mixed signs: some edge crosses
}

// feature index of the crossing edge from corner lo to corner hi (lo a subset
// of hi) of the cube
__device__ __forceinline__ unsigned ct_node(const CtGeom& g, const CtCube& cb, const unsigned short* mask,
                                            const unsigned* voff, int lo, int hi) {
  const unsigned long long v = cb.base + g.loff[lo];
  const int dir = hi ^ lo;
  return voff[v] + __popc((unsigned)mask[v] & ((1u << (dir - 1)) - 1u));
}

// the edge from corner lo starts on an upper boundary face (its lower vertex
// is no hypercube base): the reference's first pass does not visit it
__device__ __forceinline__ bool ct_late(const CtGeom& g, const CtCube& cb, int lo) {
  for (int k = 0; k < g.d; ++k)
    if (cb.c[k] + ((lo >> k) & 1) == g.L[k] - 1) return true;
  return false;
}

// The crossing edges of one Kuhn simplex in the order the reference's
// marching functions meet them, as (lower, upper) path positions: a 1-vs-rest
// split pairs the lone vertex with the others in order; otherwise every
// positive vertex with every other vertex, positives outer (2D+t 2-2 split).
// Returns the count (the pentatope 2-3 split is handled by its caller).
__device__ __forceinline__ int ct_lone(int npos, int nvtx, const bool* ps) {
  if (npos == 1) {
    for (int i = 0; i < nvtx; ++i)
      if (ps[i]) return i;
  }
  for (int i = 0; i < nvtx; ++i)
    if (!ps[i]) return i;
  return 0;
}

__global__ void ct_first_kernel(CtGeom g, const unsigned char* __restrict__ pos,
                                const unsigned short* __restrict__ mask, const unsigned* __restrict__ voff,
                                unsigned long long* __restrict__ first) {
  for (unsigned long long q = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; q < g.ncube;
       q += (unsigned long long)gridDim.x * blockDim.x) {
    CtCube cb;
    if (!ct_load_cube(g, q, pos, &cb)) continue;
    for (int p_idx = 0; p_idx < 6; ++p_idx) {
      int ax[4];
      ct_perm(p_idx, 3, ax);
      int pe[4];
      pe[0] = 0;
      for (int i = 0; i < 3; ++i) pe[i + 1] = pe[i] | (1 << ax[i]);
      bool ps[4];
      int npos = 0;
      for (int i = 0; i < 4; ++i) {
        ps[i] = (cb.sgn >> pe[i]) & 1u;
        npos += ps[i];
      }
      if (npos == 0 || npos == 4) continue;
      int lo_i[4], hi_i[4], ne = 0;
      if (npos == 1 || npos == 3) {
        const int lone = ct_lone(npos, 4, ps);
        for (int o = 0; o < 4; ++o) {
          if (o == lone) continue;
          lo_i[ne] = min(lone, o);
          hi_i[ne] = max(lone, o);
          ++ne;
        }
      } else {
        for (int a = 0; a < 4; ++a) {
          if (!ps[a]) continue;
          for (int b = 0; b < 4; ++b) {
            if (ps[b]) continue;
            lo_i[ne] = min(a, b);
            hi_i[ne] = max(a, b);
            ++ne;
          }
        }
      }
      for (int k = 0; k < ne; ++k) {
        const int lo = pe[lo_i[k]], hi = pe[hi_i[k]];
        if (!ct_late(g, cb, lo)) continue;
        const unsigned nd = ct_node(g, cb, mask, voff, lo, hi);
        const unsigned long long key = ((cb.base * 6ull) + (unsigned long long)p_idx) * 4ull + (unsigned long long)k;
        atomicMin(first + nd, key);
      }
    }
  }
}

template <int K>
__device__ __forceinline__ void ct_sort_small(unsigned* v) {
#pragma unroll
  for (int i = 1; i < K; ++i)
#pragma unroll
    for (int j = i; j > 0; --j)
      if (v[j - 1] > v[j]) {
        const unsigned x = v[j - 1];
        v[j - 1] = v[j];
        v[j] = x;
      }
}

template <int K>
__device__ __forceinline__ void ct_put(const unsigned* cell, unsigned* cells, unsigned* cnt, unsigned cap,
                                       unsigned* parent, unsigned* err) {
  unsigned v[K];
#pragma unroll
  for (int i = 0; i < K; ++i) v[i] = cell[i];
  ct_sort_small<K>(v);
  const unsigned slot = atomicAdd(cnt, 1u);
  if (slot < cap) {
#pragma unroll
    for (int i = 0; i < K; ++i) cells[(size_t)slot * K + i] = v[i];
  }
#pragma unroll
  for (int i = 1; i < K; ++i) uf_unite(parent, v[0], v[i], err);
}

__global__ void ct_cells_kernel(CtGeom g, const unsigned char* __restrict__ pos,
                                const unsigned short* __restrict__ mask, const unsigned* __restrict__ voff,
                                const unsigned long long* __restrict__ first, unsigned n, unsigned* __restrict__ cells,
                                unsigned* cnt, unsigned cap, unsigned* parent, unsigned* err) {
  const int d = g.d;
  const int np = d == 3 ? 6 : 24;
  for (unsigned long long q = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; q < g.ncube;
       q += (unsigned long long)gridDim.x * blockDim.x) {
    CtCube cb;
    if (!ct_load_cube(g, q, pos, &cb)) continue;
    for (int p_idx = 0; p_idx < np; ++p_idx) {
      int ax[4];
      ct_perm(p_idx, d, ax);
      int pe[5];
      pe[0] = 0;
      for (int i = 0; i < d; ++i) pe[i + 1] = pe[i] | (1 << ax[i]);
      bool ps[5];
      int npos = 0;
      for (int i = 0; i <= d; ++i) {
        ps[i] = (cb.sgn >> pe[i]) & 1u;
        npos += ps[i];
      }
      if (npos == 0 || npos == d + 1) continue;
      auto node = [&](int i, int j) {
        const int a = min(i, j), b = max(i, j);
        return ct_node(g, cb, mask, voff, pe[a], pe[b]);
      };
      if (npos == 1 || npos == d) {
        const int lone = ct_lone(npos, d + 1, ps);
        unsigned cell[4];
        int k = 0;
        for (int o = 0; o <= d; ++o)
          if (o != lone) cell[k++] = node(lone, o);
        if (d == 3) ct_put<3>(cell, cells, cnt, cap, parent, err);
        else ct_put<4>(cell, cells, cnt, cap, parent, err);
      } else if (d == 3) {
        // 2-2 split: the quad of the four crossing edges, cut along the
        // diagonal from its node the reference numbered first
        unsigned nd[4];
        unsigned long long key[4];
        int k = 0;
        for (int a = 0; a < 4; ++a) {
          if (!ps[a]) continue;
          for (int b = 0; b < 4; ++b) {
            if (ps[b]) continue;
            nd[k] = node(a, b);
            const unsigned long long f = first[nd[k]];
            key[k] = f == ~0ull ? (unsigned long long)nd[k] : (unsigned long long)n + f;
            ++k;
          }
        }
        for (int i = 1; i < 4; ++i)
          for (int j = i; j > 0 && key[j - 1] > key[j]; --j) {
            const unsigned long long kx = key[j - 1];
            key[j - 1] = key[j];
            key[j] = kx;
            const unsigned nx = nd[j - 1];
            nd[j - 1] = nd[j];
            nd[j] = nx;
          }
        const unsigned t1[3] = {nd[0], nd[1], nd[2]};
        const unsigned t2[3] = {nd[0], nd[2], nd[3]};
        ct_put<3>(t1, cells, cnt, cap, parent, err);
        ct_put<3>(t2, cells, cnt, cap, parent, err);
      } else {
        // pentatope 2-3 split: T0 / T1 = crossing edges from the pair's first /
        // second vertex to the triple, in order; three tets
        const bool two_pos = npos == 2;
        int two[2], three[3], n2 = 0, n3 = 0;
        for (int i = 0; i < 5; ++i) {
          if (ps[i] == two_pos) two[n2++] = i;
          else three[n3++] = i;
        }
        unsigned T0[3], T1[3];
        for (int t = 0; t < 3; ++t) {
          T0[t] = node(two[0], three[t]);
          T1[t] = node(two[1], three[t]);
        }
        const unsigned c0[4] = {T0[0], T0[1], T0[2], T1[2]};
        const unsigned c1[4] = {T0[0], T0[1], T1[1], T1[2]};
        const unsigned c2[4] = {T0[0], T1[0], T1[1], T1[2]};
        ct_put<4>(c0, cells, cnt, cap, parent, err);
        ct_put<4>(c1, cells, cnt, cap, parent, err);
        ct_put<4>(c2, cells, cnt, cap, parent, err);
      }
    }
  }
}

__global__ void ct_iota_kernel(unsigned* __restrict__ v, unsigned n) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

__global__ void ct_fill_u64_kernel(unsigned long long* __restrict__ v, unsigned long long x, unsigned n) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = x;
}

// sort keys: pass 0 the last two entries (k-2, k-1) of each cell, pass 1 the
// leading ones (entry 0 of a triangle, entries 0 and 1 of a tet), read through
// the permutation of pass 0
__global__ void ct_key_kernel(const unsigned* __restrict__ cells, const unsigned* cnt_ptr, unsigned cap, int k,
                              unsigned long long n, int pass, const unsigned* __restrict__ perm_in,
                              unsigned long long* __restrict__ key, unsigned* __restrict__ val) {
  const unsigned m = min(*cnt_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const unsigned src = pass == 0 ? i : perm_in[i];
    const unsigned* c = cells + (size_t)src * k;
    if (pass == 0) key[i] = (unsigned long long)c[k - 2] * n + c[k - 1];
    else key[i] = k == 3 ? (unsigned long long)c[0] : (unsigned long long)c[0] * n + c[1];
    val[i] = src;
  }
}

__global__ void ct_gather_kernel(const unsigned* __restrict__ cells, const unsigned* __restrict__ perm,
                                 const unsigned* cnt_ptr, unsigned cap, int k, unsigned* __restrict__ out,
                                 unsigned* err) {
  const unsigned m = min(*cnt_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const unsigned* c = cells + (size_t)perm[i] * k;
    bool same = i > 0;
    const unsigned* p = i > 0 ? cells + (size_t)perm[i - 1] * k : c;
    for (int j = 0; j < k; ++j) {
      out[(size_t)i * k + j] = c[j];
      same = same && p[j] == c[j];
    }
    if (same) atomicOr(err, 2u);
  }
}

int bitlen(unsigned long long x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b < 1 ? 1 : b;
}

unsigned grid_of(unsigned long long work, int threads, unsigned long long max_blocks) {
  unsigned long long b = (work + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (unsigned)b;
}

ftk2b_status cfail(ftk2b_ctx* ctx, ftk2b_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  ctx->err = buf;
  return st;
}

#define C_TRY(call)                                                                             \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return cfail(ctx, e_ == cudaErrorMemoryAllocation ? FTK2B_OOM : FTK2B_CUDA_ERROR,          \
                   "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

enum {
  kBufField = 0, kBufPos, kBufMask, kBufBlk, kBufVoff, kBufSimp, kBufLam, kBufBary, kBufFirst, kBufParent,
  kBufCells, kBufKey0, kBufKey1, kBufVal0, kBufVal1, kBufHist, kBufCellsOut, kBufTrack, kBufCount
};

template <typename T>
ftk2b_status run_contour(ftk2b_ctx* ctx, const CtGeom& g, const void* field, T thr, double q,
                         ftk2b_contour_result* res) {
  cudaStream_t st = ctx->stream;
  DevBuf* B = ctx->contour;
  const int d = g.d;
  const unsigned long long nblk = (g.nv + kCtThreads - 1) / kCtThreads;
  C_TRY(B[kBufPos].ensure(g.nv));
  C_TRY(B[kBufMask].ensure(2 * g.nv));
  C_TRY(B[kBufVoff].ensure(4 * g.nv));
  C_TRY(B[kBufBlk].ensure(4 * (nblk + 1)));
  C_TRY(B[kBufCount].ensure(64));
  auto* pos = static_cast<unsigned char*>(B[kBufPos].p);
  auto* mask = static_cast<unsigned short*>(B[kBufMask].p);
  auto* voff = static_cast<unsigned*>(B[kBufVoff].p);
  auto* blk = static_cast<unsigned*>(B[kBufBlk].p);
  auto* counts = static_cast<unsigned*>(B[kBufCount].p);  // [0] n, [1] cells, [2] roots, [3] err
  auto* total64 = reinterpret_cast<unsigned long long*>(counts + 8);
  const T* a = static_cast<const T*>(field);
  const unsigned sms = (unsigned)ctx->num_sms;

  C_TRY(cudaMemsetAsync(counts, 0, 64, st));
  C_TRY(cudaEventRecord(ctx->ev0, st));
  ct_sign_kernel<T><<<grid_of(g.nv, 256, 32ull * sms), 256, 0, st>>>(g, a, thr, q, pos);
  ct_mask_kernel<<<(unsigned)nblk, kCtThreads, 0, st>>>(g, pos, mask, blk, total64);
  C_TRY(launch_scan(blk, (unsigned)nblk, counts + 0, nullptr, st));
  ctx->launches += 3;
  unsigned long long n64 = 0;
  C_TRY(cudaMemcpyAsync(&n64, total64, 8, cudaMemcpyDeviceToHost, st));
  C_TRY(ctx->sync());
  // features are indexed with 32 bits
  if (n64 >= 0xFFFFFFF0ull) return cfail(ctx, FTK2B_UNSUPPORTED, "more than 2^32 - 16 crossing edges");
  const unsigned n = (unsigned)n64;
  const size_t ncap = n ? n : 1;
  C_TRY(B[kBufSimp].ensure(16 * ncap));
  C_TRY(B[kBufLam].ensure(16 * ncap));
  C_TRY(B[kBufBary].ensure(8 * ncap));
  C_TRY(B[kBufParent].ensure(4 * ncap));
  C_TRY(B[kBufTrack].ensure(8 * ncap));
  if (d == 3) C_TRY(B[kBufFirst].ensure(8 * ncap));
  auto* simp = static_cast<unsigned long long*>(B[kBufSimp].p);
  auto* lam = static_cast<double*>(B[kBufLam].p);
  auto* bary = static_cast<float*>(B[kBufBary].p);
  auto* parent = static_cast<unsigned*>(B[kBufParent].p);
  auto* track = static_cast<unsigned long long*>(B[kBufTrack].p);
  auto* first = d == 3 ? static_cast<unsigned long long*>(B[kBufFirst].p) : nullptr;
  ct_emit_kernel<T><<<(unsigned)nblk, kCtThreads, 0, st>>>(g, a, thr, mask, blk, voff, simp, lam, bary);
  ctx->launches += 1;
  if (d == 3 && n) {
    ct_fill_u64_kernel<<<grid_of(n, 256, 8ull * sms), 256, 0, st>>>(first, ~0ull, n);
    ct_first_kernel<<<grid_of(g.ncube, 256, 64ull * sms), 256, 0, st>>>(g, pos, mask, voff, first);
    ctx->launches += 2;
  }

  // manifold cells: a few per feature (about 2 per node on 2D+t, 4 to 6 on
  // 3D+t), grown once to the exact count if short
  unsigned cap = (unsigned)std::min<unsigned long long>(
      0x7FFFFFFFull, std::max<unsigned long long>(1024ull, (d == 4 ? 8ull : 4ull) * n));
  unsigned ncell = 0;
  const int kc = d;  // entries per cell: 3 (triangles) or 4 (tets)
  for (int attempt = 0; attempt < 2; ++attempt) {
    C_TRY(B[kBufCells].ensure((size_t)4 * kc * cap));
    auto* cells = static_cast<unsigned*>(B[kBufCells].p);
    C_TRY(cudaMemsetAsync(counts + 1, 0, 12, st));
    if (n) ct_iota_kernel<<<grid_of(n, 256, 8ull * sms), 256, 0, st>>>(parent, n);
    ct_cells_kernel<<<grid_of(g.ncube, 256, 64ull * sms), 256, 0, st>>>(g, pos, mask, voff, first, n, cells,
                                                                        counts + 1, cap, parent, counts + 3);
    ctx->launches += 2;
    C_TRY(cudaMemcpyAsync(&ncell, counts + 1, 4, cudaMemcpyDeviceToHost, st));
    C_TRY(ctx->sync());
    if (ncell <= cap) break;
    if (ncell >= 0x7FFFFFFFu) return cfail(ctx, FTK2B_UNSUPPORTED, "more than 2^31 manifold cells");
    cap = ncell;
  }
  auto* cells = static_cast<unsigned*>(B[kBufCells].p);

  // lexicographic order of the cells: a stable pass on the trailing pair,
  // then one on the leading entry (or pair)
  const unsigned ccap = ncell ? ncell : 1;
  const int grid = ctx->sort_grid(ccap);
  C_TRY(B[kBufKey0].ensure(8ull * ccap));
  C_TRY(B[kBufKey1].ensure(8ull * ccap));
  C_TRY(B[kBufVal0].ensure(4ull * ccap));
  C_TRY(B[kBufVal1].ensure(4ull * ccap));
  C_TRY(B[kBufHist].ensure(4ull * 256 * grid));
  C_TRY(B[kBufCellsOut].ensure(4ull * kc * ccap));
  auto* k0 = static_cast<unsigned long long*>(B[kBufKey0].p);
  auto* k1 = static_cast<unsigned long long*>(B[kBufKey1].p);
  auto* v0 = static_cast<unsigned*>(B[kBufVal0].p);
  auto* v1 = static_cast<unsigned*>(B[kBufVal1].p);
  auto* hist = static_cast<unsigned*>(B[kBufHist].p);
  auto* cells_out = static_cast<unsigned*>(B[kBufCellsOut].p);
  const unsigned long long nn = n ? n : 1;
  const int bits_pair = bitlen(nn * nn - 1);
  const unsigned cg = grid_of(ccap, 256, 8ull * sms);
  const unsigned* perm = nullptr;
  if (ncell) {
    ct_key_kernel<<<cg, 256, 0, st>>>(cells, counts + 1, cap, kc, nn, 0, nullptr, k0, v0);
    const bool alt0 = radix_sort(k0, v0, k1, v1, counts + 1, ccap, bits_pair, hist, grid, st, &ctx->launches);
    const unsigned* perm0 = alt0 ? v1 : v0;
    // pass 1 reads pass 0's permutation into the other value buffer's pair
    unsigned long long* kk = alt0 ? k0 : k1;
    unsigned* vv = alt0 ? v0 : v1;
    unsigned long long* kk2 = alt0 ? k1 : k0;
    unsigned* vv2 = alt0 ? v1 : v0;
    ct_key_kernel<<<cg, 256, 0, st>>>(cells, counts + 1, cap, kc, nn, 1, perm0, kk, vv);
    const int bits1 = kc == 3 ? bitlen(nn - 1) : bits_pair;
    const bool alt1 = radix_sort(kk, vv, kk2, vv2, counts + 1, ccap, bits1, hist, grid, st, &ctx->launches);
    perm = alt1 ? vv2 : vv;
    ct_gather_kernel<<<cg, 256, 0, st>>>(cells, perm, counts + 1, cap, kc, cells_out, counts + 3);
    ctx->launches += 3;
  }
  if (n) {
    C_TRY(launch_uf_label(parent, counts + 0, n, track, counts + 2, st));
    ctx->launches += 1;
  }
  C_TRY(cudaEventRecord(ctx->ev1, st));

  // results to the host
  unsigned hc[4] = {0, 0, 0, 0};
  C_TRY(cudaMemcpyAsync(hc, counts, 16, cudaMemcpyDeviceToHost, st));
  res->n_features = n;
  res->cell_dim = d - 1;
  res->n_cells = ncell;
  res->simplices = static_cast<uint64_t*>(std::malloc(16 * ncap));
  res->lambda = static_cast<double*>(std::malloc(16 * ncap));
  res->barycentric = static_cast<float*>(std::malloc(8 * ncap));
  res->track_id = static_cast<uint64_t*>(std::malloc(8 * ncap));
  res->scalar = static_cast<float*>(std::malloc(4 * ncap));
  res->cells = static_cast<uint32_t*>(std::malloc(4ull * kc * ccap));
  if (!res->simplices || !res->lambda || !res->barycentric || !res->track_id || !res->scalar || !res->cells)
    return cfail(ctx, FTK2B_OOM, "host result allocation failed");
  if (n) {
    C_TRY(cudaMemcpyAsync(res->simplices, simp, 16ull * n, cudaMemcpyDeviceToHost, st));
    C_TRY(cudaMemcpyAsync(res->lambda, lam, 16ull * n, cudaMemcpyDeviceToHost, st));
    C_TRY(cudaMemcpyAsync(res->barycentric, bary, 8ull * n, cudaMemcpyDeviceToHost, st));
    C_TRY(cudaMemcpyAsync(res->track_id, track, 8ull * n, cudaMemcpyDeviceToHost, st));
  }
  if (ncell) C_TRY(cudaMemcpyAsync(res->cells, cells_out, 4ull * kc * ncell, cudaMemcpyDeviceToHost, st));
  C_TRY(ctx->sync());
  if (hc[3] & 1u) return cfail(ctx, FTK2B_CUDA_ERROR, "union-find did not settle");
  if (hc[3] & 2u) return cfail(ctx, FTK2B_CUDA_ERROR, "duplicate manifold cell");
  const float sc = (float)thr;
  for (unsigned i = 0; i < n; ++i) res->scalar[i] = sc;
  res->n_tracks = hc[2];
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  res->device_ms = ms;
  return FTK2B_OK;
}

}  // namespace

extern "C" ftk2b_status ftk2b_contour_extract(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                                              const ftk2b_field_desc* field, double threshold, double sos_q,
                                              ftk2b_contour_result** out) {
  if (!ctx) return FTK2B_INVALID_ARG;
  if (!mesh || !field || !out) return cfail(ctx, FTK2B_INVALID_ARG, "null argument");
  *out = nullptr;
  if (mesh->kind != FTK2B_MESH_REGULAR) return cfail(ctx, FTK2B_UNSUPPORTED, "level sets need a regular mesh");
  const int d = mesh->ndims;
  if (d != 3 && d != 4) return cfail(ctx, FTK2B_UNSUPPORTED, "regular meshes have 3 or 4 dims (got %d)", d);
  if (field->dtype != FTK2B_F32 && field->dtype != FTK2B_F64)
    return cfail(ctx, FTK2B_INVALID_ARG, "dtype must be FTK2B_F32 or FTK2B_F64");
  if (field->ncomp != 1 || field->layout != FTK2B_LAYOUT_SEPARATE || !field->comp[0])
    return cfail(ctx, FTK2B_INVALID_ARG, "level sets read one scalar array (ncomp 1, layout SEPARATE)");
  if (!(sos_q > 0)) return cfail(ctx, FTK2B_INVALID_ARG, "sos_q must be positive");
  CtGeom g;
  std::memset(&g, 0, sizeof(g));
  g.d = d;
  unsigned long long nv = 1, ncube = 1, gstride = 1;
  for (int k = 0; k < d; ++k) {
    const unsigned long long L = mesh->local_dims[k], G = mesh->global_dims[k], O = mesh->offset[k];
    if (L < 1) return cfail(ctx, FTK2B_INVALID_ARG, "local dim %d is 0", k);
    if (G < O + L) return cfail(ctx, FTK2B_INVALID_ARG, "dim %d: offset + local exceeds the global dim", k);
    g.L[k] = L;
    g.gs[k] = gstride;
    g.g0 += O * gstride;
    gstride *= G;
    nv *= L;
    ncube *= L - 1;
  }
  g.nv = nv;
  g.ncube = ncube;
  const size_t es = field->dtype == FTK2B_F64 ? 8 : 4;
  size_t nelem = 1;
  if (field->nd == 1) {
    g.per_vertex = 1;
    nelem = field->dims[0];
    if (nelem < gstride) return cfail(ctx, FTK2B_INVALID_ARG, "per-vertex array shorter than the global vertex count");
  } else {
    if (field->nd != d) return cfail(ctx, FTK2B_INVALID_ARG, "the scalar array needs nd == mesh dims (or 1)");
    unsigned long long s = 1;
    for (int k = 0; k < d; ++k) {
      if (field->dims[k] < g.L[k]) return cfail(ctx, FTK2B_INVALID_ARG, "array dim %d smaller than the local dim", k);
      g.as[k] = s;
      s *= field->dims[k];
    }
    nelem = s;
  }
  if (nv >= (1ull << 40)) return cfail(ctx, FTK2B_UNSUPPORTED, "mesh too large");
  unsigned long long ls = 1, lstr[4] = {0, 0, 0, 0};
  for (int k = 0; k < d; ++k) {
    lstr[k] = ls;
    ls *= g.L[k];
  }
  for (int e = 0; e < (1 << d); ++e)
    for (int k = 0; k < d; ++k)
      if ((e >> k) & 1) {
        g.loff[e] += lstr[k];
        g.goff[e] += g.gs[k];
        g.aoff[e] += g.as[k];
      }
  if (cudaSetDevice(ctx->device) != cudaSuccess) return cfail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  const void* dev = field->comp[0];
  if (field->location != FTK2B_DEVICE) {
    C_TRY(ctx->contour[kBufField].ensure(nelem * es));
    C_TRY(cudaMemcpyAsync(ctx->contour[kBufField].p, field->comp[0], nelem * es, cudaMemcpyHostToDevice,
                          ctx->stream));
    dev = ctx->contour[kBufField].p;
  }
  auto* res = new (std::nothrow) ftk2b_contour_result;
  if (!res) return cfail(ctx, FTK2B_OOM, "result allocation failed");
  std::memset(res, 0, sizeof(*res));
  unsigned long long edges = 0;
  for (int e = 1; e < (1 << d); ++e) {
    unsigned long long c = 1;
    for (int k = 0; k < d; ++k) c *= ((e >> k) & 1) ? g.L[k] - 1 : g.L[k];
    edges += c;
  }
  res->n_simplices = edges;
  const ftk2b_status st =
      field->dtype == FTK2B_F64
          ? run_contour<double>(ctx, g, dev, (double)threshold, sos_q, res)
          : run_contour<float>(ctx, g, dev, (float)threshold, sos_q, res);
  if (st != FTK2B_OK) {
    ftk2b_contour_result_free(res);
    return st;
  }
  *out = res;
  return FTK2B_OK;
}

extern "C" void ftk2b_contour_result_free(ftk2b_contour_result* r) {
  if (!r) return;
  std::free(r->simplices);
  std::free(r->lambda);
  std::free(r->barycentric);
  std::free(r->track_id);
  std::free(r->scalar);
  std::free(r->cells);
  delete r;
}
