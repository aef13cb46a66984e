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
//   buckets    cells into lexicographic order: counted and scattered by
//              their leading node, each bucket's few rows sorted, duplicates
//              flagged
//   label      track id = the component's smallest feature index
#include <sys/mman.h>

#include <algorithm>
#include <array>
#include <vector>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
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
  unsigned long long lstr[4];   // local linear strides
  unsigned char perm[24][4];    // axis order of the p-th Kuhn simplex (CPU mesh order)
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

// Mixed hypercubes (corner signs not all equal) are listed once, each as one
// word: base vertex (local linear index) << 20 | upper-face axes << 16 |
// corner signs (bit e: corner e positive).  An upper-face axis k is one where
// the cube's corners with bit k set lie on the mesh's last layer (c_k = L_k - 2).
constexpr int kCtBaseShift = 20;

__global__ void ct_mixed_kernel(CtGeom g, const unsigned char* __restrict__ pos,
                                unsigned long long* __restrict__ list, unsigned* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int ne = 1 << g.d;
  for (unsigned long long q0 = blockIdx.x * (unsigned long long)blockDim.x; q0 < g.ncube;
       q0 += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long q = q0 + threadIdx.x;
    unsigned long long word = 0;
    bool mixed = false;
    if (q < g.ncube) {
      unsigned long long base = 0, r = q;
      unsigned upper = 0;
      for (int k = 0; k < g.d; ++k) {
        const unsigned long long n = g.L[k] - 1, c = r % n;
        r /= n;
        base += c * g.lstr[k];
        if (c + 2 == g.L[k]) upper |= 1u << k;
      }
      unsigned sgn = 0;
      for (int e = 0; e < ne; ++e) sgn |= (unsigned)pos[base + g.loff[e]] << e;
      mixed = sgn != 0 && sgn != (1u << ne) - 1u;
      word = (base << kCtBaseShift) | ((unsigned long long)upper << 16) | sgn;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, mixed);
    unsigned wbase = 0;
    if (lane == 0 && bal) wbase = atomicAdd(cnt, (unsigned)__popc(bal));
    wbase = __shfl_sync(0xffffffffu, wbase, 0);
    if (mixed) list[wbase + __popc(bal & ((1u << lane) - 1u))] = word;
  }
}

// One Kuhn simplex of a listed cube, for the lane that owns it: path corners
// (corner bit masks along the CPU mesh's permutation order) and signs.
struct CtSimplex {
  int pe[5];      // corner of path vertex i
  unsigned ps;    // bit i: path vertex i positive
  int npos;
};

__device__ __forceinline__ void ct_simplex(const CtGeom& g, unsigned sgn, int p_idx, CtSimplex* x) {
  x->pe[0] = 0;
  x->ps = sgn & 1u;
  x->npos = (int)(sgn & 1u);
  for (int i = 0; i < g.d; ++i) {
    x->pe[i + 1] = x->pe[i] | (1 << g.perm[p_idx][i]);
    const unsigned b = (sgn >> x->pe[i + 1]) & 1u;
    x->ps |= b << (i + 1);
    x->npos += (int)b;
  }
}

// feature index of the crossing edge from path vertex a to path vertex b of
// the cube at local vertex base
__device__ __forceinline__ unsigned ct_node(const CtGeom& g, unsigned long long base, const CtSimplex& x,
                                            const unsigned short* __restrict__ mask,
                                            const unsigned* __restrict__ voff, int a, int b) {
  const int lo = x.pe[min(a, b)], hi = x.pe[max(a, b)];
  const unsigned long long v = base + g.loff[lo];
  const int dir = hi ^ lo;
  return __ldg(voff + v) + __popc((unsigned)__ldg(mask + v) & ((1u << (dir - 1)) - 1u));
}

// The crossing edges of a 1-vs-rest or 2D+t 2-2 split in the order the
// reference's marching functions meet them, as path-vertex pairs: the lone
// vertex with the others in order; positives outer, others inner.
__device__ __forceinline__ int ct_crossings(const CtSimplex& x, int nvtx, int* ea, int* eb) {
  int ne = 0;
  if (x.npos == 1 || x.npos == nvtx - 1) {
    const bool lone_pos = x.npos == 1;
    int lone = 0;
    for (int i = 0; i < nvtx; ++i)
      if ((((x.ps >> i) & 1u) != 0) == lone_pos) lone = i;
    for (int o = 0; o < nvtx; ++o)
      if (o != lone) {
        ea[ne] = lone;
        eb[ne] = o;
        ++ne;
      }
  } else {
    for (int a = 0; a < nvtx; ++a) {
      if (!((x.ps >> a) & 1u)) continue;
      for (int b = 0; b < nvtx; ++b) {
        if ((x.ps >> b) & 1u) continue;
        ea[ne] = a;
        eb[ne] = b;
        ++ne;
      }
    }
  }
  return ne;
}

// lanes of a warp: np lanes per listed cube (one per Kuhn simplex), 32 / np
// cubes per warp
struct CtLane {
  int np, per, sub, p_idx;
  bool active;
};

__device__ __forceinline__ CtLane ct_lane(int d) {
  CtLane l;
  const int lane = threadIdx.x & 31;
  l.np = d == 3 ? 6 : 24;
  l.per = 32 / l.np;
  l.sub = lane / l.np;
  l.p_idx = lane % l.np;
  l.active = l.sub < l.per;
  return l;
}

// (2D+t) where the reference's sequential patching first meets each node whose
// edge starts on an upper boundary face: (cube base, permutation index,
// position in the marching enumeration), minimised over every meeting
__global__ void ct_first_kernel(CtGeom g, const unsigned long long* __restrict__ list, const unsigned* list_cnt,
                                const unsigned short* __restrict__ mask, const unsigned* __restrict__ voff,
                                unsigned long long* __restrict__ first) {
  const CtLane ln = ct_lane(3);
  const unsigned nl = *list_cnt;
  const unsigned long long warp = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long it = warp * ln.per + ln.sub; ln.active && it < nl; it += nwarps * ln.per) {
    const unsigned long long w = list[it];
    const unsigned long long base = w >> kCtBaseShift;
    const unsigned upper = (unsigned)(w >> 16) & 0xFu, sgn = (unsigned)w & 0xFFFFu;
    CtSimplex x;
    ct_simplex(g, sgn, ln.p_idx, &x);
    if (x.npos == 0 || x.npos == 4) continue;
    int ea[4], eb[4];
    const int ne = ct_crossings(x, 4, ea, eb);
    for (int k = 0; k < ne; ++k) {
      const int lo = x.pe[min(ea[k], eb[k])];
      if (!(lo & (int)upper)) continue;  // the edge starts at a hypercube base
      const unsigned nd = ct_node(g, base, x, mask, voff, ea[k], eb[k]);
      const unsigned long long key = ((base * 6ull) + (unsigned long long)ln.p_idx) * 4ull + (unsigned long long)k;
      atomicMin(first + nd, key);
    }
  }
}

__device__ __forceinline__ void ct_sort4(unsigned* v, int k) {
  for (int i = 1; i < k; ++i)
    for (int j = i; j > 0 && v[j - 1] > v[j]; --j) {
      const unsigned x = v[j - 1];
      v[j - 1] = v[j];
      v[j] = x;
    }
}

// Marching tetrahedra (2D+t) / pentatopes (3D+t) on the listed cubes, one
// Kuhn simplex per lane: up to three cells each, slots reserved per warp;
// the simplex's crossing nodes are joined in the union-find by a star from its
// first node (the same components as joining every cell's nodes).
__global__ void ct_cells_kernel(CtGeom g, const unsigned long long* __restrict__ list, const unsigned* list_cnt,
                                const unsigned short* __restrict__ mask, const unsigned* __restrict__ voff,
                                const unsigned long long* __restrict__ first, unsigned n,
                                unsigned* __restrict__ cells, unsigned long long* cnt, unsigned cap,
                                unsigned* parent,
                                unsigned* err) {
  const int d = g.d;
  const int kc = d;  // entries per cell
  const CtLane ln = ct_lane(d);
  const int lane = threadIdx.x & 31;
  const unsigned nl = *list_cnt;
  const unsigned long long warp = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long it0 = warp * ln.per; it0 < nl; it0 += nwarps * ln.per) {
    const unsigned long long it = it0 + ln.sub;
    unsigned cell[3][4];
    unsigned nodes[6];
    int nn = 0, ncell = 0;
    if (ln.active && it < nl) {
      const unsigned long long w = list[it];
      const unsigned long long base = w >> kCtBaseShift;
      CtSimplex x;
      ct_simplex(g, (unsigned)w & 0xFFFFu, ln.p_idx, &x);
      if (x.npos != 0 && x.npos != d + 1) {
        if (x.npos == 1 || x.npos == d || d == 3) {
          int ea[6], eb[6];
          const int ne = ct_crossings(x, d + 1, ea, eb);
          for (int k = 0; k < ne; ++k) nodes[k] = ct_node(g, base, x, mask, voff, ea[k], eb[k]);
          nn = ne;
          if (ne == d) {  // 1-vs-rest: one cell
            for (int k = 0; k < d; ++k) cell[0][k] = nodes[k];
            ncell = 1;
          } else {  // 2D+t 2-2 split: the quad cut along the diagonal from the
                    // node the reference numbered first
            unsigned nd[4];
            unsigned long long key[4];
            for (int k = 0; k < 4; ++k) {
              nd[k] = nodes[k];
              const unsigned long long f = first[nd[k]];
              key[k] = f == ~0ull ? (unsigned long long)nd[k] : (unsigned long long)n + f;
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
            cell[0][0] = nd[0], cell[0][1] = nd[1], cell[0][2] = nd[2];
            cell[1][0] = nd[0], cell[1][1] = nd[2], cell[1][2] = nd[3];
            ncell = 2;
          }
        } else {  // pentatope 2-3 split
          const bool two_pos = x.npos == 2;
          int two[2], three[3], n2 = 0, n3 = 0;
          for (int i = 0; i < 5; ++i) {
            if ((((x.ps >> i) & 1u) != 0) == two_pos) two[n2++] = i;
            else three[n3++] = i;
          }
          unsigned T0[3], T1[3];
          for (int t = 0; t < 3; ++t) {
            T0[t] = ct_node(g, base, x, mask, voff, two[0], three[t]);
            T1[t] = ct_node(g, base, x, mask, voff, two[1], three[t]);
          }
          cell[0][0] = T0[0], cell[0][1] = T0[1], cell[0][2] = T0[2], cell[0][3] = T1[2];
          cell[1][0] = T0[0], cell[1][1] = T0[1], cell[1][2] = T1[1], cell[1][3] = T1[2];
          cell[2][0] = T0[0], cell[2][1] = T1[0], cell[2][2] = T1[1], cell[2][3] = T1[2];
          for (int t = 0; t < 3; ++t) nodes[t] = T0[t], nodes[3 + t] = T1[t];
          nn = 6;
          ncell = 3;
        }
      }
    }
    // slots for the warp's cells
    unsigned incl = (unsigned)ncell;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const unsigned wtot = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long wbase = 0;
    if (lane == 31 && wtot) wbase = atomicAdd(cnt, (unsigned long long)wtot);
    wbase = __shfl_sync(0xffffffffu, wbase, 31);
    unsigned long long slot = wbase + incl - (unsigned)ncell;
    for (int c = 0; c < ncell; ++c, ++slot) {
      ct_sort4(cell[c], kc);
      if (slot < cap)
        for (int k = 0; k < kc; ++k) cells[(size_t)slot * kc + k] = cell[c][k];
    }
    for (int k = 1; k < nn; ++k) uf_unite(parent, nodes[0], nodes[k], err);
  }
}

__global__ void ct_iota_kernel(unsigned* __restrict__ v, unsigned n) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

__global__ void ct_fill_u64_kernel(unsigned long long* __restrict__ v, unsigned long long x, unsigned n) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = x;
}

// Lexicographic order of the cells.  Each row is sorted, so the rows fall
// into buckets by their leading node: counts per leading node, a scan, a
// scatter into the buckets, then a small sort of each bucket's rows (a few
// rows: the cells at one crossing edge).
__global__ void ct_bucket_count_kernel(const unsigned* __restrict__ cells, unsigned m, int k,
                                       unsigned* __restrict__ bcount) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    atomicAdd(bcount + cells[(size_t)i * k], 1u);
}

__global__ void ct_bucket_scatter_kernel(const unsigned* __restrict__ cells, unsigned m, int k,
                                         const unsigned* __restrict__ boff, unsigned* __restrict__ bcur,
                                         unsigned* __restrict__ out) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const unsigned* c = cells + (size_t)i * k;
    const unsigned a = c[0];
    const unsigned dst = boff[a] + atomicAdd(bcur + a, 1u);
    for (int j = 0; j < k; ++j) out[(size_t)dst * k + j] = c[j];
  }
}

__device__ __forceinline__ bool ct_row_less(const unsigned* x, const unsigned* y, int k) {
  for (int j = 1; j < k; ++j)
    if (x[j] != y[j]) return x[j] < y[j];
  return false;
}

// one thread per leading node: insertion sort of its bucket's rows by their
// remaining entries.  Without uniq, equal neighbours (duplicate cells) raise
// bit 1 of *err; with uniq, they are dropped (the unique rows stay at the
// start of the bucket, their count in uniq[a]).
__global__ void ct_bucket_sort_kernel(unsigned* __restrict__ rows, const unsigned* __restrict__ boff, unsigned n,
                                      int k, unsigned* err, unsigned* __restrict__ uniq) {
  for (unsigned a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const unsigned lo = boff[a], hi = boff[a + 1];
    for (unsigned i = lo + 1; i < hi; ++i) {
      unsigned cur[4];
      for (int j = 0; j < k; ++j) cur[j] = rows[(size_t)i * k + j];
      unsigned p = i;
      while (p > lo && ct_row_less(cur, rows + (size_t)(p - 1) * k, k)) {
        for (int j = 0; j < k; ++j) rows[(size_t)p * k + j] = rows[(size_t)(p - 1) * k + j];
        --p;
      }
      for (int j = 0; j < k; ++j) rows[(size_t)p * k + j] = cur[j];
    }
    if (!uniq) {
      for (unsigned i = lo + 1; i < hi; ++i)
        if (!ct_row_less(rows + (size_t)(i - 1) * k, rows + (size_t)i * k, k)) atomicOr(err, 2u);
    } else {
      unsigned w = lo;
      for (unsigned i = lo; i < hi; ++i) {
        if (i > lo && !ct_row_less(rows + (size_t)(w - 1) * k, rows + (size_t)i * k, k)) continue;
        if (w != i)
          for (int j = 0; j < k; ++j) rows[(size_t)w * k + j] = rows[(size_t)i * k + j];
        ++w;
      }
      uniq[a] = w - lo;
    }
  }
}

// unique rows of every bucket to their place in the output (uoff: scanned
// unique counts)
__global__ void ct_bucket_compact_kernel(const unsigned* __restrict__ rows, const unsigned* __restrict__ boff,
                                         const unsigned* __restrict__ uoff, unsigned n, int k,
                                         unsigned* __restrict__ out) {
  for (unsigned a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const unsigned lo = boff[a], cnt = uoff[a + 1] - uoff[a], dst = uoff[a];
    for (unsigned i = 0; i < cnt; ++i)
      for (int j = 0; j < k; ++j) out[(size_t)(dst + i) * k + j] = rows[(size_t)(lo + i) * k + j];
  }
}

// Exclusive scan of n counters in place (n up to 2^32 - 1): per-block scans
// of 2048 entries with their totals, a scan of the totals, the block offsets
// added back.
constexpr int kScanPer = 8;  // entries per thread
__global__ void ct_scan_blocks_kernel(unsigned* __restrict__ a, unsigned n, unsigned* __restrict__ tot) {
  __shared__ unsigned btot;
  const unsigned long long b0 = (unsigned long long)blockIdx.x * kCtThreads * kScanPer;
  const unsigned long long t0 = b0 + (unsigned long long)threadIdx.x * kScanPer;
  unsigned v[kScanPer], sum = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    v[j] = t0 + j < n ? a[t0 + j] : 0u;
    sum += v[j];
  }
  unsigned run = ct_block_scan(sum, &btot);
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    if (t0 + j < n) a[t0 + j] = run;
    run += v[j];
  }
  if (threadIdx.x == 0) tot[blockIdx.x] = btot;
}

__global__ void ct_scan_add_kernel(unsigned* __restrict__ a, unsigned n, const unsigned* __restrict__ tot) {
  const unsigned long long b0 = (unsigned long long)blockIdx.x * kCtThreads * kScanPer;
  const unsigned add = tot[blockIdx.x];
  for (int j = threadIdx.x; j < kCtThreads * kScanPer; j += kCtThreads)
    if (b0 + j < n) a[b0 + j] += add;
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

// Device -> pageable host memory through two pinned chunks: the device copy
// of one chunk overlaps the host copy of the previous one (a pageable
// cudaMemcpy of a large result runs at a few GB/s).
cudaError_t ct_d2h(ftk2b_ctx* ctx, void* dst, const void* src, size_t bytes) {
  constexpr size_t kChunk = size_t(32) << 20;
  if (!bytes) return cudaSuccess;
  for (int i = 0; i < 2; ++i) {
    if (!ctx->d2h_pin[i]) {
      cudaError_t e = cudaHostAlloc(&ctx->d2h_pin[i], kChunk, cudaHostAllocDefault);
      if (e) {
        ctx->d2h_pin[i] = nullptr;
        return e;
      }
    }
    if (!ctx->d2h_ev[i]) {
      cudaError_t e = cudaEventCreateWithFlags(&ctx->d2h_ev[i], cudaEventDisableTiming);
      if (e) return e;
    }
  }
  auto* out = static_cast<unsigned char*>(dst);
  const auto* in = static_cast<const unsigned char*>(src);
  size_t off = 0, prev_off = 0, prev_n = 0;
  int cur = 0, prev = -1;
  while (off < bytes || prev >= 0) {
    size_t n = 0;
    if (off < bytes) {
      n = std::min(kChunk, bytes - off);
      cudaError_t e = cudaMemcpyAsync(ctx->d2h_pin[cur], in + off, n, cudaMemcpyDeviceToHost, ctx->stream);
      if (!e) e = cudaEventRecord(ctx->d2h_ev[cur], ctx->stream);
      if (e) return e;
    }
    if (prev >= 0) {
      cudaError_t e = cudaEventSynchronize(ctx->d2h_ev[prev]);
      if (e) return e;
      std::memcpy(out + prev_off, ctx->d2h_pin[prev], prev_n);
    }
    if (off < bytes) {
      prev = cur;
      prev_off = off;
      prev_n = n;
      off += n;
      cur ^= 1;
    } else {
      prev = -1;
    }
  }
  return cudaSuccess;
}

// Host memory for large results (released with free()): 2 MB-aligned and
// advised for huge pages, so the first touch while copying in faults once per
// 2 MB instead of once per 4 KB (about half the copy time for a 1 GB result).
void* ct_host_alloc(size_t bytes) {
  constexpr size_t kHuge = size_t(2) << 20;
  if (bytes < (size_t(64) << 20)) return std::malloc(bytes ? bytes : 1);
  void* p = nullptr;
  if (posix_memalign(&p, kHuge, (bytes + kHuge - 1) / kHuge * kHuge) != 0) return nullptr;
  madvise(p, (bytes + kHuge - 1) / kHuge * kHuge, MADV_HUGEPAGE);
  return p;
}

enum {
  kBufField = 0, kBufPos, kBufMask, kBufBlk, kBufVoff, kBufSimp, kBufLam, kBufBary, kBufFirst, kBufParent,
  kBufCells, kBufKey0, kBufKey1, kBufVal0, kBufVal1, kBufHist, kBufCellsOut, kBufTrack, kBufCount, kBufList,
  kBufField2, kBufUpOff, kBufUpNbr, kBufBaseCells,
  // fiber surfaces on extruded meshes
  kBufFeTris, kBufFeEdges, kBufFeSimp, kBufFeLam, kBufFeBary, kBufFePhase, kBufFeDisc, kBufFeFlag, kBufFeHi,
  kBufFeLo, kBufCount_
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
  auto* cell64 = reinterpret_cast<unsigned long long*>(counts + 10);  // manifold cells (64-bit)
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
  // the mixed hypercubes, once: every later stage walks this list
  C_TRY(B[kBufList].ensure(8 * (g.ncube ? g.ncube : 1)));
  auto* list = static_cast<unsigned long long*>(B[kBufList].p);
  unsigned* list_cnt = counts + 4;
  ct_mixed_kernel<<<grid_of(g.ncube, 256, 64ull * sms), 256, 0, st>>>(g, pos, list, list_cnt);
  ctx->launches += 1;
  const unsigned wgrid = 16u * sms;  // 8 warps per block
  if (d == 3 && n) {
    ct_fill_u64_kernel<<<grid_of(n, 256, 8ull * sms), 256, 0, st>>>(first, ~0ull, n);
    ct_first_kernel<<<wgrid, 256, 0, st>>>(g, list, list_cnt, mask, voff, first);
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
    C_TRY(cudaMemsetAsync(cell64, 0, 8, st));
    if (n) ct_iota_kernel<<<grid_of(n, 256, 8ull * sms), 256, 0, st>>>(parent, n);
    ct_cells_kernel<<<wgrid, 256, 0, st>>>(g, list, list_cnt, mask, voff, first, n, cells, cell64, cap, parent,
                                           counts + 3);
    ctx->launches += 2;
    unsigned long long nc64 = 0;
    C_TRY(cudaMemcpyAsync(&nc64, cell64, 8, cudaMemcpyDeviceToHost, st));
    C_TRY(ctx->sync());
    if (nc64 >= 0x7FFFFFFFull) return cfail(ctx, FTK2B_UNSUPPORTED, "more than 2^31 - 1 manifold cells");
    ncell = (unsigned)nc64;
    if (ncell <= cap) break;
    cap = ncell;
  }
  auto* cells = static_cast<unsigned*>(B[kBufCells].p);

  // lexicographic order of the cells: buckets by leading node, then each
  // bucket's rows sorted
  const unsigned ccap = ncell ? ncell : 1;
  const unsigned nb = n + 1;  // bucket offsets, the last one the total
  const unsigned sblocks = (unsigned)((nb + kCtThreads * kScanPer - 1) / (kCtThreads * kScanPer));
  C_TRY(B[kBufKey0].ensure(4ull * nb));            // counts, then offsets
  C_TRY(B[kBufKey1].ensure(4ull * nb));            // scatter cursors
  C_TRY(B[kBufVal0].ensure(4ull * (sblocks + 1)));  // scan block totals
  C_TRY(B[kBufCellsOut].ensure(4ull * kc * ccap));
  auto* boff = static_cast<unsigned*>(B[kBufKey0].p);
  auto* bcur = static_cast<unsigned*>(B[kBufKey1].p);
  auto* btot = static_cast<unsigned*>(B[kBufVal0].p);
  auto* cells_out = static_cast<unsigned*>(B[kBufCellsOut].p);
  const unsigned cg = grid_of(ccap, 256, 16ull * sms);
  if (ncell) {
    C_TRY(cudaMemsetAsync(boff, 0, 4ull * nb, st));
    C_TRY(cudaMemsetAsync(bcur, 0, 4ull * nb, st));
    ct_bucket_count_kernel<<<cg, 256, 0, st>>>(cells, ncell, kc, boff);
    ct_scan_blocks_kernel<<<sblocks, kCtThreads, 0, st>>>(boff, nb, btot);
    C_TRY(launch_scan(btot, sblocks, nullptr, nullptr, st));
    ct_scan_add_kernel<<<sblocks, kCtThreads, 0, st>>>(boff, nb, btot);
    ct_bucket_scatter_kernel<<<cg, 256, 0, st>>>(cells, ncell, kc, boff, bcur, cells_out);
    ct_bucket_sort_kernel<<<grid_of(n, 128, 32ull * sms), 128, 0, st>>>(cells_out, boff, n, kc, counts + 3,
                                                                         nullptr);
    ctx->launches += 6;
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
  res->simplices = static_cast<uint64_t*>(ct_host_alloc(16 * ncap));
  res->lambda = static_cast<double*>(ct_host_alloc(16 * ncap));
  res->barycentric = static_cast<float*>(ct_host_alloc(8 * ncap));
  res->track_id = static_cast<uint64_t*>(ct_host_alloc(8 * ncap));
  res->scalar = static_cast<float*>(ct_host_alloc(4 * ncap));
  res->cells = static_cast<uint32_t*>(ct_host_alloc(4ull * kc * ccap));
  if (!res->simplices || !res->lambda || !res->barycentric || !res->track_id || !res->scalar || !res->cells)
    return cfail(ctx, FTK2B_OOM, "host result allocation failed");
  C_TRY(ctx->sync());
  C_TRY(ct_d2h(ctx, res->simplices, simp, 16ull * n));
  C_TRY(ct_d2h(ctx, res->lambda, lam, 16ull * n));
  C_TRY(ct_d2h(ctx, res->barycentric, bary, 8ull * n));
  C_TRY(ct_d2h(ctx, res->track_id, track, 8ull * n));
  C_TRY(ct_d2h(ctx, res->cells, cells_out, 4ull * kc * ncell));
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

// ---------------------------------------------------------------------------
// Fiber surfaces: FiberPredicate<T> on a regular 3D+t mesh (predicate.hpp:
// 341-362; form_general_manifold_patches with k = 2, engine.hpp:1341-1418).
// Features are the mesh triangles where both fields minus their thresholds
// have the origin inside (simulation of simplicity, 2-D).  Every triangle of
// the Freudenthal mesh is (c, c + a, c + b) for corner masks 0 < a < b, a a
// subset of b (50 types in a 4-cube), so triangles in simplex order are
// (c, a, b) in vertex order, then a, then b as binary numbers: ranks again
// come from per-vertex masks and a scan.  The reference's node code
// (v_min << 24 | a << 4 | b, mesh.hpp:736-749) orders triangles the same way,
// so its star centres are the smallest ranks.

struct FsTables {
  unsigned char ta[50], tb[50];  // corner masks of the second and third vertex, by type
  unsigned char idx[16][16];     // type of (a, b), 255 where (a, b) is no triangle
};

// per vertex and component: bit 2j positive (quantised >= 1), bit 2j+1
// negative (<= -1); zero leaves both clear
template <typename T>
__global__ void fs_class_kernel(CtGeom g, const T* __restrict__ f0, const T* __restrict__ f1, T t0, T t1,
                                double q, unsigned char* __restrict__ cls) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < g.nv;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long c[4];
    ct_coords(g, i, c);
    const unsigned long long gid = ct_gid(g, c), ai = ct_aidx(g, c);
    unsigned char b = 0;
    const T v[2] = {ct_adj(g, f0, ai, gid, t0), ct_adj(g, f1, ai, gid, t1)};
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const double x = __dadd_rn(__dmul_rn((double)v[j], q), v[j] > T(0) ? 0.5 : -0.5);
      if (x >= 1.0) b |= (unsigned char)(1u << (2 * j));
      if (x <= -1.0) b |= (unsigned char)(2u << (2 * j));
    }
    cls[i] = b;
  }
}

template <typename T>
__device__ __forceinline__ void fs_values(const CtGeom& g, const T* f0, const T* f1, T t0, T t1,
                                          unsigned long long ai, unsigned long long gid, int a, int b, T v[3][2]) {
  const unsigned long long ao[3] = {0ull, g.aoff[a], g.aoff[b]}, go[3] = {0ull, g.goff[a], g.goff[b]};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    v[i][0] = ct_adj(g, f0, ai + ao[i], gid + go[i], t0);
    v[i][1] = ct_adj(g, f1, ai + ao[i], gid + go[i], t1);
  }
}

// per vertex: bit t of the 50-bit mask = triangle type t from this vertex is
// a feature.  One component of one strict sign at all three vertices keeps
// the origin outside whatever the ties (exact pre-test); the rest go through
// the exact 2-D test.
template <typename T>
__global__ void fs_mask_kernel(CtGeom g, FsTables tb, const T* __restrict__ f0, const T* __restrict__ f1, T t0,
                               T t1, double q, const unsigned char* __restrict__ cls,
                               unsigned long long* __restrict__ mask, unsigned* __restrict__ blk,
                               unsigned long long* __restrict__ total64) {
  __shared__ unsigned tot;
  const unsigned long long i = blockIdx.x * (unsigned long long)kCtThreads + threadIdx.x;
  unsigned long long m = 0;
  if (i < g.nv) {
    unsigned long long c[4];
    ct_coords(g, i, c);
    const unsigned inb = ct_inbounds(g, c);
    const unsigned long long gid = ct_gid(g, c), ai = ct_aidx(g, c);
    const unsigned c0 = cls[i];
    for (int t = 0; t < 50; ++t) {
      const int a = tb.ta[t], b = tb.tb[t];
      if (b & ~inb) continue;
      const unsigned all = c0 & cls[i + g.loff[a]] & cls[i + g.loff[b]];
      if (all) continue;
      T v[3][2];
      fs_values(g, f0, f1, t0, t1, ai, gid, a, b, v);
      if (sos_inside2<T>(v, q)) m |= 1ull << t;
    }
    mask[i] = m;
  }
  ct_block_scan((unsigned)__popcll(m), &tot);
  if (threadIdx.x == 0) {
    blk[blockIdx.x] = tot;
    atomicAdd(total64, (unsigned long long)tot);
  }
}

template <typename T>
__global__ void fs_emit_kernel(CtGeom g, FsTables tb, const T* __restrict__ f0, const T* __restrict__ f1, T t0,
                               T t1, const unsigned long long* __restrict__ mask,
                               const unsigned* __restrict__ blk_off, unsigned* __restrict__ voff,
                               unsigned long long* __restrict__ simp, double* __restrict__ lam,
                               float* __restrict__ bary) {
  __shared__ unsigned tot;
  const unsigned long long i = blockIdx.x * (unsigned long long)kCtThreads + threadIdx.x;
  const unsigned long long m = i < g.nv ? mask[i] : 0ull;
  const unsigned base = blk_off[blockIdx.x] + ct_block_scan((unsigned)__popcll(m), &tot);
  if (i >= g.nv) return;
  voff[i] = base;
  if (!m) return;
  unsigned long long c[4];
  ct_coords(g, i, c);
  const unsigned long long gid = ct_gid(g, c), ai = ct_aidx(g, c);
  unsigned r = base;
  for (int t = 0; t < 50; ++t) {
    if (!((m >> t) & 1ull)) continue;
    const int a = tb.ta[t], b = tb.tb[t];
    T v[3][2];
    fs_values(g, f0, f1, t0, t1, ai, gid, a, b, v);
    T l[3];
    if (!solve_exact<2, T>(v, l))  // FiberPredicate keeps the centroid: (T)1.0 / 3.0
      for (int k = 0; k < 3; ++k) l[k] = (T)((double)(T)1.0 / 3.0);
    simp[3 * (size_t)r] = gid;
    simp[3 * (size_t)r + 1] = gid + g.goff[a];
    simp[3 * (size_t)r + 2] = gid + g.goff[b];
    for (int k = 0; k < 3; ++k) {
      lam[3 * (size_t)r + k] = (double)l[k];
      bary[3 * (size_t)r + k] = (float)l[k];
    }
    ++r;
  }
}

// hypercubes with a feature triangle at one of their lower corners (a
// superset of the cubes whose pentatopes hold features)
__global__ void fs_list_kernel(CtGeom g, const unsigned long long* __restrict__ mask,
                               unsigned long long* __restrict__ list, unsigned* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  for (unsigned long long q0 = blockIdx.x * (unsigned long long)blockDim.x; q0 < g.ncube;
       q0 += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long q = q0 + threadIdx.x;
    bool any = false;
    unsigned long long base = 0;
    if (q < g.ncube) {
      unsigned long long r = q;
      for (int k = 0; k < g.d; ++k) {
        const unsigned long long n = g.L[k] - 1, c = r % n;
        r /= n;
        base += c * g.lstr[k];
      }
      for (int e = 0; e < 15 && !any; ++e) any = mask[base + g.loff[e]] != 0ull;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, any);
    unsigned wbase = 0;
    if (lane == 0 && bal) wbase = atomicAdd(cnt, (unsigned)__popc(bal));
    wbase = __shfl_sync(0xffffffffu, wbase, 0);
    if (any) list[wbase + __popc(bal & ((1u << lane) - 1u))] = base;
  }
}

// One pentatope per lane (24 per listed cube): its feature triangles in rank
// order (the reference's code order), the star centre h_S = the first; per
// tet face (path vertex i left out), the face's feature triangles in order,
// h_T the first, and a triangle {h_S, h_T, n} for every later n, unless h_S is
// h_T or n (engine.hpp:1388-1413).  Two passes: count, reserve per warp, write.
__global__ void fs_cells_kernel(CtGeom g, FsTables tb, const unsigned long long* __restrict__ list,
                                const unsigned* list_cnt, const unsigned long long* __restrict__ mask,
                                const unsigned* __restrict__ voff, unsigned* __restrict__ cells,
                                unsigned long long* cnt, unsigned cap, unsigned* parent, unsigned* err) {
  const int lane = threadIdx.x & 31;
  const unsigned nl = *list_cnt;
  const unsigned long long warp = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long it = warp; it < nl; it += nwarps) {
    unsigned rank[10], vset[10];
    int nn = 0;
    if (lane < 24) {
      const unsigned long long base = list[it];
      int pe[5];
      pe[0] = 0;
      for (int i = 0; i < 4; ++i) pe[i + 1] = pe[i] | (1 << g.perm[lane][i]);
      for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 4; ++j)
          for (int k = j + 1; k < 5; ++k) {
            const int lo = pe[i], t = tb.idx[pe[j] ^ lo][pe[k] ^ lo];
            const unsigned long long v = base + g.loff[lo];
            const unsigned long long mv = __ldg(mask + v);
            if (!((mv >> t) & 1ull)) continue;
            unsigned rk = __ldg(voff + v) + (unsigned)__popcll(mv & ((1ull << t) - 1ull));
            unsigned vs = (1u << i) | (1u << j) | (1u << k);
            int p = nn++;
            while (p > 0 && rank[p - 1] > rk) {
              rank[p] = rank[p - 1];
              vset[p] = vset[p - 1];
              --p;
            }
            rank[p] = rk;
            vset[p] = vs;
          }
    }
    // pass 1: count
    unsigned mine = 0;
    if (nn >= 2) {
      const unsigned hs = rank[0];
      for (int f = 0; f < 5; ++f) {
        int seen = 0;
        unsigned ht = 0;
        for (int x = 0; x < nn; ++x) {
          if (vset[x] & (1u << f)) continue;
          if (seen++ == 0) {
            ht = rank[x];
            continue;
          }
          if (hs != ht && hs != rank[x]) ++mine;
        }
      }
    }
    unsigned incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const unsigned wtot = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long wbase = 0;
    if (lane == 31 && wtot) wbase = atomicAdd(cnt, (unsigned long long)wtot);
    wbase = __shfl_sync(0xffffffffu, wbase, 31);
    unsigned long long slot = wbase + incl - mine;
    // pass 2: write and join
    if (mine) {
      const unsigned hs = rank[0];
      for (int f = 0; f < 5; ++f) {
        int seen = 0;
        unsigned ht = 0;
        for (int x = 0; x < nn; ++x) {
          if (vset[x] & (1u << f)) continue;
          if (seen++ == 0) {
            ht = rank[x];
            continue;
          }
          if (hs == ht || hs == rank[x]) continue;
          unsigned tri[3] = {hs, ht, rank[x]};
          ct_sort4(tri, 3);
          if (slot < cap)
            for (int k = 0; k < 3; ++k) cells[(size_t)slot * 3 + k] = tri[k];
          ++slot;
          uf_unite(parent, tri[0], tri[1], err);
          uf_unite(parent, tri[0], tri[2], err);
        }
      }
    }
  }
}

template <typename T>
ftk2b_status run_fiber_surface(ftk2b_ctx* ctx, const CtGeom& g, const FsTables& tb, const void* fa,
                               const void* fb, T t0, T t1, double q, ftk2b_fiber_surface_result* res) {
  cudaStream_t st = ctx->stream;
  DevBuf* B = ctx->contour;
  const unsigned long long nblk = (g.nv + kCtThreads - 1) / kCtThreads;
  if (nblk >= 0xFFFFFFF0ull) return cfail(ctx, FTK2B_UNSUPPORTED, "mesh too large");
  C_TRY(B[kBufPos].ensure(g.nv));
  C_TRY(B[kBufHist].ensure(8 * g.nv));
  C_TRY(B[kBufVoff].ensure(4 * g.nv));
  C_TRY(B[kBufBlk].ensure(4 * (nblk + 1)));
  C_TRY(B[kBufCount].ensure(64));
  auto* cls = static_cast<unsigned char*>(B[kBufPos].p);
  auto* mask = static_cast<unsigned long long*>(B[kBufHist].p);
  auto* voff = static_cast<unsigned*>(B[kBufVoff].p);
  auto* blk = static_cast<unsigned*>(B[kBufBlk].p);
  auto* counts = static_cast<unsigned*>(B[kBufCount].p);  // [0] n, [1] cells, [2] roots, [3] err, [4] cubes
  auto* total64 = reinterpret_cast<unsigned long long*>(counts + 8);
  auto* cell64 = reinterpret_cast<unsigned long long*>(counts + 10);  // manifold cells (64-bit)
  const T* a0 = static_cast<const T*>(fa);
  const T* a1 = static_cast<const T*>(fb);
  const unsigned sms = (unsigned)ctx->num_sms;
  C_TRY(cudaMemsetAsync(counts, 0, 64, st));
  C_TRY(cudaEventRecord(ctx->ev0, st));
  fs_class_kernel<T><<<grid_of(g.nv, 256, 32ull * sms), 256, 0, st>>>(g, a0, a1, t0, t1, q, cls);
  fs_mask_kernel<T><<<(unsigned)nblk, kCtThreads, 0, st>>>(g, tb, a0, a1, t0, t1, q, cls, mask, blk, total64);
  C_TRY(launch_scan(blk, (unsigned)nblk, counts + 0, nullptr, st));  // counts[0]: feature count (labels)
  ctx->launches += 3;
  unsigned long long n64 = 0;
  C_TRY(cudaMemcpyAsync(&n64, total64, 8, cudaMemcpyDeviceToHost, st));
  C_TRY(ctx->sync());
  if (n64 >= 0xFFFFFFF0ull) return cfail(ctx, FTK2B_UNSUPPORTED, "more than 2^32 - 16 feature triangles");
  const unsigned n = (unsigned)n64;
  const size_t ncap = n ? n : 1;
  C_TRY(B[kBufSimp].ensure(24 * ncap));
  C_TRY(B[kBufLam].ensure(24 * ncap));
  C_TRY(B[kBufBary].ensure(12 * ncap));
  C_TRY(B[kBufParent].ensure(4 * ncap));
  C_TRY(B[kBufTrack].ensure(8 * ncap));
  auto* simp = static_cast<unsigned long long*>(B[kBufSimp].p);
  auto* lam = static_cast<double*>(B[kBufLam].p);
  auto* bary = static_cast<float*>(B[kBufBary].p);
  auto* parent = static_cast<unsigned*>(B[kBufParent].p);
  auto* track = static_cast<unsigned long long*>(B[kBufTrack].p);
  fs_emit_kernel<T><<<(unsigned)nblk, kCtThreads, 0, st>>>(g, tb, a0, a1, t0, t1, mask, blk, voff, simp, lam, bary);
  C_TRY(B[kBufList].ensure(8 * (g.ncube ? g.ncube : 1)));
  auto* list = static_cast<unsigned long long*>(B[kBufList].p);
  unsigned* list_cnt = counts + 4;
  fs_list_kernel<<<grid_of(g.ncube, 256, 64ull * sms), 256, 0, st>>>(g, mask, list, list_cnt);
  ctx->launches += 2;

  unsigned cap = (unsigned)std::min<unsigned long long>(0x7FFFFFFFull, std::max<unsigned long long>(1024ull, 4ull * n));
  unsigned ncell = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    C_TRY(B[kBufCells].ensure((size_t)12 * cap));
    auto* cells = static_cast<unsigned*>(B[kBufCells].p);
    C_TRY(cudaMemsetAsync(counts + 1, 0, 12, st));
    C_TRY(cudaMemsetAsync(cell64, 0, 8, st));
    if (n) ct_iota_kernel<<<grid_of(n, 256, 8ull * sms), 256, 0, st>>>(parent, n);
    fs_cells_kernel<<<16u * sms, 256, 0, st>>>(g, tb, list, list_cnt, mask, voff, cells, cell64, cap, parent,
                                              counts + 3);
    ctx->launches += 2;
    unsigned long long nc64 = 0;
    C_TRY(cudaMemcpyAsync(&nc64, cell64, 8, cudaMemcpyDeviceToHost, st));
    C_TRY(ctx->sync());
    if (nc64 >= 0x7FFFFFFFull) return cfail(ctx, FTK2B_UNSUPPORTED, "more than 2^31 - 1 manifold triangles");
    ncell = (unsigned)nc64;
    if (ncell <= cap) break;
    cap = ncell;
  }
  auto* cells = static_cast<unsigned*>(B[kBufCells].p);

  // sorted, unique triangles: buckets by leading node, each sorted and made
  // unique, compacted
  const unsigned ccap = ncell ? ncell : 1;
  const unsigned nb = n + 1;
  const unsigned sblocks = (unsigned)((nb + kCtThreads * kScanPer - 1) / (kCtThreads * kScanPer));
  C_TRY(B[kBufKey0].ensure(4ull * nb));
  C_TRY(B[kBufKey1].ensure(4ull * nb));
  C_TRY(B[kBufVal0].ensure(4ull * (sblocks + 1)));
  C_TRY(B[kBufVal1].ensure(4ull * nb));
  C_TRY(B[kBufCellsOut].ensure(12ull * ccap));
  C_TRY(B[kBufMask].ensure(12ull * ccap));
  auto* boff = static_cast<unsigned*>(B[kBufKey0].p);
  auto* bcur = static_cast<unsigned*>(B[kBufKey1].p);
  auto* btot = static_cast<unsigned*>(B[kBufVal0].p);
  auto* uoff = static_cast<unsigned*>(B[kBufVal1].p);
  auto* rows = static_cast<unsigned*>(B[kBufCellsOut].p);
  auto* cells_out = static_cast<unsigned*>(B[kBufMask].p);
  const unsigned cg = grid_of(ccap, 256, 16ull * sms);
  unsigned nuniq = 0;
  if (ncell) {
    C_TRY(cudaMemsetAsync(boff, 0, 4ull * nb, st));
    C_TRY(cudaMemsetAsync(bcur, 0, 4ull * nb, st));
    C_TRY(cudaMemsetAsync(uoff, 0, 4ull * nb, st));
    ct_bucket_count_kernel<<<cg, 256, 0, st>>>(cells, ncell, 3, boff);
    ct_scan_blocks_kernel<<<sblocks, kCtThreads, 0, st>>>(boff, nb, btot);
    C_TRY(launch_scan(btot, sblocks, nullptr, nullptr, st));
    ct_scan_add_kernel<<<sblocks, kCtThreads, 0, st>>>(boff, nb, btot);
    ct_bucket_scatter_kernel<<<cg, 256, 0, st>>>(cells, ncell, 3, boff, bcur, rows);
    ct_bucket_sort_kernel<<<grid_of(n, 128, 32ull * sms), 128, 0, st>>>(rows, boff, n, 3, counts + 3, uoff);
    ct_scan_blocks_kernel<<<sblocks, kCtThreads, 0, st>>>(uoff, nb, btot);
    C_TRY(launch_scan(btot, sblocks, nullptr, nullptr, st));
    ct_scan_add_kernel<<<sblocks, kCtThreads, 0, st>>>(uoff, nb, btot);
    ct_bucket_compact_kernel<<<grid_of(n, 128, 32ull * sms), 128, 0, st>>>(rows, boff, uoff, n, 3, cells_out);
    ctx->launches += 10;
    C_TRY(cudaMemcpyAsync(&nuniq, uoff + n, 4, cudaMemcpyDeviceToHost, st));
  }
  if (n) {
    C_TRY(launch_uf_label(parent, counts + 0, n, track, counts + 2, st));
    ctx->launches += 1;
  }
  C_TRY(cudaEventRecord(ctx->ev1, st));
  unsigned hc[4] = {0, 0, 0, 0};
  C_TRY(cudaMemcpyAsync(hc, counts, 16, cudaMemcpyDeviceToHost, st));
  C_TRY(ctx->sync());
  res->n_features = n;
  res->n_cells = nuniq;
  res->simplices = static_cast<uint64_t*>(ct_host_alloc(24 * ncap));
  res->lambda = static_cast<double*>(ct_host_alloc(24 * ncap));
  res->barycentric = static_cast<float*>(ct_host_alloc(12 * ncap));
  res->track_id = static_cast<uint64_t*>(ct_host_alloc(8 * ncap));
  res->scalar = static_cast<float*>(std::calloc(ncap, 4));
  res->cells = static_cast<uint32_t*>(ct_host_alloc(12ull * (nuniq ? nuniq : 1)));
  if (!res->simplices || !res->lambda || !res->barycentric || !res->track_id || !res->scalar || !res->cells)
    return cfail(ctx, FTK2B_OOM, "host result allocation failed");
  C_TRY(ct_d2h(ctx, res->simplices, simp, 24ull * n));
  C_TRY(ct_d2h(ctx, res->lambda, lam, 24ull * n));
  C_TRY(ct_d2h(ctx, res->barycentric, bary, 12ull * n));
  C_TRY(ct_d2h(ctx, res->track_id, track, 8ull * n));
  C_TRY(ct_d2h(ctx, res->cells, cells_out, 12ull * nuniq));
  if (hc[3] & 1u) return cfail(ctx, FTK2B_CUDA_ERROR, "union-find did not settle");
  res->n_tracks = hc[2];
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  res->device_ms = ms;
  return FTK2B_OK;
}

// ---------------------------------------------------------------------------
// Level sets on ExtrudedSimplicialMesh(UnstructuredSimplicialMesh, L)
// (mesh.hpp:542-599): vertex ids v = s + t * S (S base vertices, layers
// t = 0 .. L), the field per vertex.  The mesh's edges from a lower vertex
// a + tS, in id order, are its spatial edges to b + tS (base edges a < b),
// its vertical edge to a + (t + 1)S and the prism diagonals to b + (t + 1)S
// (the Kuhn split of a prism over a sorted base cell joins v_a at t to v_b at
// t + 1 only for a < b), so ranks again come from a per-vertex mask over
// 2 deg(a) + 1 candidates and a scan.  The reference's first pass visits the
// spatial and vertical edges only (iterate_simplices(1)); the diagonals it
// meets while marching over the cells, which it visits by layer, base cell
// (in stored order, each sorted) and Kuhn index j (vertices v_0..v_j at t,
// v_j..v_k at t + 1), one worker at a time.

struct CeGeom {
  int d;                       // spacetime dims: 3 (triangle base) or 4 (tet base)
  unsigned long long S, L;     // base vertices, layers
  unsigned long long nv;       // S * (L + 1)
  unsigned long long ncell;    // base cells
  const unsigned* up_off;      // CSR of base neighbours b > a: up_nbr[up_off[a] .. up_off[a + 1])
  const unsigned* up_nbr;
  const unsigned* cells;       // ncell * d sorted base vertex ids
};

__device__ __forceinline__ int ce_nbr_index(const CeGeom& g, unsigned a, unsigned b) {
  const unsigned lo = g.up_off[a], hi = g.up_off[a + 1];
  for (unsigned i = lo; i < hi; ++i)
    if (g.up_nbr[i] == b) return (int)(i - lo);
  return -1;
}

// mask bit of the edge (x, y), x < y, in x's candidate order
__device__ __forceinline__ int ce_bit(const CeGeom& g, unsigned long long x, unsigned long long y) {
  const unsigned long long t = x / g.S;
  const unsigned a = (unsigned)(x - t * g.S);
  const int deg = (int)(g.up_off[a + 1] - g.up_off[a]);
  if (y < (t + 1) * g.S) return ce_nbr_index(g, a, (unsigned)(y - t * g.S));
  if (y == x + g.S) return deg;
  return deg + 1 + ce_nbr_index(g, a, (unsigned)(y - (t + 1) * g.S));
}

__device__ __forceinline__ unsigned ce_node(const CeGeom& g, const unsigned long long* __restrict__ mask,
                                            const unsigned* __restrict__ voff, unsigned long long x,
                                            unsigned long long y) {
  const int bit = max(ce_bit(g, x, y), 0);  // every cell pair is a base edge, so the index exists
  return voff[x] + (unsigned)__popcll(mask[x] & ((1ull << bit) - 1ull));
}

template <typename T>
__global__ void ce_sign_kernel(CeGeom g, const T* __restrict__ a, T thr, double q, unsigned char* __restrict__ pos) {
  for (unsigned long long v = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; v < g.nv;
       v += (unsigned long long)gridDim.x * blockDim.x)
    pos[v] = ct_positive(fp<T>::sub(__ldg(a + v), thr), v, q) ? 1 : 0;
}

__global__ void ce_mask_kernel(CeGeom g, const unsigned char* __restrict__ pos, unsigned long long* __restrict__ mask,
                               unsigned* __restrict__ blk, unsigned long long* __restrict__ total64) {
  __shared__ unsigned tot;
  const unsigned long long v = blockIdx.x * (unsigned long long)kCtThreads + threadIdx.x;
  unsigned long long m = 0;
  if (v < g.nv) {
    const unsigned long long t = v / g.S;
    const unsigned a = (unsigned)(v - t * g.S);
    const unsigned lo = g.up_off[a], hi = g.up_off[a + 1];
    const int deg = (int)(hi - lo);
    const unsigned char p = pos[v];
    for (unsigned i = lo; i < hi; ++i)
      if (pos[g.up_nbr[i] + t * g.S] != p) m |= 1ull << (i - lo);
    if (t < g.L) {
      if (pos[v + g.S] != p) m |= 1ull << deg;
      for (unsigned i = lo; i < hi; ++i)
        if (pos[g.up_nbr[i] + (t + 1) * g.S] != p) m |= 1ull << (deg + 1 + (int)(i - lo));
    }
    mask[v] = m;
  }
  ct_block_scan((unsigned)__popcll(m), &tot);
  if (threadIdx.x == 0) {
    blk[blockIdx.x] = tot;
    atomicAdd(total64, (unsigned long long)tot);
  }
}

template <typename T>
__global__ void ce_emit_kernel(CeGeom g, const T* __restrict__ a, T thr, const unsigned long long* __restrict__ mask,
                               const unsigned* __restrict__ blk_off, unsigned* __restrict__ voff,
                               unsigned long long* __restrict__ simp, double* __restrict__ lam,
                               float* __restrict__ bary) {
  __shared__ unsigned tot;
  const unsigned long long v = blockIdx.x * (unsigned long long)kCtThreads + threadIdx.x;
  const unsigned long long m = v < g.nv ? mask[v] : 0ull;
  const unsigned base = blk_off[blockIdx.x] + ct_block_scan((unsigned)__popcll(m), &tot);
  if (v >= g.nv) return;
  voff[v] = base;
  if (!m) return;
  const unsigned long long t = v / g.S;
  const unsigned aa = (unsigned)(v - t * g.S);
  const unsigned lo = g.up_off[aa];
  const int deg = (int)(g.up_off[aa + 1] - lo);
  const T a0 = fp<T>::sub(__ldg(a + v), thr);
  unsigned r = base;
  for (int bit = 0; bit < 2 * deg + 1; ++bit) {
    if (!((m >> bit) & 1ull)) continue;
    unsigned long long y;
    if (bit < deg) y = g.up_nbr[lo + bit] + t * g.S;
    else if (bit == deg) y = v + g.S;
    else y = g.up_nbr[lo + bit - deg - 1] + (t + 1) * g.S;
    const T a1 = fp<T>::sub(__ldg(a + y), thr);
    T l0, l1;
    ct_solve(a0, a1, &l0, &l1);
    simp[2 * (size_t)r] = v;
    simp[2 * (size_t)r + 1] = y;
    lam[2 * (size_t)r] = (double)l0;
    lam[2 * (size_t)r + 1] = (double)l1;
    bary[2 * (size_t)r] = (float)l0;
    bary[2 * (size_t)r + 1] = (float)l1;
    ++r;
  }
}

// vertices (global ids, ascending) and signs of spacetime cell q = (t, c, j)
__device__ __forceinline__ void ce_cell(const CeGeom& g, const unsigned char* pos, unsigned long long q,
                                        unsigned long long* vid, unsigned* ps, int* npos) {
  const int d = g.d;
  const unsigned long long j = q % d, tc = q / d, c = tc % g.ncell, t = tc / g.ncell;
  const unsigned* cv = g.cells + c * d;
  int k = 0;
  for (int l = 0; l <= (int)j; ++l) vid[k++] = cv[l] + t * g.S;
  for (int l = (int)j; l < d; ++l) vid[k++] = cv[l] + (t + 1) * g.S;
  unsigned s = 0;
  int np = 0;
  for (int i = 0; i <= d; ++i) {
    const unsigned b = pos[vid[i]];
    s |= b << i;
    np += (int)b;
  }
  *ps = s;
  *npos = np;
}

__device__ __forceinline__ bool ce_late(const CeGeom& g, unsigned long long x, unsigned long long y) {
  // a diagonal: its ends lie on consecutive layers and it is not vertical
  return y >= (x / g.S + 1) * g.S && y != x + g.S;
}

// (2D+t) first meeting of every diagonal node: (cell order, marching position)
__global__ void ce_first_kernel(CeGeom g, const unsigned char* __restrict__ pos,
                                const unsigned long long* __restrict__ mask, const unsigned* __restrict__ voff,
                                unsigned long long* __restrict__ first) {
  const unsigned long long nsc = g.L * g.ncell * 3ull;
  for (unsigned long long q = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; q < nsc;
       q += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long vid[5];
    unsigned ps;
    int npos;
    ce_cell(g, pos, q, vid, &ps, &npos);
    if (npos == 0 || npos == 4) continue;
    CtSimplex x;
    x.ps = ps;
    x.npos = npos;
    int ea[4], eb[4];
    const int ne = ct_crossings(x, 4, ea, eb);
    for (int k = 0; k < ne; ++k) {
      const unsigned long long lo = vid[min(ea[k], eb[k])], hi = vid[max(ea[k], eb[k])];
      if (!ce_late(g, lo, hi)) continue;
      atomicMin(first + ce_node(g, mask, voff, lo, hi), q * 4ull + (unsigned long long)k);
    }
  }
}

// marching on every spacetime cell, one per thread; slots reserved per warp
__global__ void ce_cells_kernel(CeGeom g, const unsigned char* __restrict__ pos,
                                const unsigned long long* __restrict__ mask, const unsigned* __restrict__ voff,
                                const unsigned long long* __restrict__ first, unsigned n,
                                unsigned* __restrict__ cells, unsigned long long* cnt, unsigned cap,
                                unsigned* parent, unsigned* err) {
  const int d = g.d, kc = d;
  const int lane = threadIdx.x & 31;
  const unsigned long long nsc = g.L * g.ncell * (unsigned long long)d;
  for (unsigned long long q0 = blockIdx.x * (unsigned long long)blockDim.x; q0 < nsc;
       q0 += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long q = q0 + threadIdx.x;
    unsigned cell[3][4];
    unsigned nodes[6];
    int nn = 0, ncell = 0;
    if (q < nsc) {
      unsigned long long vid[5];
      unsigned ps;
      int npos;
      ce_cell(g, pos, q, vid, &ps, &npos);
      CtSimplex x;
      x.ps = ps;
      x.npos = npos;
      auto node = [&](int i, int j) { return ce_node(g, mask, voff, vid[min(i, j)], vid[max(i, j)]); };
      if (npos != 0 && npos != d + 1) {
        if (npos == 1 || npos == d || d == 3) {
          int ea[6], eb[6];
          const int ne = ct_crossings(x, d + 1, ea, eb);
          for (int k = 0; k < ne; ++k) nodes[k] = node(ea[k], eb[k]);
          nn = ne;
          if (ne == d) {
            for (int k = 0; k < d; ++k) cell[0][k] = nodes[k];
            ncell = 1;
          } else {
            unsigned nd[4];
            unsigned long long key[4];
            for (int k = 0; k < 4; ++k) {
              nd[k] = nodes[k];
              const unsigned long long f = first[nd[k]];
              key[k] = f == ~0ull ? (unsigned long long)nd[k] : (unsigned long long)n + f;
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
            cell[0][0] = nd[0], cell[0][1] = nd[1], cell[0][2] = nd[2];
            cell[1][0] = nd[0], cell[1][1] = nd[2], cell[1][2] = nd[3];
            ncell = 2;
          }
        } else {
          const bool two_pos = npos == 2;
          int two[2], three[3], n2 = 0, n3 = 0;
          for (int i = 0; i < 5; ++i) {
            if ((((ps >> i) & 1u) != 0) == two_pos) two[n2++] = i;
            else three[n3++] = i;
          }
          unsigned T0[3], T1[3];
          for (int t = 0; t < 3; ++t) {
            T0[t] = node(two[0], three[t]);
            T1[t] = node(two[1], three[t]);
          }
          cell[0][0] = T0[0], cell[0][1] = T0[1], cell[0][2] = T0[2], cell[0][3] = T1[2];
          cell[1][0] = T0[0], cell[1][1] = T0[1], cell[1][2] = T1[1], cell[1][3] = T1[2];
          cell[2][0] = T0[0], cell[2][1] = T1[0], cell[2][2] = T1[1], cell[2][3] = T1[2];
          for (int t = 0; t < 3; ++t) nodes[t] = T0[t], nodes[3 + t] = T1[t];
          nn = 6;
          ncell = 3;
        }
      }
    }
    unsigned incl = (unsigned)ncell;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const unsigned wtot = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long wbase = 0;
    if (lane == 31 && wtot) wbase = atomicAdd(cnt, (unsigned long long)wtot);
    wbase = __shfl_sync(0xffffffffu, wbase, 31);
    unsigned long long slot = wbase + incl - (unsigned)ncell;
    for (int c = 0; c < ncell; ++c, ++slot) {
      ct_sort4(cell[c], kc);
      if (slot < cap)
        for (int k = 0; k < kc; ++k) cells[(size_t)slot * kc + k] = cell[c][k];
    }
    for (int k = 1; k < nn; ++k) uf_unite(parent, nodes[0], nodes[k], err);
  }
}

template <typename T>
ftk2b_status run_contour_extruded(ftk2b_ctx* ctx, CeGeom g, const void* field, T thr, double q,
                                  ftk2b_contour_result* res) {
  cudaStream_t st = ctx->stream;
  DevBuf* B = ctx->contour;
  const int d = g.d, kc = d;
  const unsigned long long nblk = (g.nv + kCtThreads - 1) / kCtThreads;
  if (nblk >= 0xFFFFFFF0ull) return cfail(ctx, FTK2B_UNSUPPORTED, "mesh too large");
  C_TRY(B[kBufPos].ensure(g.nv));
  C_TRY(B[kBufHist].ensure(8 * g.nv));
  C_TRY(B[kBufVoff].ensure(4 * g.nv));
  C_TRY(B[kBufBlk].ensure(4 * (nblk + 1)));
  C_TRY(B[kBufCount].ensure(64));
  auto* pos = static_cast<unsigned char*>(B[kBufPos].p);
  auto* mask = static_cast<unsigned long long*>(B[kBufHist].p);
  auto* voff = static_cast<unsigned*>(B[kBufVoff].p);
  auto* blk = static_cast<unsigned*>(B[kBufBlk].p);
  auto* counts = static_cast<unsigned*>(B[kBufCount].p);  // [0] n, [2] roots, [3] err
  auto* total64 = reinterpret_cast<unsigned long long*>(counts + 8);
  auto* cell64 = reinterpret_cast<unsigned long long*>(counts + 10);
  const T* a = static_cast<const T*>(field);
  const unsigned sms = (unsigned)ctx->num_sms;
  C_TRY(cudaMemsetAsync(counts, 0, 64, st));
  C_TRY(cudaEventRecord(ctx->ev0, st));
  ce_sign_kernel<T><<<grid_of(g.nv, 256, 32ull * sms), 256, 0, st>>>(g, a, thr, q, pos);
  ce_mask_kernel<<<(unsigned)nblk, kCtThreads, 0, st>>>(g, pos, mask, blk, total64);
  C_TRY(launch_scan(blk, (unsigned)nblk, counts + 0, nullptr, st));
  ctx->launches += 3;
  unsigned long long n64 = 0;
  C_TRY(cudaMemcpyAsync(&n64, total64, 8, cudaMemcpyDeviceToHost, st));
  C_TRY(ctx->sync());
  if (n64 >= 0xFFFFFFF0ull) return cfail(ctx, FTK2B_UNSUPPORTED, "more than 2^32 - 16 crossing edges");
  const unsigned n = (unsigned)n64;
  const size_t ncap = n ? n : 1;
  C_TRY(B[kBufSimp].ensure(16 * ncap));
  C_TRY(B[kBufLam].ensure(16 * ncap));
  C_TRY(B[kBufBary].ensure(8 * ncap));
  C_TRY(B[kBufParent].ensure(4 * ncap));
  C_TRY(B[kBufTrack].ensure(8 * ncap));
  C_TRY(B[kBufFirst].ensure(8 * ncap));
  auto* simp = static_cast<unsigned long long*>(B[kBufSimp].p);
  auto* lam = static_cast<double*>(B[kBufLam].p);
  auto* bary = static_cast<float*>(B[kBufBary].p);
  auto* parent = static_cast<unsigned*>(B[kBufParent].p);
  auto* track = static_cast<unsigned long long*>(B[kBufTrack].p);
  auto* first = static_cast<unsigned long long*>(B[kBufFirst].p);
  ce_emit_kernel<T><<<(unsigned)nblk, kCtThreads, 0, st>>>(g, a, thr, mask, blk, voff, simp, lam, bary);
  ctx->launches += 1;
  const unsigned long long nsc = g.L * g.ncell * (unsigned long long)d;
  if (n) ct_fill_u64_kernel<<<grid_of(n, 256, 8ull * sms), 256, 0, st>>>(first, ~0ull, n);
  if (d == 3 && n) {
    ce_first_kernel<<<grid_of(nsc, 256, 64ull * sms), 256, 0, st>>>(g, pos, mask, voff, first);
    ctx->launches += 2;
  }
  unsigned cap = (unsigned)std::min<unsigned long long>(
      0x7FFFFFFFull, std::max<unsigned long long>(1024ull, (d == 4 ? 8ull : 4ull) * n));
  unsigned ncell = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    C_TRY(B[kBufCells].ensure((size_t)4 * kc * cap));
    auto* cells = static_cast<unsigned*>(B[kBufCells].p);
    C_TRY(cudaMemsetAsync(counts + 1, 0, 12, st));
    C_TRY(cudaMemsetAsync(cell64, 0, 8, st));
    if (n) ct_iota_kernel<<<grid_of(n, 256, 8ull * sms), 256, 0, st>>>(parent, n);
    ce_cells_kernel<<<grid_of(nsc, 256, 64ull * sms), 256, 0, st>>>(g, pos, mask, voff, first, n, cells, cell64,
                                                                    cap, parent, counts + 3);
    ctx->launches += 2;
    unsigned long long nc64 = 0;
    C_TRY(cudaMemcpyAsync(&nc64, cell64, 8, cudaMemcpyDeviceToHost, st));
    C_TRY(ctx->sync());
    if (nc64 >= 0x7FFFFFFFull) return cfail(ctx, FTK2B_UNSUPPORTED, "more than 2^31 - 1 manifold cells");
    ncell = (unsigned)nc64;
    if (ncell <= cap) break;
    cap = ncell;
  }
  auto* cells = static_cast<unsigned*>(B[kBufCells].p);
  const unsigned ccap = ncell ? ncell : 1;
  const unsigned nb = n + 1;
  const unsigned sblocks = (unsigned)((nb + kCtThreads * kScanPer - 1) / (kCtThreads * kScanPer));
  C_TRY(B[kBufKey0].ensure(4ull * nb));
  C_TRY(B[kBufKey1].ensure(4ull * nb));
  C_TRY(B[kBufVal0].ensure(4ull * (sblocks + 1)));
  C_TRY(B[kBufCellsOut].ensure(4ull * kc * ccap));
  auto* boff = static_cast<unsigned*>(B[kBufKey0].p);
  auto* bcur = static_cast<unsigned*>(B[kBufKey1].p);
  auto* btot = static_cast<unsigned*>(B[kBufVal0].p);
  auto* cells_out = static_cast<unsigned*>(B[kBufCellsOut].p);
  const unsigned cg = grid_of(ccap, 256, 16ull * sms);
  if (ncell) {
    C_TRY(cudaMemsetAsync(boff, 0, 4ull * nb, st));
    C_TRY(cudaMemsetAsync(bcur, 0, 4ull * nb, st));
    ct_bucket_count_kernel<<<cg, 256, 0, st>>>(cells, ncell, kc, boff);
    ct_scan_blocks_kernel<<<sblocks, kCtThreads, 0, st>>>(boff, nb, btot);
    C_TRY(launch_scan(btot, sblocks, nullptr, nullptr, st));
    ct_scan_add_kernel<<<sblocks, kCtThreads, 0, st>>>(boff, nb, btot);
    ct_bucket_scatter_kernel<<<cg, 256, 0, st>>>(cells, ncell, kc, boff, bcur, cells_out);
    ct_bucket_sort_kernel<<<grid_of(n, 128, 32ull * sms), 128, 0, st>>>(cells_out, boff, n, kc, counts + 3,
                                                                         nullptr);
    ctx->launches += 6;
  }
  if (n) {
    C_TRY(launch_uf_label(parent, counts + 0, n, track, counts + 2, st));
    ctx->launches += 1;
  }
  C_TRY(cudaEventRecord(ctx->ev1, st));
  unsigned hc[4] = {0, 0, 0, 0};
  C_TRY(cudaMemcpyAsync(hc, counts, 16, cudaMemcpyDeviceToHost, st));
  C_TRY(ctx->sync());
  res->n_features = n;
  res->cell_dim = d - 1;
  res->n_cells = ncell;
  res->simplices = static_cast<uint64_t*>(ct_host_alloc(16 * ncap));
  res->lambda = static_cast<double*>(ct_host_alloc(16 * ncap));
  res->barycentric = static_cast<float*>(ct_host_alloc(8 * ncap));
  res->track_id = static_cast<uint64_t*>(ct_host_alloc(8 * ncap));
  res->scalar = static_cast<float*>(ct_host_alloc(4 * ncap));
  res->cells = static_cast<uint32_t*>(ct_host_alloc(4ull * kc * ccap));
  if (!res->simplices || !res->lambda || !res->barycentric || !res->track_id || !res->scalar || !res->cells)
    return cfail(ctx, FTK2B_OOM, "host result allocation failed");
  C_TRY(ct_d2h(ctx, res->simplices, simp, 16ull * n));
  C_TRY(ct_d2h(ctx, res->lambda, lam, 16ull * n));
  C_TRY(ct_d2h(ctx, res->barycentric, bary, 8ull * n));
  C_TRY(ct_d2h(ctx, res->track_id, track, 8ull * n));
  C_TRY(ct_d2h(ctx, res->cells, cells_out, 4ull * kc * ncell));
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

// Level sets on an extruded mesh: base cells sorted, the CSR of base edges by
// lower vertex, the field (one value per vertex id) staged.
ftk2b_status contour_extruded(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* field,
                              double threshold, double sos_q, ftk2b_contour_result** out) {
  const int cd = mesh->base_cell_dim;
  if (cd != 2 && cd != 3) return cfail(ctx, FTK2B_UNSUPPORTED, "extruded base cells are triangles or tets");
  if (!mesh->base_cells || !mesh->n_base_cells || !mesh->n_base_verts || mesh->n_layers < 1)
    return cfail(ctx, FTK2B_INVALID_ARG, "extruded mesh needs base cells, vertices and at least one layer");
  const unsigned long long S = mesh->n_base_verts, L = mesh->n_layers, nv = S * (L + 1);
  if (S >= 0xFFFFFFFFull || nv >= (1ull << 40)) return cfail(ctx, FTK2B_UNSUPPORTED, "mesh too large");
  if (field->nd != 1 || field->dims[0] < nv)
    return cfail(ctx, FTK2B_INVALID_ARG, "extruded meshes read a per-vertex array of at least %llu values", nv);
  const int d = cd + 1;
  const unsigned long long nc = mesh->n_base_cells;
  std::vector<unsigned> cells(nc * d);
  std::vector<unsigned long long> pairs;
  pairs.reserve(nc * d * (d - 1) / 2);
  for (unsigned long long c = 0; c < nc; ++c) {
    unsigned v[4];
    for (int k = 0; k < d; ++k) {
      const uint64_t x = mesh->base_cells[c * d + k];
      if (x >= S) return cfail(ctx, FTK2B_INVALID_ARG, "base cell %llu names vertex %llu of %llu", c,
                               (unsigned long long)x, S);
      v[k] = (unsigned)x;
    }
    std::sort(v, v + d);
    for (int k = 0; k < d; ++k) cells[c * d + k] = v[k];
    for (int i = 0; i < d; ++i)
      for (int j = i + 1; j < d; ++j) pairs.push_back(((unsigned long long)v[i] << 32) | v[j]);
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  std::vector<unsigned> up_off(S + 1, 0), up_nbr(pairs.size());
  for (unsigned long long p : pairs) ++up_off[(p >> 32) + 1];
  for (unsigned long long a = 0; a < S; ++a) {
    if (up_off[a + 1] > 31) return cfail(ctx, FTK2B_UNSUPPORTED, "base vertex with more than 31 higher neighbours");
    up_off[a + 1] += up_off[a];
  }
  for (size_t i = 0; i < pairs.size(); ++i) up_nbr[i] = (unsigned)(pairs[i] & 0xFFFFFFFFu);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return cfail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  DevBuf* B = ctx->contour;
  C_TRY(B[kBufUpOff].ensure(4 * up_off.size()));
  C_TRY(B[kBufUpNbr].ensure(4 * (up_nbr.size() + 1)));
  C_TRY(B[kBufBaseCells].ensure(4 * cells.size()));
  C_TRY(cudaMemcpyAsync(B[kBufUpOff].p, up_off.data(), 4 * up_off.size(), cudaMemcpyHostToDevice, ctx->stream));
  if (!up_nbr.empty())
    C_TRY(cudaMemcpyAsync(B[kBufUpNbr].p, up_nbr.data(), 4 * up_nbr.size(), cudaMemcpyHostToDevice, ctx->stream));
  C_TRY(cudaMemcpyAsync(B[kBufBaseCells].p, cells.data(), 4 * cells.size(), cudaMemcpyHostToDevice, ctx->stream));
  const size_t es = field->dtype == FTK2B_F64 ? 8 : 4;
  const void* dev = field->comp[0];
  if (field->location != FTK2B_DEVICE) {
    C_TRY(B[kBufField].ensure(nv * es));
    C_TRY(cudaMemcpyAsync(B[kBufField].p, field->comp[0], nv * es, cudaMemcpyHostToDevice, ctx->stream));
    dev = B[kBufField].p;
  }
  CeGeom g;
  std::memset(&g, 0, sizeof(g));
  g.d = d;
  g.S = S;
  g.L = L;
  g.nv = nv;
  g.ncell = nc;
  g.up_off = static_cast<const unsigned*>(B[kBufUpOff].p);
  g.up_nbr = static_cast<const unsigned*>(B[kBufUpNbr].p);
  g.cells = static_cast<const unsigned*>(B[kBufBaseCells].p);
  auto* res = new (std::nothrow) ftk2b_contour_result;
  if (!res) return cfail(ctx, FTK2B_OOM, "result allocation failed");
  std::memset(res, 0, sizeof(*res));
  const unsigned long long E = pairs.size();
  res->n_simplices = E * (L + 1) + S * L + E * L;  // spatial, vertical, diagonal edges
  // the upload of the host vectors must finish before they go out of scope
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    ftk2b_contour_result_free(res);
    return cfail(ctx, FTK2B_CUDA_ERROR, "mesh upload failed");
  }
  const ftk2b_status st = field->dtype == FTK2B_F64
                              ? run_contour_extruded<double>(ctx, g, dev, (double)threshold, sos_q, res)
                              : run_contour_extruded<float>(ctx, g, dev, (float)threshold, sos_q, res);
  if (st != FTK2B_OK) {
    ftk2b_contour_result_free(res);
    return st;
  }
  *out = res;
  return FTK2B_OK;
}

// ---------------------------------------------------------------------------
// Fiber surfaces on ExtrudedSimplicialMesh(UnstructuredSimplicialMesh(tets), L)
// (FiberPredicate<T>, predicate.hpp:341-362; the mesh, mesh.hpp:542-712;
// form_general_manifold_patches with k = 2, engine.hpp:1342-1417).  Vertex ids
// s + t S, two fields per vertex.  The triangles of the 4-D mesh are
//   spatial   every base triangle at every layer t = 0 .. L
//   lateral   the two Kuhn pieces over every base edge a < b between layers
//             t and t + 1: {a@t, a@t+1, b@t+1}, {a@t, b@t, b@t+1}
//   interior  the two triangles inside the prism over every base triangle
//             a < b < c: {a@t, b@t+1, c@t+1}, {a@t, b@t, c@t+1}
// The reference's phase 1 iterates the spatial and lateral ones (node ids in
// simplex order); the interior ones it finds while patching, numbered in the
// order it meets them: pentatopes by layer, base tet (stored order) and prism
// piece j, each pentatope's triangles in find_m_subsimplices order
// (engine.hpp:1645-1652) -- the order of its run on one worker.  Pipeline:
//   fe_test   one thread per candidate triangle: the 2-D origin test and the
//             solve with its centroid fallback, accepted ones compacted
//   sort      two stable radix sorts (third vertex, then the first two) give
//             the canonical order
//   fe_disc   one thread per pentatope: the first meeting position of every
//             accepted interior triangle (atomic minimum)
//   fe_fan    one thread per pentatope: its active triangles by node order,
//             the star-fan triangles {h_S, h_T, n}, union-find hooks
//   buckets   the fan triangles sorted and made unique; track ids

struct FeGeom {
  unsigned long long S, L, nv;      // base vertices, layers, S (L + 1)
  unsigned long long ntet, ntri, nedge;
  const unsigned* tets;              // 4 per base tet, ascending, stored order
  const unsigned* tris;              // unique base triangles, simplex order
  const unsigned* edges;             // unique base edges, simplex order
};

// candidate c: its vertex ids (ascending) and 1 when it lies inside a prism
__device__ __forceinline__ int fe_candidate(const FeGeom& g, unsigned long long c, unsigned long long v[3]) {
  const unsigned long long nsp = (g.L + 1) * g.ntri, nlat = 2 * g.L * g.nedge;
  if (c < nsp) {
    const unsigned long long t = c / g.ntri, i = c - t * g.ntri;
    for (int k = 0; k < 3; ++k) v[k] = g.tris[3 * i + k] + t * g.S;
    return 0;
  }
  c -= nsp;
  if (c < nlat) {
    const unsigned long long j = c & 1, q = c >> 1, t = q / g.nedge, e = q - t * g.nedge;
    const unsigned long long a = g.edges[2 * e], b = g.edges[2 * e + 1];
    v[0] = a + t * g.S;
    v[1] = j == 0 ? a + (t + 1) * g.S : b + t * g.S;
    v[2] = b + (t + 1) * g.S;
    return 0;
  }
  c -= nlat;
  const unsigned long long k = c & 1, q = c >> 1, t = q / g.ntri, i = q - t * g.ntri;
  const unsigned long long a = g.tris[3 * i], b = g.tris[3 * i + 1], cc = g.tris[3 * i + 2];
  v[0] = a + t * g.S;
  v[1] = b + (k == 0 ? t + 1 : t) * g.S;
  v[2] = cc + (t + 1) * g.S;
  return 1;
}

template <typename T>
__global__ void fe_test_kernel(FeGeom g, const T* __restrict__ f0, const T* __restrict__ f1, T t0, T t1, double q,
                               unsigned long long ncand, unsigned long long* __restrict__ simp,
                               double* __restrict__ lam, float* __restrict__ bary, unsigned* __restrict__ phase,
                               unsigned* cnt, unsigned cap) {
  const int lane = threadIdx.x & 31;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < ncand; base += stride) {
    const unsigned long long c = base + threadIdx.x;
    bool acc = false;
    unsigned long long v[3] = {0, 0, 0};
    int ph = 0;
    T l[3];
    if (c < ncand) {
      ph = fe_candidate(g, c, v);
      T val[3][2];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        val[k][0] = fp<T>::sub(__ldg(f0 + v[k]), t0);  // values[i][j] - thresholds[j]
        val[k][1] = fp<T>::sub(__ldg(f1 + v[k]), t1);
      }
      if (sos_inside2<T>(val, q)) {
        acc = true;
        if (!solve_exact<2, T>(val, l))  // FiberPredicate keeps the centroid: (T)1.0 / 3.0
          for (int k = 0; k < 3; ++k) l[k] = (T)((double)(T)1.0 / 3.0);
      }
    }
    const unsigned ball = __ballot_sync(0xFFFFFFFFu, acc);
    if (!ball) continue;
    unsigned b0 = 0;
    if (lane == 0) b0 = atomicAdd(cnt, (unsigned)__popc(ball));
    b0 = __shfl_sync(0xFFFFFFFFu, b0, 0);
    if (!acc) continue;
    const unsigned r = b0 + __popc(ball & ((1u << lane) - 1u));
    if (r >= cap) continue;
    for (int k = 0; k < 3; ++k) {
      simp[3 * (size_t)r + k] = v[k];
      lam[3 * (size_t)r + k] = (double)l[k];
      bary[3 * (size_t)r + k] = (float)l[k];
    }
    phase[r] = (unsigned)ph;
  }
}

__global__ void fe_set_kernel(unsigned* p, unsigned v) { *p = v; }

__global__ void fe_key_lo_kernel(const unsigned long long* __restrict__ simp, unsigned n,
                                 unsigned long long* __restrict__ key, unsigned* __restrict__ val) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    key[i] = simp[3 * (size_t)i + 2];
    val[i] = i;
  }
}

// keys of the first two vertices in the order of perm (the sort by the
// third vertex), written over that sort's keys
__global__ void fe_key_hi_kernel(const unsigned long long* __restrict__ simp, const unsigned* __restrict__ perm,
                                 unsigned n, unsigned long long* __restrict__ key) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned p = perm[i];
    key[i] = (simp[3 * (size_t)p] << 32) | simp[3 * (size_t)p + 1];
  }
}

// canonical order: features gathered by perm, lookup keys, vertex flags,
// first-meeting positions reset, union-find parents
__global__ void fe_gather_kernel(const unsigned* __restrict__ perm, unsigned n,
                                 const unsigned long long* __restrict__ simp_u, const double* __restrict__ lam_u,
                                 const float* __restrict__ bary_u, const unsigned* __restrict__ phase_u,
                                 unsigned long long* __restrict__ simp, double* __restrict__ lam,
                                 float* __restrict__ bary, unsigned* __restrict__ phase,
                                 unsigned long long* __restrict__ hi, unsigned* __restrict__ lo,
                                 unsigned char* __restrict__ vflag, unsigned long long* __restrict__ disc,
                                 unsigned* __restrict__ parent) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned p = perm[i];
    unsigned long long v[3];
    for (int k = 0; k < 3; ++k) {
      v[k] = simp_u[3 * (size_t)p + k];
      simp[3 * (size_t)i + k] = v[k];
      lam[3 * (size_t)i + k] = lam_u[3 * (size_t)p + k];
      bary[3 * (size_t)i + k] = bary_u[3 * (size_t)p + k];
      vflag[v[k]] = 1;
    }
    phase[i] = phase_u[p];
    hi[i] = (v[0] << 32) | v[1];
    lo[i] = (unsigned)v[2];
    disc[i] = ~0ull;
    parent[i] = i;
  }
}

__device__ __forceinline__ long long fe_find(const unsigned long long* __restrict__ hi,
                                             const unsigned* __restrict__ lo, unsigned n, unsigned long long h,
                                             unsigned l) {
  unsigned a = 0, b = n;
  while (a < b) {
    const unsigned mid = (a + b) >> 1;
    const unsigned long long hm = hi[mid];
    const unsigned lm = lo[mid];
    if (hm == h && lm == l) return mid;
    if (hm < h || (hm == h && lm < l)) a = mid + 1;
    else b = mid;
  }
  return -1;
}

// Pentatope p of the reference's iteration order: layer t, base tet c, prism
// piece j; its vertex ids (ascending), the spatial id and layer of each.
__device__ __forceinline__ void fe_pentatope(const FeGeom& g, unsigned long long p, unsigned long long cell[5],
                                             unsigned sp[5], int lay[5]) {
  const unsigned long long t = p / (4 * g.ntet), r = p - t * 4 * g.ntet, c = r >> 2;
  const int j = (int)(r & 3);
  const unsigned* w = g.tets + 4 * c;
  int k = 0;
  for (int l = 0; l <= j; ++l, ++k) {
    sp[k] = w[l];
    lay[k] = 0;
    cell[k] = w[l] + t * g.S;
  }
  for (int l = j; l <= 3; ++l, ++k) {
    sp[k] = w[l];
    lay[k] = 1;
    cell[k] = w[l] + (t + 1) * g.S;
  }
}

__global__ void fe_disc_kernel(FeGeom g, unsigned long long npent, const unsigned char* __restrict__ vflag,
                               const unsigned long long* __restrict__ hi, const unsigned* __restrict__ lo,
                               unsigned n, unsigned long long* __restrict__ disc) {
  for (unsigned long long p = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; p < npent;
       p += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long cell[5];
    unsigned sp[5];
    int lay[5];
    fe_pentatope(g, p, cell, sp, lay);
    int nf = 0;
    for (int k = 0; k < 5; ++k) nf += vflag[cell[k]];
    if (nf < 3) continue;
    int pos = 0;
    for (int a = 0; a < 5; ++a)
      for (int b = a + 1; b < 5; ++b)
        for (int c = b + 1; c < 5; ++c, ++pos) {
          // inside a prism: three distinct base vertices over both layers
          if (sp[a] == sp[b] || sp[b] == sp[c] || lay[a] == lay[c]) continue;
          const long long idx = fe_find(hi, lo, n, (cell[a] << 32) | cell[b], (unsigned)cell[c]);
          if (idx >= 0) atomicMin(&disc[idx], p * 16 + (unsigned long long)pos);
        }
  }
}

__global__ void fe_fan_kernel(FeGeom g, unsigned long long npent, const unsigned char* __restrict__ vflag,
                              const unsigned long long* __restrict__ hi, const unsigned* __restrict__ lo, unsigned n,
                              const unsigned* __restrict__ phase, const unsigned long long* __restrict__ disc,
                              unsigned* __restrict__ cells, unsigned long long* cnt, unsigned cap,
                              unsigned* parent, unsigned* err) {
  for (unsigned long long p = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; p < npent;
       p += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long cell[5];
    unsigned sp[5];
    int lay[5];
    fe_pentatope(g, p, cell, sp, lay);
    int nf = 0;
    for (int k = 0; k < 5; ++k) nf += vflag[cell[k]];
    if (nf < 3) continue;
    unsigned node[10], vs[10];
    unsigned long long ord[10];
    int nn = 0;
    for (int a = 0; a < 5; ++a)
      for (int b = a + 1; b < 5; ++b)
        for (int c = b + 1; c < 5; ++c) {
          const long long idx = fe_find(hi, lo, n, (cell[a] << 32) | cell[b], (unsigned)cell[c]);
          if (idx < 0) continue;
          // node order: phase-1 triangles in simplex order, then the others
          // by the position at which patching first met them
          const unsigned long long o = phase[idx] ? ((1ull << 63) | disc[idx]) : (unsigned long long)idx;
          int w = nn++;
          while (w > 0 && ord[w - 1] > o) {
            ord[w] = ord[w - 1];
            node[w] = node[w - 1];
            vs[w] = vs[w - 1];
            --w;
          }
          ord[w] = o;
          node[w] = (unsigned)idx;
          vs[w] = (1u << a) | (1u << b) | (1u << c);
        }
    if (nn < 2) continue;
    const unsigned hs = node[0];
    unsigned mine = 0;
    for (int f = 0; f < 5; ++f) {
      int seen = 0;
      unsigned ht = 0;
      for (int x = 0; x < nn; ++x) {
        if (vs[x] & (1u << f)) continue;
        if (seen++ == 0) {
          ht = node[x];
          continue;
        }
        if (hs != ht && hs != node[x]) ++mine;
      }
    }
    if (!mine) continue;
    unsigned long long slot = atomicAdd(cnt, (unsigned long long)mine);
    for (int f = 0; f < 5; ++f) {
      int seen = 0;
      unsigned ht = 0;
      for (int x = 0; x < nn; ++x) {
        if (vs[x] & (1u << f)) continue;
        if (seen++ == 0) {
          ht = node[x];
          continue;
        }
        if (hs == ht || hs == node[x]) continue;
        unsigned tri[3] = {hs, ht, node[x]};
        ct_sort4(tri, 3);
        if (slot < cap)
          for (int k = 0; k < 3; ++k) cells[(size_t)slot * 3 + k] = tri[k];
        ++slot;
        uf_unite(parent, tri[0], tri[1], err);
        uf_unite(parent, tri[0], tri[2], err);
      }
    }
  }
}

template <typename T>
ftk2b_status run_fiber_surface_extruded(ftk2b_ctx* ctx, const FeGeom& g, const void* fa, const void* fb, T t0, T t1,
                                        double q, ftk2b_fiber_surface_result* res) {
  cudaStream_t st = ctx->stream;
  DevBuf* B = ctx->contour;
  const unsigned sms = (unsigned)ctx->num_sms;
  const unsigned long long ncand = (g.L + 1) * g.ntri + 2 * g.L * g.nedge + 2 * g.L * g.ntri;
  const unsigned long long npent = 4 * g.L * g.ntet;
  C_TRY(B[kBufCount].ensure(64));
  auto* counts = static_cast<unsigned*>(B[kBufCount].p);  // [0] n, [1] accepted, [2] roots, [3] err
  auto* cell64 = reinterpret_cast<unsigned long long*>(counts + 10);
  const T* a0 = static_cast<const T*>(fa);
  const T* a1 = static_cast<const T*>(fb);
  C_TRY(cudaMemsetAsync(counts, 0, 64, st));
  C_TRY(cudaEventRecord(ctx->ev0, st));
  // 1. every candidate triangle, accepted ones compacted (capacity grows once)
  unsigned cap = ctx->fe_cap ? ctx->fe_cap : (1u << 18);
  unsigned n = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    C_TRY(B[kBufSimp].ensure(24ull * cap));
    C_TRY(B[kBufLam].ensure(24ull * cap));
    C_TRY(B[kBufBary].ensure(12ull * cap));
    C_TRY(B[kBufVoff].ensure(4ull * cap));
    C_TRY(cudaMemsetAsync(counts + 1, 0, 4, st));
    fe_test_kernel<T><<<grid_of(ncand, 256, 64ull * sms), 256, 0, st>>>(
        g, a0, a1, t0, t1, q, ncand, static_cast<unsigned long long*>(B[kBufSimp].p),
        static_cast<double*>(B[kBufLam].p), static_cast<float*>(B[kBufBary].p), static_cast<unsigned*>(B[kBufVoff].p),
        counts + 1, cap);
    ctx->launches += 1;
    C_TRY(cudaMemcpyAsync(ctx->h_counters, counts + 1, 4, cudaMemcpyDeviceToHost, st));
    C_TRY(ctx->sync());
    n = ctx->h_counters[0];
    if (n <= cap) break;
    if (n >= 0x7FFFFFF0u) return cfail(ctx, FTK2B_UNSUPPORTED, "more than 2^31 feature triangles");
    cap = n + n / 8 + 1024;
    ctx->fe_cap = cap;
  }
  const size_t ncap = n ? n : 1;
  auto* simp_u = static_cast<unsigned long long*>(B[kBufSimp].p);
  // 2. canonical order
  C_TRY(B[kBufKey0].ensure(8 * ncap));
  C_TRY(B[kBufKey1].ensure(8 * ncap));
  C_TRY(B[kBufVal0].ensure(4 * ncap));
  C_TRY(B[kBufVal1].ensure(4 * ncap));
  const int sgrid = ctx->sort_grid((unsigned)ncap);
  C_TRY(B[kBufHist].ensure(4ull * 256 * sgrid));
  auto* k0 = static_cast<unsigned long long*>(B[kBufKey0].p);
  auto* k1 = static_cast<unsigned long long*>(B[kBufKey1].p);
  auto* v0 = static_cast<unsigned*>(B[kBufVal0].p);
  auto* v1 = static_cast<unsigned*>(B[kBufVal1].p);
  auto* hist = static_cast<unsigned*>(B[kBufHist].p);
  int vb = 1;
  while (vb < 64 && (g.nv >> vb) != 0) ++vb;
  fe_set_kernel<<<1, 1, 0, st>>>(counts + 0, n);
  fe_key_lo_kernel<<<grid_of(ncap, 256, 16ull * sms), 256, 0, st>>>(simp_u, n, k0, v0);
  unsigned long long nl = 0;
  const bool alt1 = radix_sort(k0, v0, k1, v1, counts + 0, (unsigned)ncap, vb, hist, sgrid, st, &nl);
  unsigned long long* kr = alt1 ? k1 : k0;
  unsigned* vr = alt1 ? v1 : v0;
  fe_key_hi_kernel<<<grid_of(ncap, 256, 16ull * sms), 256, 0, st>>>(simp_u, vr, n, kr);
  const bool alt2 = radix_sort(kr, vr, alt1 ? k0 : k1, alt1 ? v0 : v1, counts + 0, (unsigned)ncap, 32 + vb, hist,
                               sgrid, st, &nl);
  const unsigned* perm = alt2 ? (alt1 ? v0 : v1) : vr;
  ctx->launches += nl + 3;
  C_TRY(B[kBufFeSimp].ensure(24 * ncap));
  C_TRY(B[kBufFeLam].ensure(24 * ncap));
  C_TRY(B[kBufFeBary].ensure(12 * ncap));
  C_TRY(B[kBufFePhase].ensure(4 * ncap));
  C_TRY(B[kBufFeDisc].ensure(8 * ncap));
  C_TRY(B[kBufFeHi].ensure(8 * ncap));
  C_TRY(B[kBufFeLo].ensure(4 * ncap));
  C_TRY(B[kBufFeFlag].ensure(g.nv));
  C_TRY(B[kBufParent].ensure(4 * ncap));
  C_TRY(B[kBufTrack].ensure(8 * ncap));
  auto* simp = static_cast<unsigned long long*>(B[kBufFeSimp].p);
  auto* lam = static_cast<double*>(B[kBufFeLam].p);
  auto* bary = static_cast<float*>(B[kBufFeBary].p);
  auto* phase = static_cast<unsigned*>(B[kBufFePhase].p);
  auto* disc = static_cast<unsigned long long*>(B[kBufFeDisc].p);
  auto* hi = static_cast<unsigned long long*>(B[kBufFeHi].p);
  auto* lo = static_cast<unsigned*>(B[kBufFeLo].p);
  auto* vflag = static_cast<unsigned char*>(B[kBufFeFlag].p);
  auto* parent = static_cast<unsigned*>(B[kBufParent].p);
  auto* track = static_cast<unsigned long long*>(B[kBufTrack].p);
  C_TRY(cudaMemsetAsync(vflag, 0, g.nv, st));
  fe_gather_kernel<<<grid_of(ncap, 256, 16ull * sms), 256, 0, st>>>(
      perm, n, simp_u, static_cast<const double*>(B[kBufLam].p), static_cast<const float*>(B[kBufBary].p),
      static_cast<const unsigned*>(B[kBufVoff].p), simp, lam, bary, phase, hi, lo, vflag, disc, parent);
  // 3. first meeting positions of the interior triangles
  fe_disc_kernel<<<grid_of(npent, 256, 64ull * sms), 256, 0, st>>>(g, npent, vflag, hi, lo, n, disc);
  ctx->launches += 2;
  // 4. star-fan triangles
  unsigned ccap = (unsigned)std::min<unsigned long long>(0x7FFFFFFFull, std::max<unsigned long long>(1024ull, 4ull * n));
  unsigned ncell = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    C_TRY(B[kBufCells].ensure((size_t)12 * ccap));
    C_TRY(cudaMemsetAsync(cell64, 0, 8, st));
    if (attempt) ct_iota_kernel<<<grid_of(ncap, 256, 8ull * sms), 256, 0, st>>>(parent, n);
    fe_fan_kernel<<<grid_of(npent, 256, 64ull * sms), 256, 0, st>>>(g, npent, vflag, hi, lo, n, phase, disc,
                                                                    static_cast<unsigned*>(B[kBufCells].p), cell64,
                                                                    ccap, parent, counts + 3);
    ctx->launches += 1;
    unsigned long long nc64 = 0;
    C_TRY(cudaMemcpyAsync(&nc64, cell64, 8, cudaMemcpyDeviceToHost, st));
    C_TRY(ctx->sync());
    if (nc64 >= 0x7FFFFFFFull) return cfail(ctx, FTK2B_UNSUPPORTED, "more than 2^31 - 1 manifold triangles");
    ncell = (unsigned)nc64;
    if (ncell <= ccap) break;
    ccap = ncell;
  }
  auto* cells = static_cast<unsigned*>(B[kBufCells].p);
  // 5. sorted, unique triangles: buckets by leading node
  const unsigned nb = n + 1;
  const unsigned sblocks = (unsigned)((nb + kCtThreads * kScanPer - 1) / (kCtThreads * kScanPer));
  const unsigned cc = ncell ? ncell : 1;
  C_TRY(B[kBufKey0].ensure(4ull * nb));
  C_TRY(B[kBufKey1].ensure(4ull * nb));
  C_TRY(B[kBufVal0].ensure(4ull * (sblocks + 1)));
  C_TRY(B[kBufVal1].ensure(4ull * nb));
  C_TRY(B[kBufCellsOut].ensure(12ull * cc));
  C_TRY(B[kBufMask].ensure(12ull * cc));
  auto* boff = static_cast<unsigned*>(B[kBufKey0].p);
  auto* bcur = static_cast<unsigned*>(B[kBufKey1].p);
  auto* btot = static_cast<unsigned*>(B[kBufVal0].p);
  auto* uoff = static_cast<unsigned*>(B[kBufVal1].p);
  auto* rows = static_cast<unsigned*>(B[kBufCellsOut].p);
  auto* cells_out = static_cast<unsigned*>(B[kBufMask].p);
  const unsigned cg = grid_of(cc, 256, 16ull * sms);
  unsigned nuniq = 0;
  if (ncell) {
    C_TRY(cudaMemsetAsync(boff, 0, 4ull * nb, st));
    C_TRY(cudaMemsetAsync(bcur, 0, 4ull * nb, st));
    C_TRY(cudaMemsetAsync(uoff, 0, 4ull * nb, st));
    ct_bucket_count_kernel<<<cg, 256, 0, st>>>(cells, ncell, 3, boff);
    ct_scan_blocks_kernel<<<sblocks, kCtThreads, 0, st>>>(boff, nb, btot);
    C_TRY(launch_scan(btot, sblocks, nullptr, nullptr, st));
    ct_scan_add_kernel<<<sblocks, kCtThreads, 0, st>>>(boff, nb, btot);
    ct_bucket_scatter_kernel<<<cg, 256, 0, st>>>(cells, ncell, 3, boff, bcur, rows);
    ct_bucket_sort_kernel<<<grid_of(n, 128, 32ull * sms), 128, 0, st>>>(rows, boff, n, 3, counts + 3, uoff);
    ct_scan_blocks_kernel<<<sblocks, kCtThreads, 0, st>>>(uoff, nb, btot);
    C_TRY(launch_scan(btot, sblocks, nullptr, nullptr, st));
    ct_scan_add_kernel<<<sblocks, kCtThreads, 0, st>>>(uoff, nb, btot);
    ct_bucket_compact_kernel<<<grid_of(n, 128, 32ull * sms), 128, 0, st>>>(rows, boff, uoff, n, 3, cells_out);
    ctx->launches += 10;
    C_TRY(cudaMemcpyAsync(&nuniq, uoff + n, 4, cudaMemcpyDeviceToHost, st));
  }
  if (n) {
    C_TRY(launch_uf_label(parent, counts + 0, n, track, counts + 2, st));
    ctx->launches += 1;
  }
  C_TRY(cudaEventRecord(ctx->ev1, st));
  unsigned hc[4] = {0, 0, 0, 0};
  C_TRY(cudaMemcpyAsync(hc, counts, 16, cudaMemcpyDeviceToHost, st));
  C_TRY(ctx->sync());
  res->n_features = n;
  res->n_cells = nuniq;
  res->simplices = static_cast<uint64_t*>(ct_host_alloc(24 * ncap));
  res->lambda = static_cast<double*>(ct_host_alloc(24 * ncap));
  res->barycentric = static_cast<float*>(ct_host_alloc(12 * ncap));
  res->track_id = static_cast<uint64_t*>(ct_host_alloc(8 * ncap));
  res->scalar = static_cast<float*>(std::calloc(ncap, 4));
  res->cells = static_cast<uint32_t*>(ct_host_alloc(12ull * (nuniq ? nuniq : 1)));
  if (!res->simplices || !res->lambda || !res->barycentric || !res->track_id || !res->scalar || !res->cells)
    return cfail(ctx, FTK2B_OOM, "host result allocation failed");
  C_TRY(ct_d2h(ctx, res->simplices, simp, 24ull * n));
  C_TRY(ct_d2h(ctx, res->lambda, lam, 24ull * n));
  C_TRY(ct_d2h(ctx, res->barycentric, bary, 12ull * n));
  C_TRY(ct_d2h(ctx, res->track_id, track, 8ull * n));
  C_TRY(ct_d2h(ctx, res->cells, cells_out, 12ull * nuniq));
  if (hc[3] & 1u) return cfail(ctx, FTK2B_TIMEOUT, "union-find retry bound reached");
  res->n_tracks = hc[2];
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  res->device_ms = ms;
  return FTK2B_OK;
}

// Fiber surfaces on an extruded mesh over tets: base tets sorted, the unique
// base triangles and edges in simplex order, both fields (one value per
// vertex id) staged.
ftk2b_status fiber_surface_extruded(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* field,
                                    const double thr[2], double sos_q, ftk2b_fiber_surface_result** out) {
  if (mesh->base_cell_dim != 3 || mesh->ndims != 4)
    return cfail(ctx, FTK2B_UNSUPPORTED, "fiber surfaces on extruded meshes need tet base cells (ndims 4)");
  if (!mesh->base_cells || !mesh->n_base_cells || !mesh->n_base_verts || mesh->n_layers < 1)
    return cfail(ctx, FTK2B_INVALID_ARG, "extruded mesh needs base cells, vertices and at least one layer");
  const unsigned long long S = mesh->n_base_verts, L = mesh->n_layers, nv = S * (L + 1);
  if (S >= 0xFFFFFFFFull || nv >= 0xFFFFFFFFull) return cfail(ctx, FTK2B_UNSUPPORTED, "mesh too large");
  if ((field->layout != FTK2B_LAYOUT_SEPARATE && field->layout != FTK2B_LAYOUT_PER_VERTEX) || field->nd != 1 ||
      field->dims[0] < nv)
    return cfail(ctx, FTK2B_INVALID_ARG, "extruded meshes read two per-vertex arrays of at least %llu values", nv);
  const unsigned long long nc = mesh->n_base_cells;
  std::vector<unsigned> tets(nc * 4);
  std::vector<unsigned long long> tri_keys, edge_keys;
  tri_keys.reserve(nc * 4);
  edge_keys.reserve(nc * 6);
  for (unsigned long long c = 0; c < nc; ++c) {
    unsigned v[4];
    for (int k = 0; k < 4; ++k) {
      const uint64_t x = mesh->base_cells[c * 4 + k];
      if (x >= S) return cfail(ctx, FTK2B_INVALID_ARG, "base cell %llu names vertex %llu of %llu", c,
                               (unsigned long long)x, S);
      v[k] = (unsigned)x;
    }
    std::sort(v, v + 4);
    for (int k = 0; k < 4; ++k) tets[c * 4 + k] = v[k];
    for (int r = 0; r < 4; ++r) {
      unsigned w[3];
      int k = 0;
      for (int i = 0; i < 4; ++i)
        if (i != r) w[k++] = v[i];
      // 21 bits per id when they fit, else the rows are sorted as triples
      tri_keys.push_back(((unsigned long long)w[0] << 42) | ((unsigned long long)w[1] << 21) | w[2]);
    }
    for (int i = 0; i < 4; ++i)
      for (int j = i + 1; j < 4; ++j) edge_keys.push_back(((unsigned long long)v[i] << 32) | v[j]);
  }
  std::vector<unsigned> tris;
  if (S < (1ull << 21)) {
    std::sort(tri_keys.begin(), tri_keys.end());
    tri_keys.erase(std::unique(tri_keys.begin(), tri_keys.end()), tri_keys.end());
    tris.resize(3 * tri_keys.size());
    for (size_t i = 0; i < tri_keys.size(); ++i) {
      tris[3 * i] = (unsigned)(tri_keys[i] >> 42);
      tris[3 * i + 1] = (unsigned)((tri_keys[i] >> 21) & 0x1FFFFF);
      tris[3 * i + 2] = (unsigned)(tri_keys[i] & 0x1FFFFF);
    }
  } else {
    std::vector<std::array<unsigned, 3>> t3;
    t3.reserve(nc * 4);
    for (unsigned long long c = 0; c < nc; ++c)
      for (int r = 0; r < 4; ++r) {
        std::array<unsigned, 3> w;
        int k = 0;
        for (int i = 0; i < 4; ++i)
          if (i != r) w[k++] = tets[c * 4 + i];
        t3.push_back(w);
      }
    std::sort(t3.begin(), t3.end());
    t3.erase(std::unique(t3.begin(), t3.end()), t3.end());
    tris.resize(3 * t3.size());
    for (size_t i = 0; i < t3.size(); ++i)
      for (int k = 0; k < 3; ++k) tris[3 * i + k] = t3[i][k];
  }
  std::sort(edge_keys.begin(), edge_keys.end());
  edge_keys.erase(std::unique(edge_keys.begin(), edge_keys.end()), edge_keys.end());
  std::vector<unsigned> edges(2 * edge_keys.size());
  for (size_t i = 0; i < edge_keys.size(); ++i) {
    edges[2 * i] = (unsigned)(edge_keys[i] >> 32);
    edges[2 * i + 1] = (unsigned)(edge_keys[i] & 0xFFFFFFFFu);
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) return cfail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  DevBuf* B = ctx->contour;
  C_TRY(B[kBufBaseCells].ensure(4 * tets.size()));
  C_TRY(B[kBufFeTris].ensure(4 * tris.size()));
  C_TRY(B[kBufFeEdges].ensure(4 * edges.size()));
  C_TRY(cudaMemcpyAsync(B[kBufBaseCells].p, tets.data(), 4 * tets.size(), cudaMemcpyHostToDevice, ctx->stream));
  C_TRY(cudaMemcpyAsync(B[kBufFeTris].p, tris.data(), 4 * tris.size(), cudaMemcpyHostToDevice, ctx->stream));
  C_TRY(cudaMemcpyAsync(B[kBufFeEdges].p, edges.data(), 4 * edges.size(), cudaMemcpyHostToDevice, ctx->stream));
  const size_t es = field->dtype == FTK2B_F64 ? 8 : 4;
  const void* dev[2] = {field->comp[0], field->comp[1]};
  if (field->location != FTK2B_DEVICE) {
    const int slot[2] = {kBufField, kBufField2};
    for (int j = 0; j < 2; ++j) {
      C_TRY(B[slot[j]].ensure(nv * es));
      C_TRY(cudaMemcpyAsync(B[slot[j]].p, field->comp[j], nv * es, cudaMemcpyHostToDevice, ctx->stream));
      dev[j] = B[slot[j]].p;
    }
  }
  // the upload of the host vectors must finish before they go out of scope
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return cfail(ctx, FTK2B_CUDA_ERROR, "mesh upload failed");
  FeGeom g;
  std::memset(&g, 0, sizeof(g));
  g.S = S;
  g.L = L;
  g.nv = nv;
  g.ntet = nc;
  g.ntri = tris.size() / 3;
  g.nedge = edges.size() / 2;
  g.tets = static_cast<const unsigned*>(B[kBufBaseCells].p);
  g.tris = static_cast<const unsigned*>(B[kBufFeTris].p);
  g.edges = static_cast<const unsigned*>(B[kBufFeEdges].p);
  auto* res = new (std::nothrow) ftk2b_fiber_surface_result;
  if (!res) return cfail(ctx, FTK2B_OOM, "result allocation failed");
  std::memset(res, 0, sizeof(*res));
  res->n_simplices = (L + 1) * g.ntri + 2 * L * g.nedge + 2 * L * g.ntri;
  const ftk2b_status st =
      field->dtype == FTK2B_F64
          ? run_fiber_surface_extruded<double>(ctx, g, dev[0], dev[1], thr[0], thr[1], sos_q, res)
          : run_fiber_surface_extruded<float>(ctx, g, dev[0], dev[1], (float)thr[0], (float)thr[1], sos_q, res);
  if (st != FTK2B_OK) {
    ftk2b_fiber_surface_result_free(res);
    return st;
  }
  *out = res;
  return FTK2B_OK;
}

}  // namespace

// Geometry of a regular mesh and its scalar array(s) for the level-set and
// fiber-surface pipelines; *nelem receives the element count of one array.
static ftk2b_status ct_geometry(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* field,
                                CtGeom& g, size_t* nelem_out);

extern "C" ftk2b_status ftk2b_contour_extract(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                                              const ftk2b_field_desc* field, double threshold, double sos_q,
                                              ftk2b_contour_result** out) {
  ftk2b::NvtxRange nvtx_range("ftk2b_contour_extract");
  if (!ctx) return FTK2B_INVALID_ARG;
  if (!mesh || !field || !out) return cfail(ctx, FTK2B_INVALID_ARG, "null argument");
  *out = nullptr;
  if (field->dtype != FTK2B_F32 && field->dtype != FTK2B_F64)
    return cfail(ctx, FTK2B_INVALID_ARG, "dtype must be FTK2B_F32 or FTK2B_F64");
  if (field->ncomp != 1 || !field->comp[0] ||
      (field->layout != FTK2B_LAYOUT_SEPARATE && field->layout != FTK2B_LAYOUT_PER_VERTEX))
    return cfail(ctx, FTK2B_INVALID_ARG, "level sets read one scalar array (ncomp 1, layout SEPARATE)");
  if (!(sos_q > 0)) return cfail(ctx, FTK2B_INVALID_ARG, "sos_q must be positive");
  if (mesh->kind == FTK2B_MESH_EXTRUDED) return contour_extruded(ctx, mesh, field, threshold, sos_q, out);
  if (mesh->kind != FTK2B_MESH_REGULAR) return cfail(ctx, FTK2B_INVALID_ARG, "unknown mesh kind %d", mesh->kind);
  const int d = mesh->ndims;
  if (d != 3 && d != 4) return cfail(ctx, FTK2B_UNSUPPORTED, "regular meshes have 3 or 4 dims (got %d)", d);
  CtGeom g;
  size_t nelem = 1;
  {
    const ftk2b_status gs = ct_geometry(ctx, mesh, field, g, &nelem);
    if (gs != FTK2B_OK) return gs;
  }
  const size_t es = field->dtype == FTK2B_F64 ? 8 : 4;
  const unsigned long long nv = g.nv;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return cfail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  const void* dev = field->comp[0];
  if (field->location != FTK2B_DEVICE) {
    C_TRY(ctx->contour[kBufField].ensure(nelem * es));
    C_TRY(cudaMemcpyAsync(ctx->contour[kBufField].p, field->comp[0], nelem * es, cudaMemcpyHostToDevice,
                          ctx->stream));
    dev = ctx->contour[kBufField].p;
  }
  (void)nv;
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

static ftk2b_status ct_geometry(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* field,
                                CtGeom& g, size_t* nelem_out) {
  const int d = mesh->ndims;
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
  for (int k = 0; k < d; ++k) g.lstr[k] = lstr[k];
  // axis order of the p-th Kuhn simplex as the CPU mesh decodes it
  // (mesh.hpp:407-409): successive swaps p[i] <-> p[i + j], j = p % (d - i)
  const int np = d == 3 ? 6 : 24;
  for (int p = 0; p < np; ++p) {
    int ax[4] = {0, 1, 2, 3}, t = p;
    for (int i = 0; i < d; ++i) {
      const int j = t % (d - i);
      std::swap(ax[i], ax[i + j]);
      t /= d - i;
    }
    for (int i = 0; i < 4; ++i) g.perm[p][i] = (unsigned char)ax[i];
  }
  for (int e = 0; e < (1 << d); ++e)
    for (int k = 0; k < d; ++k)
      if ((e >> k) & 1) {
        g.loff[e] += lstr[k];
        g.goff[e] += g.gs[k];
        g.aoff[e] += g.as[k];
      }
  *nelem_out = nelem;
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_fiber_surface_extract(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                                                    const ftk2b_field_desc* field, const double thresholds[2],
                                                    double sos_q, ftk2b_fiber_surface_result** out) {
  ftk2b::NvtxRange nvtx_range("ftk2b_fiber_surface_extract");
  if (!ctx) return FTK2B_INVALID_ARG;
  if (!mesh || !field || !thresholds || !out) return cfail(ctx, FTK2B_INVALID_ARG, "null argument");
  *out = nullptr;
  if (field->dtype != FTK2B_F32 && field->dtype != FTK2B_F64)
    return cfail(ctx, FTK2B_INVALID_ARG, "dtype must be FTK2B_F32 or FTK2B_F64");
  if (!(sos_q > 0)) return cfail(ctx, FTK2B_INVALID_ARG, "sos_q must be positive");
  if (mesh->kind == FTK2B_MESH_EXTRUDED) {
    if (field->ncomp != 2 || !field->comp[0] || !field->comp[1])
      return cfail(ctx, FTK2B_INVALID_ARG, "fiber surfaces read two scalar arrays (ncomp 2)");
    return fiber_surface_extruded(ctx, mesh, field, thresholds, sos_q, out);
  }
  if (mesh->kind != FTK2B_MESH_REGULAR || mesh->ndims != 4)
    return cfail(ctx, FTK2B_UNSUPPORTED, "fiber surfaces run on 3D+t meshes (ndims 4)");
  if (field->ncomp != 2 || field->layout != FTK2B_LAYOUT_SEPARATE || !field->comp[0] || !field->comp[1])
    return cfail(ctx, FTK2B_INVALID_ARG, "fiber surfaces read two scalar arrays (ncomp 2, layout SEPARATE)");
  CtGeom g;
  size_t nelem = 1;
  {
    const ftk2b_status gs = ct_geometry(ctx, mesh, field, g, &nelem);
    if (gs != FTK2B_OK) return gs;
  }
  if (g.nv >= 0xFFFFFFF0ull) return cfail(ctx, FTK2B_UNSUPPORTED, "mesh too large for fiber surfaces");
  // triangle types of a 4-cube: corner masks 0 < a < b with a a subset of b,
  // in (a, b) order
  FsTables tb;
  std::memset(&tb, 255, sizeof(tb));
  int nt = 0;
  for (int a = 1; a < 16; ++a)
    for (int b = a + 1; b < 16; ++b)
      if ((a & b) == a) {
        tb.ta[nt] = (unsigned char)a;
        tb.tb[nt] = (unsigned char)b;
        tb.idx[a][b] = (unsigned char)nt;
        ++nt;
      }
  if (nt != 50) return cfail(ctx, FTK2B_CUDA_ERROR, "triangle table has %d types", nt);
  const size_t es = field->dtype == FTK2B_F64 ? 8 : 4;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return cfail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  const void* dev[2] = {field->comp[0], field->comp[1]};
  if (field->location != FTK2B_DEVICE) {
    const int slot[2] = {kBufField, kBufField2};
    for (int j = 0; j < 2; ++j) {
      C_TRY(ctx->contour[slot[j]].ensure(nelem * es));
      C_TRY(cudaMemcpyAsync(ctx->contour[slot[j]].p, field->comp[j], nelem * es, cudaMemcpyHostToDevice,
                            ctx->stream));
      dev[j] = ctx->contour[slot[j]].p;
    }
  }
  auto* res = new (std::nothrow) ftk2b_fiber_surface_result;
  if (!res) return cfail(ctx, FTK2B_OOM, "result allocation failed");
  std::memset(res, 0, sizeof(*res));
  // triangles of the mesh: for each type, the corners c with c + b inside
  unsigned long long tris = 0;
  for (int t = 0; t < 50; ++t) {
    unsigned long long c = 1;
    for (int k = 0; k < 4; ++k) c *= ((tb.tb[t] >> k) & 1) ? g.L[k] - 1 : g.L[k];
    tris += c;
  }
  res->n_simplices = tris;
  const ftk2b_status st =
      field->dtype == FTK2B_F64
          ? run_fiber_surface<double>(ctx, g, tb, dev[0], dev[1], (double)thresholds[0], (double)thresholds[1],
                                      sos_q, res)
          : run_fiber_surface<float>(ctx, g, tb, dev[0], dev[1], (float)thresholds[0], (float)thresholds[1], sos_q,
                                     res);
  if (st != FTK2B_OK) {
    ftk2b_fiber_surface_result_free(res);
    return st;
  }
  *out = res;
  return FTK2B_OK;
}

extern "C" void ftk2b_fiber_surface_result_free(ftk2b_fiber_surface_result* r) {
  if (!r) return;
  std::free(r->simplices);
  std::free(r->lambda);
  std::free(r->barycentric);
  std::free(r->track_id);
  std::free(r->scalar);
  std::free(r->cells);
  delete r;
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
