// Critical-point extraction over an extruded unstructured spacetime mesh:
// ExtrudedSimplicialMesh(UnstructuredSimplicialMesh(cells), n_layers)
// (mesh.hpp:542-730, unstructured_mesh.hpp:12-116) with per-vertex fields
// indexed by vertex id = spatial id + t * n_spatial (engine.hpp:999-1009).
//
// The spacetime mesh has three kinds of m-simplices (m = base cell dim):
//   spatial   every base cell at every time layer t = 0..L
//   lateral   the m Kuhn pieces of the prism over every (m-1)-face of the
//             base between layers t and t+1: f[0..j]@t + f[j..m-1]@t+1
//   interior  the m simplices between consecutive top cells of the prism
//             over a base cell: u[0..s-1]@t + u[s..m]@t+1, s = 1..m
// whose top cells are the m+1 pieces u[0..p]@t + u[p..m]@t+1 of each prism.
// Spatial and lateral simplices are what the reference's phase 1 iterates
// (mesh.hpp:568-599); interior ones it finds while patching (engine.hpp:
// 1352-1367), so they number after all phase-1 nodes.
//
// Pipeline (all on the context's stream):
//   0. base-mesh preparation, cached by content: cells sorted and narrowed to
//      32 bits, every (m-1)-face keyed, radix-sorted, de-duplicated, and the
//      coface cells of each unique face gathered (unstructured_mesh.hpp:44-53)
//   1. cull words of every spacetime vertex: one coalesced pass over the field
//   2. one thread per (spatial cell | base face | base cell, layer): the AND of
//      each simplex's vertex words culls it or it runs the exact integer SoS
//      and the bit-exact solve; accepted simplices are compacted by ballot
//   3. canonical order: two stable radix sorts on the packed vertex tuple
//   4. star edges per top cell, centre = smallest node id (phase, then
//      canonical position: engine.hpp:1375-1387 for non-regular meshes)
//   5. union-find over the edges, plus for 4-D meshes the extra coface unions
//      of get_complex (engine.hpp:896-963) as ExtrudedSimplicialMesh::cofaces
//      reports them (mesh.hpp:601-712), then labels = component minimum.
#include <algorithm>
#include <cstring>
#include <vector>

#include "cp_api_internal.h"
#include "cp_stream.h"
#include "cp_stream_kernels.cuh"
#include "cp_cull.cuh"
#include "cp_device.cuh"
#include "cp_uf.cuh"

namespace ftk2b {

namespace {

enum { kCountPrepEntries = 5, kCountFaces = 6 };
enum { kErrBadVertex = 4u, kErrCofaces = 8u };

constexpr int kThreadsX = 256;
constexpr int kMaxOthers = 32;  // star partners of one centre: 8 coface cells x 4

struct ExtMeshDev {
  int cd;                            // base cell dim = m = number of components
  unsigned ns;                       // spatial vertices: vertex id = s + t * ns
  unsigned L;                        // time slabs; vertex layers t0..t0+L
  unsigned t0;                       // global layer of the first local layer
  unsigned tflip;                    // storage slot of local layer l = l xor tflip
  int skip_first_spatial;            // 1: no spatial simplices at local layer 0
  unsigned ncell, nface;
  int fbits;                         // bits per base vertex id in a face key
  const unsigned* cells;             // [ncell][cd+1], ascending
  const unsigned long long* fkeys;   // [nface], ascending packed faces
  const unsigned* cof_start;         // [nface+1]
  const unsigned* cof;               // coface cells, grouped by face
};

struct ExtSink {
  unsigned long long* hi;   // packed v0, v1
  unsigned long long* lo;   // packed v2, v3 (m = 3) or v2 (m = 2)
  unsigned* phase;          // 0 = spatial / lateral, 1 = interior
  double* lam;
  float* bary4;
  float* scalar;
  unsigned* count;
  unsigned cap;
};

__device__ __forceinline__ unsigned long long face_key(const unsigned* w, int n, int fbits) {
  unsigned long long k = 0;
  for (int i = 0; i < n; ++i) k = (k << fbits) | w[i];
  return k;
}

template <int M>
__device__ __forceinline__ void pack_tuple(const unsigned long long* v, int vb, unsigned long long& hi,
                                           unsigned long long& lo) {
  hi = (v[0] << vb) | v[1];
  lo = (M == 3) ? ((v[2] << vb) | v[3]) : v[2];
}

template <int M>
__device__ __forceinline__ void unpack_tuple(unsigned long long hi, unsigned long long lo, int vb,
                                             unsigned long long* v) {
  const unsigned long long mask = (vb >= 64) ? ~0ull : ((1ull << vb) - 1ull);
  v[0] = hi >> vb;
  v[1] = hi & mask;
  if (M == 3) {
    v[2] = lo >> vb;
    v[3] = lo & mask;
  } else {
    v[2] = lo;
  }
}

__device__ __forceinline__ long long find_tuple(const unsigned long long* __restrict__ H,
                                                const unsigned long long* __restrict__ Lo, unsigned n,
                                                unsigned long long h, unsigned long long l) {
  unsigned a = 0, b = n;
  while (a < b) {
    const unsigned mid = (a + b) >> 1;
    const unsigned long long hm = H[mid], lm = Lo[mid];
    if (hm == h && lm == l) return mid;
    if (hm < h || (hm == h && lm < l)) a = mid + 1;
    else b = mid;
  }
  return -1;
}

__device__ __forceinline__ long long find_face(const ExtMeshDev& X, unsigned long long k) {
  unsigned a = 0, b = X.nface;
  while (a < b) {
    const unsigned mid = (a + b) >> 1;
    const unsigned long long v = X.fkeys[mid];
    if (v == k) return mid;
    if (v < k) a = mid + 1;
    else b = mid;
  }
  return -1;
}

// ---------------------------------------------------------------------------
// 0. base-mesh preparation

__global__ void ext_prep_cells_kernel(const unsigned long long* __restrict__ cells64, unsigned ncell,
                                      int cd, unsigned ns, int fbits, unsigned* __restrict__ cells,
                                      unsigned long long* __restrict__ fkey, unsigned* __restrict__ fval,
                                      unsigned* counters, unsigned* err) {
  const unsigned nv = (unsigned)cd + 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) counters[kCountPrepEntries] = ncell * nv;
  for (unsigned c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    unsigned v[4] = {0, 0, 0, 0};
    for (unsigned i = 0; i < nv; ++i) {
      const unsigned long long x = cells64[(size_t)c * nv + i];
      if (x >= ns) atomicOr(err, kErrBadVertex);
      v[i] = x < ns ? (unsigned)x : 0u;
    }
    for (unsigned i = 1; i < nv; ++i)
      for (unsigned j = i; j > 0 && v[j - 1] > v[j]; --j) {
        const unsigned t = v[j];
        v[j] = v[j - 1];
        v[j - 1] = t;
      }
    for (unsigned i = 0; i < nv; ++i) cells[(size_t)c * nv + i] = v[i];
    for (unsigned r = 0; r < nv; ++r) {
      unsigned w[3];
      int k = 0;
      for (unsigned i = 0; i < nv; ++i)
        if (i != r) w[k++] = v[i];
      fkey[(size_t)c * nv + r] = face_key(w, cd, fbits);
      fval[(size_t)c * nv + r] = c * nv + r;
    }
  }
}

__global__ void ext_face_flags_kernel(const unsigned long long* __restrict__ k, unsigned n,
                                      unsigned* __restrict__ flag) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    flag[i] = (i == 0 || k[i] != k[i - 1]) ? 1u : 0u;
}

// pos = exclusive scan of the head flags: entry i belongs to face pos[i]
// (a head) or pos[i] - 1
__global__ void ext_face_build_kernel(const unsigned long long* __restrict__ k,
                                      const unsigned* __restrict__ v, const unsigned* __restrict__ pos,
                                      unsigned n, int cd, unsigned long long* __restrict__ fkeys,
                                      unsigned* __restrict__ cof_start, unsigned* __restrict__ cof) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool head = i == 0 || k[i] != k[i - 1];
    const unsigned f = head ? pos[i] : pos[i] - 1;
    if (head) {
      fkeys[f] = k[i];
      cof_start[f] = i;
    }
    if (i == n - 1) cof_start[f + 1] = n;
    cof[i] = v[i] / (unsigned)(cd + 1);
  }
}

// ---------------------------------------------------------------------------
// 1. cull words of every spacetime vertex

template <typename T, int M>
__global__ void __launch_bounds__(256) ext_words_kernel(FieldAccess fa, unsigned long long nv,
                                                        unsigned* __restrict__ words) {
  __shared__ unsigned band_tbl[kBandTable];
  fill_band_table<T>(band_tbl, threadIdx.x, blockDim.x);
  __syncthreads();
  const T* c0 = static_cast<const T*>(fa.comp[0]);
  const T* c1 = static_cast<const T*>(fa.comp[1]);
  const T* c2 = static_cast<const T*>(fa.comp[M == 3 ? 2 : 1]);
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < nv;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned h[M];
    h[0] = hi_word<T>(__ldcs(c0 + i));
    h[1] = hi_word<T>(__ldcs(c1 + i));
    if (M == 3) h[M - 1] = hi_word<T>(__ldcs(c2 + i));
    words[i] = vertex_word_hi<T, M>(h, band_tbl);
  }
}

// ---------------------------------------------------------------------------
// 2. per-simplex exact test

template <typename T, int M>
__device__ __forceinline__ bool ext_test(const FieldAccess& fa, const ExtractConfig& cfg,
                                         const unsigned long long* sidx, double lam_out[4],
                                         float bary_out[4], float& sc_out) {
  T vals[M + 1][M];
#pragma unroll
  for (int i = 0; i <= M; ++i)
#pragma unroll
    for (int j = 0; j < M; ++j) {
      vals[i][j] = static_cast<const T*>(fa.comp[j])[sidx[i]];
      if (cfg.fiber) vals[i][j] = fp<T>::sub(vals[i][j], (T)cfg.fthr[j]);  // values[i][j] - thresholds[j]
    }
  bool inside;
  if constexpr (M == 2) inside = sos_inside2<T>(vals, cfg.Q);
  else inside = sos_inside3<T>(vals, cfg.Q);
  if (!inside) return false;
  T lam[M + 1];
  if (!solve_exact<M, T>(vals, lam)) {
    if (!cfg.fiber) return false;
    // FiberPredicate keeps the simplex at the centroid: (T)1.0 / 3.0
#pragma unroll
    for (int i = 0; i <= M; ++i) lam[i] = (T)((double)(T)1.0 / 3.0);
  }
#pragma unroll
  for (int i = 0; i <= M; ++i) {
    lam_out[i] = (double)lam[i];
    bary_out[i] = (float)lam[i];
  }
  if (fa.has_scalar) {
    using F = fp<T>;
    const T* s = static_cast<const T*>(fa.scalar);
    T sc = T(0);
#pragma unroll
    for (int i = 0; i <= M; ++i) sc = F::add(sc, F::mul(lam[i], s[sidx[i]]));
    sc_out = (float)sc;
  }
  if (cfg.refined) {
    double rr[M + 1];
    if (solve_refined<M, T>(vals, rr))
#pragma unroll
      for (int i = 0; i <= M; ++i) lam_out[i] = rr[i];
  }
  return true;
}

// grid: x over the items of one layer, y = local layer t.  Items of layer t:
// [0, ncell) spatial cells, then (t < L only) [ncell, ncell + nface) base
// faces (m lateral pieces each) and [ncell + nface, 2 ncell + nface) base
// cells (m interior simplices each).  Values and words of local layer l sit
// at storage layer l xor tflip; vertex ids use the global layer t0 + l.
template <typename T, int M>
__global__ void __launch_bounds__(kThreadsX) ext_extract_kernel(ExtMeshDev X, FieldAccess fa,
                                                                const unsigned* __restrict__ words,
                                                                ExtractConfig cfg, ExtSink sink, int vb) {
  const unsigned t = blockIdx.y;
  const unsigned nitems = (t < X.L) ? 2u * X.ncell + X.nface : X.ncell;
  const unsigned first = (X.skip_first_spatial && t == 0) ? X.ncell : 0u;
  const unsigned long long bt = (unsigned long long)(X.t0 + t) * X.ns, bt1 = bt + X.ns;
  const unsigned long long st = (unsigned long long)(t ^ X.tflip) * X.ns;
  const unsigned long long st1 = (unsigned long long)((t + 1) ^ X.tflip) * X.ns;
  const int lane = threadIdx.x & 31;
  const unsigned fmask = (X.fbits >= 32) ? 0xFFFFFFFFu : ((1u << X.fbits) - 1u);
  for (unsigned base = blockIdx.x * kThreadsX; base < nitems; base += gridDim.x * kThreadsX) {
    const unsigned i = base + threadIdx.x;
    const bool valid = i < nitems && i >= first;
    int kind = 0;
    unsigned u[M + 1];
    unsigned wa[M + 1], wb[M + 1];
#pragma unroll
    for (int k = 0; k <= M; ++k) {
      u[k] = 0;
      wa[k] = kAbsent;
      wb[k] = kAbsent;
    }
    if (valid) {
      if (i < X.ncell) {
        kind = 0;
#pragma unroll
        for (int k = 0; k <= M; ++k) u[k] = X.cells[(size_t)i * (M + 1) + k];
      } else if (i < X.ncell + X.nface) {
        kind = 1;
        const unsigned long long key = X.fkeys[i - X.ncell];
#pragma unroll
        for (int k = 0; k < M; ++k) u[k] = (unsigned)(key >> (X.fbits * (M - 1 - k))) & fmask;
      } else {
        kind = 2;
        const unsigned c = i - X.ncell - X.nface;
#pragma unroll
        for (int k = 0; k <= M; ++k) u[k] = X.cells[(size_t)c * (M + 1) + k];
      }
      const int nu = (kind == 1) ? M : M + 1;
#pragma unroll
      for (int k = 0; k <= M; ++k)
        if (k < nu) {
          wa[k] = words[st + u[k]];
          if (kind != 0) wb[k] = words[st1 + u[k]];
        }
    }
#pragma unroll
    for (int p = 0; p < M; ++p) {
      const bool live = valid && (kind != 0 || p == 0);
      unsigned long long vid[M + 1], sidx[M + 1];
      unsigned wacc = kAbsent;
      if (kind == 0) {
#pragma unroll
        for (int k = 0; k <= M; ++k) {
          vid[k] = bt + u[k];
          sidx[k] = st + u[k];
          wacc &= wa[k];
        }
      } else if (kind == 1) {
        // lateral piece j = p: f[0..j]@t, f[j..m-1]@t+1
        int w = 0;
#pragma unroll
        for (int k = 0; k < M; ++k)
          if (k <= p) {
            sidx[w] = st + u[k];
            vid[w++] = bt + u[k];
            wacc &= wa[k];
          }
#pragma unroll
        for (int k = 0; k < M; ++k)
          if (k >= p) {
            sidx[w] = st1 + u[k];
            vid[w++] = bt1 + u[k];
            wacc &= wb[k];
          }
      } else {
        // interior s = p + 1: u[0..s-1]@t, u[s..m]@t+1
#pragma unroll
        for (int k = 0; k <= M; ++k) {
          const bool lo = k <= p;
          vid[k] = (lo ? bt : bt1) + u[k];
          sidx[k] = (lo ? st : st1) + u[k];
          wacc &= lo ? wa[k] : wb[k];
        }
      }
      bool acc = false;
      double lam_out[4] = {0, 0, 0, 0};
      float bary_out[4] = {0.f, 0.f, 0.f, 0.f};
      float sc_out = 0.f;
      // the cull words assume an accepted simplex has a successful solve,
      // which fibers do not require
      if (live && (cfg.fiber || !word_culled(wacc))) acc = ext_test<T, M>(fa, cfg, sidx, lam_out, bary_out, sc_out);
      const unsigned ball = __ballot_sync(0xFFFFFFFFu, acc);
      if (ball) {
        unsigned basei = 0;
        const int leader = __ffs(ball) - 1;
        if (lane == leader) basei = atomicAdd(sink.count, (unsigned)__popc(ball));
        basei = __shfl_sync(0xFFFFFFFFu, basei, leader);
        if (acc) {
          const unsigned idx = basei + __popc(ball & ((1u << lane) - 1));
          if (idx < sink.cap) {
            unsigned long long hi, lo;
            pack_tuple<M>(vid, vb, hi, lo);
            sink.hi[idx] = hi;
            sink.lo[idx] = lo;
            sink.phase[idx] = kind == 2 ? 1u : 0u;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              sink.lam[4 * (size_t)idx + k] = lam_out[k];
              sink.bary4[4 * (size_t)idx + k] = bary_out[k];
            }
            sink.scalar[idx] = sc_out;
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// 3. canonical order

__global__ void ext_gather_by_perm_kernel(const unsigned long long* __restrict__ src,
                                          const unsigned* __restrict__ perm, const unsigned* n_ptr,
                                          unsigned cap, unsigned long long* __restrict__ dst) {
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}

template <int M>
__global__ void ext_finalize_kernel(const unsigned* __restrict__ perm, const unsigned* n_ptr, unsigned cap,
                                    int vb, ExtSink in, unsigned long long* __restrict__ hi_s,
                                    unsigned long long* __restrict__ lo_s, unsigned* __restrict__ phase_s,
                                    double* __restrict__ lam_s, float* __restrict__ sc_s,
                                    unsigned long long* __restrict__ simplices, float* __restrict__ bary) {
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned p = perm[i];
    const unsigned long long h = in.hi[p], l = in.lo[p];
    hi_s[i] = h;
    lo_s[i] = l;
    phase_s[i] = in.phase[p];
#pragma unroll
    for (int k = 0; k < 4; ++k) lam_s[4 * (size_t)i + k] = in.lam[4 * (size_t)p + k];
    sc_s[i] = in.scalar[p];
    unsigned long long v[4];
    unpack_tuple<M>(h, l, vb, v);
#pragma unroll
    for (int k = 0; k <= M; ++k) {
      simplices[(size_t)i * (M + 1) + k] = v[k];
      bary[(size_t)i * (M + 1) + k] = in.bary4[4 * (size_t)p + k];
    }
  }
}

// ---------------------------------------------------------------------------
// 4. star edges and 5. coface unions

struct ExtFeatures {
  const unsigned long long* hi;
  const unsigned long long* lo;
  const unsigned* phase;
  const unsigned* n_ptr;
  unsigned cap;
  int vb;
};

// Calls visit(cell) for every top cell (m+2 ascending vertex ids) that has
// the feature's simplex v[0..m] as a face.
template <int M, typename F>
__device__ __forceinline__ void for_each_coface(const ExtMeshDev& X, const unsigned long long* v, F visit) {
  const unsigned long long ns = X.ns;
  const unsigned long long t = v[0] / ns;
  unsigned long long tl[M + 1];
  unsigned sp[M + 1];
  int n_at_t = 0;
#pragma unroll
  for (int k = 0; k <= M; ++k) {
    tl[k] = v[k] / ns;
    sp[k] = (unsigned)(v[k] - tl[k] * ns);
    n_at_t += tl[k] == t;
  }
  unsigned long long cell[M + 2];
  auto piece = [&](const unsigned* u, unsigned long long tt, int p) {
    int w = 0;
    for (int k = 0; k <= p; ++k) cell[w++] = tt * ns + u[k];
    for (int k = p; k <= M; ++k) cell[w++] = (tt + 1) * ns + u[k];
  };
  if (n_at_t == M + 1) {
    // spatial simplex (a base cell at layer t): piece m of slab t, piece 0 of slab t-1
    if (t < (unsigned long long)X.t0 + X.L) {
      piece(sp, t, M);
      visit(cell);
    }
    if (t > X.t0) {
      piece(sp, t - 1, 0);
      visit(cell);
    }
    return;
  }
  const int j = n_at_t - 1;
  if (sp[j] == sp[j + 1]) {
    // lateral piece j over base face f: piece j + (e <= j) of every cell u
    // containing f, e = position of u's vertex outside f
    unsigned f[M];
    int w = 0;
    for (int k = 0; k <= M; ++k)
      if (k != j + 1) f[w++] = sp[k];
    const long long fi = find_face(X, face_key(f, M, X.fbits));
    if (fi < 0) return;
    for (unsigned q = X.cof_start[fi]; q < X.cof_start[fi + 1]; ++q) {
      const unsigned* u = X.cells + (size_t)X.cof[q] * (M + 1);
      int e = -1, wi = 0;
      for (int k = 0; k <= M; ++k) {
        if (wi < M && u[k] == f[wi]) ++wi;
        else e = k;
      }
      if (e < 0) continue;
      piece(u, t, j + (e <= j ? 1 : 0));
      visit(cell);
    }
  } else {
    // interior s = j + 1 of the prism over base cell sp: pieces s-1 and s
    piece(sp, t, j);
    visit(cell);
    piece(sp, t, j + 1);
    visit(cell);
  }
}

// Indices of the features among the m+2 faces of a top cell.
template <int M>
__device__ __forceinline__ int cell_features(const ExtFeatures& Fs, unsigned n, const unsigned long long* cell,
                                             long long* out) {
  int na = 0;
#pragma unroll
  for (int r = 0; r <= M + 1; ++r) {
    unsigned long long face[M + 1];
    int w = 0;
#pragma unroll
    for (int k = 0; k <= M + 1; ++k)
      if (k != r) face[w++] = cell[k];
    unsigned long long h, l;
    pack_tuple<M>(face, Fs.vb, h, l);
    const long long idx = find_tuple(Fs.hi, Fs.lo, n, h, l);
    if (idx >= 0) out[na++] = idx;
  }
  return na;
}

// pass 0: number of star edges each feature emits as a centre; pass 1: the
// edges themselves, packed (min << 32 | max), at the scanned offsets
template <int M, int PASS>
__global__ void ext_edges_kernel(ExtMeshDev X, ExtFeatures Fs, unsigned* __restrict__ cnt,
                                 const unsigned* __restrict__ off, unsigned long long* __restrict__ ekeys,
                                 unsigned edge_cap, unsigned* err) {
  const unsigned n = min(*Fs.n_ptr, Fs.cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned long long v[4];
    unpack_tuple<M>(Fs.hi[i], Fs.lo[i], Fs.vb, v);
    unsigned others[kMaxOthers];
    int no = 0;
    bool over = false;
    for_each_coface<M>(X, v, [&](const unsigned long long* cell) {
      long long act[M + 2];
      const int na = cell_features<M>(Fs, n, cell, act);
      if (na < 2) return;
      int c = 0;
      for (int a = 1; a < na; ++a) {
        const unsigned pa = Fs.phase[act[a]], pc = Fs.phase[act[c]];
        if (pa < pc || (pa == pc && act[a] < act[c])) c = a;
      }
      if (act[c] != (long long)i) return;
      for (int a = 0; a < na; ++a)
        if (a != c) {
          if (no < kMaxOthers) others[no++] = (unsigned)act[a];
          else over = true;
        }
    });
    if (over) atomicOr(err, kErrCofaces);
    if (PASS == 0) {
      cnt[i] = (unsigned)no;
    } else {
      const unsigned o = off[i];
      for (int a = 0; a < no; ++a)
        if (o + a < edge_cap) {
          const unsigned x = others[a];
          const unsigned lo = min(x, i), hi = max(x, i);
          ekeys[o + a] = ((unsigned long long)lo << 32) | hi;
        }
    }
  }
}

__global__ void ext_unpack_edges_kernel(const unsigned long long* __restrict__ ekeys, const unsigned* ne_ptr,
                                        unsigned edge_cap, unsigned* __restrict__ edges) {
  const unsigned ne = min(*ne_ptr, edge_cap);
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    const unsigned long long k = ekeys[e];
    edges[2 * (size_t)e] = (unsigned)(k >> 32);
    edges[2 * (size_t)e + 1] = (unsigned)k;
  }
}

// 4-D meshes: every non-spatial feature is united with the features among the
// faces of the top cells that ExtrudedSimplicialMesh::cofaces lists for it.
// That routine lifts the base face obtained by dropping the vertex after the
// last layer-t vertex: for a lateral piece that is its own base face (the true
// cofaces); for an interior simplex it is a face of its cell, and the pieces
// of the neighbouring cell across that face join the component as well.
// ids: union-find index of each feature (null: the feature index itself)
__global__ void ext_coface_union_kernel(ExtMeshDev X, ExtFeatures Fs, const unsigned* __restrict__ ids,
                                        unsigned* parent, unsigned* err) {
  constexpr int M = 3;
  const unsigned n = min(*Fs.n_ptr, Fs.cap);
  const unsigned long long ns = X.ns;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned long long v[4];
    unpack_tuple<M>(Fs.hi[i], Fs.lo[i], Fs.vb, v);
    const unsigned long long t = v[0] / ns;
    unsigned sp[4];
    int n_at_t = 0;
    for (int k = 0; k <= M; ++k) {
      const unsigned long long tk = v[k] / ns;
      sp[k] = (unsigned)(v[k] - tk * ns);
      n_at_t += tk == t;
    }
    if (n_at_t == M + 1) continue;  // spatial: its cofaces are its star cells
    const int j0 = n_at_t - 1;
    unsigned bs[3];
    int bi = 0;
    for (int k = 0; k <= j0; ++k) bs[bi++] = sp[k];
    for (int k = j0 + 2; k <= M; ++k) bs[bi++] = sp[k];
    const long long fi = find_face(X, face_key(bs, M, X.fbits));
    if (fi < 0) continue;
    for (unsigned q = X.cof_start[fi]; q < X.cof_start[fi + 1]; ++q) {
      const unsigned* u = X.cells + (size_t)X.cof[q] * (M + 1);
      int e = -1, wi = 0;
      for (int k = 0; k <= M; ++k) {
        if (wi < M && u[k] == bs[wi]) ++wi;
        else e = k;
      }
      if (e < 0) continue;
      const int jp = j0 + (e <= j0 ? 1 : 0);
      unsigned long long cell[5];
      int w = 0;
      for (int k = 0; k <= jp; ++k) cell[w++] = t * ns + u[k];
      for (int k = jp; k <= M; ++k) cell[w++] = (t + 1) * ns + u[k];
      long long act[5];
      const int na = cell_features<M>(Fs, n, cell, act);
      for (int a = 0; a < na; ++a)
        uf_unite(parent, ids ? ids[i] : i, ids ? ids[act[a]] : (unsigned)act[a], err);
    }
  }
}

// ---------------------------------------------------------------------------
// host side

int bits_of(unsigned long long v) {
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b < 1 ? 1 : b;
}

int grid_of(unsigned long long n, int threads, int max_blocks) {
  unsigned long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (unsigned long long)max_blocks) b = max_blocks;
  return (int)b;
}

uint64_t hash_cells(const uint64_t* p, uint64_t n) {
  uint64_t h = 0x9E3779B97F4A7C15ull ^ n;
  for (uint64_t i = 0; i < n; ++i) {
    h ^= p[i] + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    h *= 0xBF58476D1CE4E5B9ull;
  }
  return h;
}

ftk2b_status ext_fail(ftk2b_ctx* ctx, ftk2b_status st, const std::string& msg) {
  ctx->err = msg;
  return st;
}

#define EXT_TRY(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return ext_fail(ctx, e_ == cudaErrorMemoryAllocation ? FTK2B_OOM : FTK2B_CUDA_ERROR,          \
                      std::string(#call) + " failed: " + cudaGetErrorString(e_));                  \
  } while (0)

ftk2b_status validate_mesh(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, int* fbits) {
  const int cd = mesh->base_cell_dim;
  if (cd != 2 && cd != 3)
    return ext_fail(ctx, FTK2B_UNSUPPORTED, "extruded meshes need triangle (2) or tet (3) base cells");
  if (mesh->n_base_verts < 1) return ext_fail(ctx, FTK2B_INVALID_ARG, "extruded mesh without base vertices");
  if (mesh->n_base_cells > 0 && !mesh->base_cells)
    return ext_fail(ctx, FTK2B_INVALID_ARG, "base_cells is null");
  if (mesh->n_base_cells * (uint64_t)(cd + 1) >= (1ull << 31))
    return ext_fail(ctx, FTK2B_UNSUPPORTED, "more than 2^31 base cell vertices");
  if (mesh->n_layers >= 65535) return ext_fail(ctx, FTK2B_UNSUPPORTED, "n_layers must be below 65535");
  if (mesh->n_base_verts * (mesh->n_layers + 1) > 0xFFFFFFFFull)
    return ext_fail(ctx, FTK2B_UNSUPPORTED, "spacetime vertex ids exceed 32 bits");
  *fbits = bits_of(mesh->n_base_verts - 1);
  if (*fbits * cd > 64)
    return ext_fail(ctx, FTK2B_UNSUPPORTED, "base vertex ids too wide to pack a face into 64 bits");
  return FTK2B_OK;
}

// Builds (or reuses) the device copy of the base mesh.
ftk2b_status prepare_base(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, int fbits, unsigned long long* nl,
                          const uint64_t* known_hash = nullptr) {
  ExtCache& C = ctx->ext;
  const int cd = mesh->base_cell_dim;
  const uint64_t nent64 = mesh->n_base_cells * (uint64_t)(cd + 1);
  const uint64_t h = known_hash ? *known_hash : hash_cells(mesh->base_cells, nent64);
  if (C.valid && C.hash == h && C.ncell == mesh->n_base_cells && C.ns == mesh->n_base_verts && C.cd == cd)
    return FTK2B_OK;
  C.valid = false;
  const unsigned nent = (unsigned)nent64;
  const unsigned ncell = (unsigned)mesh->n_base_cells;
  const size_t ne = nent ? nent : 1;
  EXT_TRY(C.cells.ensure(sizeof(unsigned) * ne));
  EXT_TRY(C.fkeys.ensure(sizeof(unsigned long long) * ne));
  EXT_TRY(C.cof_start.ensure(sizeof(unsigned) * (ne + 1)));
  EXT_TRY(C.cof.ensure(sizeof(unsigned) * ne));
  EXT_TRY(C.ekeys.ensure(sizeof(unsigned long long) * ne));
  EXT_TRY(C.sort_k.ensure(sizeof(unsigned long long) * ne));
  EXT_TRY(C.sort_k2.ensure(sizeof(unsigned long long) * ne));
  EXT_TRY(C.sort_v.ensure(sizeof(unsigned) * ne));
  EXT_TRY(C.sort_v2.ensure(sizeof(unsigned) * ne));
  EXT_TRY(ctx->counters.ensure(sizeof(unsigned) * kNumCounters));
  const int sgrid = ctx->sort_grid(nent);
  EXT_TRY(ctx->hist.ensure(sizeof(unsigned) * 256 * (size_t)(sgrid > 1 ? sgrid : 1) + 1024));
  cudaStream_t st = ctx->stream;
  unsigned* counters = (unsigned*)ctx->counters.p;
  EXT_TRY(cudaMemsetAsync(counters, 0, sizeof(unsigned) * kNumCounters, st));
  unsigned nface = 0;
  if (nent) {
    EXT_TRY(cudaMemcpyAsync(C.ekeys.p, mesh->base_cells, sizeof(uint64_t) * nent, cudaMemcpyHostToDevice, st));
    ext_prep_cells_kernel<<<grid_of(ncell, 256, 8 * ctx->num_sms), 256, 0, st>>>(
        (const unsigned long long*)C.ekeys.p, ncell, cd, (unsigned)mesh->n_base_verts, fbits,
        (unsigned*)C.cells.p, (unsigned long long*)C.sort_k.p, (unsigned*)C.sort_v.p, counters,
        counters + kCountErr);
    *nl += 1;
    const bool alt = radix_sort((unsigned long long*)C.sort_k.p, (unsigned*)C.sort_v.p,
                                (unsigned long long*)C.sort_k2.p, (unsigned*)C.sort_v2.p,
                                counters + kCountPrepEntries, nent, fbits * cd, (unsigned*)ctx->hist.p,
                                sgrid, st, nl);
    const unsigned long long* k = (const unsigned long long*)(alt ? C.sort_k2.p : C.sort_k.p);
    const unsigned* v = (const unsigned*)(alt ? C.sort_v2.p : C.sort_v.p);
    unsigned* flags = (unsigned*)(alt ? C.sort_v.p : C.sort_v2.p);
    const int g = grid_of(nent, 256, 16 * ctx->num_sms);
    ext_face_flags_kernel<<<g, 256, 0, st>>>(k, nent, flags);
    EXT_TRY(launch_scan(flags, nent, counters + kCountFaces, nullptr, st));
    ext_face_build_kernel<<<g, 256, 0, st>>>(k, v, flags, nent, cd, (unsigned long long*)C.fkeys.p,
                                             (unsigned*)C.cof_start.p, (unsigned*)C.cof.p);
    *nl += 3;
    EXT_TRY(cudaGetLastError());
    EXT_TRY(cudaMemcpyAsync(ctx->h_counters, counters, sizeof(unsigned) * kNumCounters,
                            cudaMemcpyDeviceToHost, st));
    EXT_TRY(ctx->sync());
    if (ctx->h_counters[kCountErr] & kErrBadVertex)
      return ext_fail(ctx, FTK2B_INVALID_ARG, "a base cell lists a vertex id >= n_base_verts");
    nface = ctx->h_counters[kCountFaces];
  }
  C.hash = h;
  C.ncell = mesh->n_base_cells;
  C.ns = mesh->n_base_verts;
  C.cd = cd;
  C.nface = nface;
  C.fbits = fbits;
  C.valid = true;
  return FTK2B_OK;
}

template <typename T, int M>
cudaError_t enqueue_extract(ftk2b_ctx* ctx, const ExtMeshDev& X, const FieldAccess& fa,
                            const ExtractConfig& cfg, const ExtSink& sink, int vb, unsigned long long nv,
                            unsigned long long* nl) {
  cudaStream_t st = ctx->stream;
  ext_words_kernel<T, M><<<grid_of(nv, 256, 32 * ctx->num_sms), 256, 0, st>>>(fa, nv,
                                                                              (unsigned*)ctx->ext.words.p);
  const unsigned long long items = 2ull * X.ncell + X.nface;
  dim3 grid((unsigned)grid_of(items, kThreadsX, 1 << 20), X.L + 1);
  ext_extract_kernel<T, M><<<grid, kThreadsX, 0, st>>>(X, fa, (const unsigned*)ctx->ext.words.p, cfg, sink, vb);
  *nl += 2;
  return cudaGetLastError();
}

template <int M>
cudaError_t enqueue_post(ftk2b_ctx* ctx, const ExtMeshDev& X, const ExtSink& sink, unsigned cap,
                         unsigned edge_cap, int vb, int want_edges, unsigned long long* nl) {
  cudaStream_t st = ctx->stream;
  ExtCache& C = ctx->ext;
  unsigned* counters = (unsigned*)ctx->counters.p;
  unsigned* count = counters + kCountFeatures;
  const int sgrid = ctx->sort_grid(cap);
  unsigned* hist = (unsigned*)ctx->hist.p;
  const int g = grid_of(cap, 256, 4096);
  cudaError_t e;
  // canonical order: stable sort by the low word, then by the high word
  if ((e = cudaMemcpyAsync(C.sort_k.p, sink.lo, sizeof(unsigned long long) * cap, cudaMemcpyDeviceToDevice, st)))
    return e;
  if ((e = launch_iota((unsigned*)ctx->perm0.p, count, cap, st))) return e;
  const int lo_bits = (M == 3) ? 2 * vb : vb;
  bool alt = radix_sort((unsigned long long*)C.sort_k.p, (unsigned*)ctx->perm0.p,
                        (unsigned long long*)C.sort_k2.p, (unsigned*)ctx->perm1.p, count, cap, lo_bits,
                        hist, sgrid, st, nl);
  unsigned* p1 = (unsigned*)(alt ? ctx->perm1.p : ctx->perm0.p);
  unsigned* p1_other = (unsigned*)(alt ? ctx->perm0.p : ctx->perm1.p);
  ext_gather_by_perm_kernel<<<g, 256, 0, st>>>(sink.hi, p1, count, cap, (unsigned long long*)C.sort_k.p);
  alt = radix_sort((unsigned long long*)C.sort_k.p, p1, (unsigned long long*)C.sort_k2.p, p1_other, count, cap,
                   2 * vb, hist, sgrid, st, nl);
  const unsigned* perm = alt ? p1_other : p1;
  ext_finalize_kernel<M><<<g, 256, 0, st>>>(perm, count, cap, vb, sink, (unsigned long long*)C.hi_s.p,
                                            (unsigned long long*)C.lo_s.p, (unsigned*)C.phase_s.p,
                                            (double*)ctx->lam_s.p, (float*)ctx->scalar_s.p,
                                            (unsigned long long*)ctx->simplices.p, (float*)ctx->bary.p);
  *nl += 3;  // iota, gather, finalize
  if (!want_edges) return cudaGetLastError();
  ExtFeatures Fs;
  Fs.hi = (const unsigned long long*)C.hi_s.p;
  Fs.lo = (const unsigned long long*)C.lo_s.p;
  Fs.phase = (const unsigned*)C.phase_s.p;
  Fs.n_ptr = count;
  Fs.cap = cap;
  Fs.vb = vb;
  unsigned* err = counters + kCountErr;
  unsigned* n_edges = counters + kCountEdges;
  unsigned* ecnt = (unsigned*)ctx->edge_cnt.p;
  unsigned long long* ekeys = (unsigned long long*)C.ekeys.p;
  ext_edges_kernel<M, 0><<<g, 256, 0, st>>>(X, Fs, ecnt, nullptr, ekeys, edge_cap, err);
  if ((e = launch_scan(ecnt, cap, n_edges, count, st))) return e;
  ext_edges_kernel<M, 1><<<g, 256, 0, st>>>(X, Fs, nullptr, ecnt, ekeys, edge_cap, err);
  // (min, max) pairs sorted lexicographically; a pair spans exactly one top
  // cell, so there are no duplicates
  const int eb = 2 * 32;
  const bool ealt = radix_sort(ekeys, (unsigned*)C.sort_v.p, (unsigned long long*)C.sort_k2.p,
                               (unsigned*)C.sort_v2.p, n_edges, edge_cap, eb, hist, ctx->sort_grid(edge_cap), st,
                               nl);
  const unsigned long long* es = ealt ? (const unsigned long long*)C.sort_k2.p : ekeys;
  ext_unpack_edges_kernel<<<grid_of(edge_cap, 256, 4096), 256, 0, st>>>(es, n_edges, edge_cap,
                                                                       (unsigned*)ctx->edges.p);
  if ((e = launch_uf((unsigned*)ctx->parent.p, count, cap, (const unsigned*)ctx->edges.p, n_edges, edge_cap, err,
                     st)))
    return e;
  if (M == 3) ext_coface_union_kernel<<<g, 256, 0, st>>>(X, Fs, nullptr, (unsigned*)ctx->parent.p, err);
  if ((e = launch_uf_label((unsigned*)ctx->parent.p, count, cap, (unsigned long long*)ctx->track.p,
                           counters + kCountRoots, st)))
    return e;
  *nl += 8 + (M == 3 ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace

}  // namespace ftk2b

using namespace ftk2b;

// ---------------------------------------------------------------------------
// extruded time streams (the driver and its contract: cp_stream.cu)

namespace ftk2b {
namespace {

enum { kSWin = 5, kSWinEdges = 6, kSPrev = 7 };
constexpr int kStreamVb = 32;  // fixed id width of a stream's packed tuples

__global__ void ext_window_build_kernel(const unsigned long long* __restrict__ lo, const unsigned* __restrict__ prev,
                                        unsigned n_prev, unsigned first_new, unsigned n_new,
                                        unsigned long long* __restrict__ k_out, unsigned* __restrict__ id_out) {
  const unsigned nS = n_prev + n_new;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < nS; i += gridDim.x * blockDim.x) {
    const unsigned id = i < n_prev ? prev[i] : first_new + (i - n_prev);
    k_out[i] = lo[id];
    id_out[i] = id;
  }
}

__global__ void ext_gather_key_kernel(const unsigned long long* __restrict__ src, const unsigned* __restrict__ ids,
                                      const unsigned* n_ptr, unsigned cap, unsigned long long* __restrict__ dst) {
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[ids[i]];
}

__global__ void ext_window_fill_kernel(const unsigned* __restrict__ ids, const unsigned* n_ptr, unsigned cap,
                                       const unsigned long long* __restrict__ hi,
                                       const unsigned long long* __restrict__ lo, const unsigned* __restrict__ phase,
                                       unsigned long long* __restrict__ hi_s, unsigned long long* __restrict__ lo_s,
                                       unsigned* __restrict__ phase_s) {
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned id = ids[i];
    hi_s[i] = hi[id];
    lo_s[i] = lo[id];
    phase_s[i] = phase[id];
  }
}

// window star edges (packed window indices) -> stream ids, united and stored
__global__ void ext_append_edges_kernel(const unsigned long long* __restrict__ ek, const unsigned* n_ptr,
                                        unsigned cap, const unsigned* __restrict__ ids, unsigned* parent,
                                        unsigned* __restrict__ out, unsigned base, unsigned out_cap, unsigned* err) {
  const unsigned n = min(*n_ptr, cap);
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const unsigned a = ids[(unsigned)(ek[e] >> 32)], b = ids[(unsigned)ek[e]];
    uf_unite(parent, a, b, err);
    if (base + e < out_cap) {
      out[2 * (size_t)(base + e)] = a;
      out[2 * (size_t)(base + e) + 1] = b;
    }
  }
}

template <int M>
__global__ void ext_collect_spatial_kernel(const unsigned long long* __restrict__ hi,
                                           const unsigned long long* __restrict__ lo, unsigned first_new,
                                           unsigned n_new, unsigned long long ns, unsigned long long t,
                                           unsigned* __restrict__ prev, unsigned* prev_n) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += gridDim.x * blockDim.x) {
    const unsigned id = first_new + i;
    unsigned long long v[4];
    unpack_tuple<M>(hi[id], lo[id], kStreamVb, v);
    if (v[0] / ns == t && v[M] / ns == t) prev[atomicAdd(prev_n, 1u)] = id;
  }
}

template <int M>
__global__ void ext_stream_expand_kernel(const unsigned* __restrict__ perm, unsigned n,
                                         const unsigned long long* __restrict__ hi,
                                         const unsigned long long* __restrict__ lo, const float* __restrict__ bary4_s,
                                         unsigned long long* __restrict__ simplices, float* __restrict__ bary) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned p = perm[i];
    unsigned long long v[4];
    unpack_tuple<M>(hi[p], lo[p], kStreamVb, v);
    for (int k = 0; k <= M; ++k) {
      simplices[(size_t)i * (M + 1) + k] = v[k];
      bary[(size_t)i * (M + 1) + k] = bary4_s[4 * (size_t)i + k];
    }
  }
}

ExtMeshDev stream_mesh(ftk2b_ctx* ctx, const ftk2b_stream* s, unsigned t0, unsigned L) {
  ExtCache& C = ctx->ext;
  ExtMeshDev X;
  X.cd = s->m;
  X.ns = (unsigned)s->emesh.n_base_verts;
  X.L = L;
  X.t0 = t0;
  X.tflip = t0 & 1u;
  X.skip_first_spatial = 0;
  X.ncell = (unsigned)C.ncell;
  X.nface = C.nface;
  X.fbits = C.fbits;
  X.cells = (const unsigned*)C.cells.p;
  X.fkeys = (const unsigned long long*)C.fkeys.p;
  X.cof_start = (const unsigned*)C.cof_start.p;
  X.cof = (const unsigned*)C.cof.p;
  return X;
}

// sorts ids [0, n) (in k0/v0 order of the window or store) by (hi, lo);
// returns the buffer holding the sorted ids
unsigned* sort_by_tuple(ftk2b_ctx* ctx, ftk2b_stream* s, const unsigned* n_ptr, unsigned cap, int bits,
                        unsigned long long* nl) {
  cudaStream_t st = ctx->stream;
  const int sgrid = ctx->sort_grid(cap);
  unsigned* hist = (unsigned*)ctx->hist.p;
  bool alt = radix_sort((unsigned long long*)s->s_key.p, (unsigned*)s->s_id.p, (unsigned long long*)s->s_key2.p,
                        (unsigned*)s->s_id2.p, n_ptr, cap, bits, hist, sgrid, st, nl);
  unsigned* ids = (unsigned*)(alt ? s->s_id2.p : s->s_id.p);
  unsigned* ids_other = (unsigned*)(alt ? s->s_id.p : s->s_id2.p);
  unsigned long long* kfree = (unsigned long long*)(alt ? s->s_key.p : s->s_key2.p);
  unsigned long long* kother = (unsigned long long*)(alt ? s->s_key2.p : s->s_key.p);
  ext_gather_key_kernel<<<grid_of(cap, 256, 4096), 256, 0, st>>>((const unsigned long long*)s->hi.p, ids, n_ptr, cap,
                                                                 kfree);
  alt = radix_sort(kfree, ids, kother, ids_other, n_ptr, cap, bits, hist, sgrid, st, nl);
  *nl += 1;
  return alt ? ids_other : ids;
}

template <typename T, int M>
ftk2b_status push_extruded_t(ftk2b_stream* s) {
  ftk2b_ctx* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  unsigned long long nl = 0;
  int fbits = 0;
  ftk2b_status rc = validate_mesh(ctx, &s->emesh, &fbits);
  if (rc) return rc;
  const uint64_t tnow = s->T;
  const unsigned long long ns = s->emesh.n_base_verts;
  if (ns * (tnow + 1) > 0xFFFFFFFFull) return ext_fail(ctx, FTK2B_UNSUPPORTED, "spacetime vertex ids exceed 32 bits");
  rc = prepare_base(ctx, &s->emesh, fbits, &nl, &s->ebase_hash);
  if (rc) return rc;
  const unsigned t0 = tnow ? (unsigned)(tnow - 1) : 0u, L = tnow ? 1u : 0u;
  ExtMeshDev X = stream_mesh(ctx, s, t0, L);
  X.skip_first_spatial = tnow > 0;
  FieldAccess fa;
  memset(&fa, 0, sizeof(fa));
  fa.per_vertex = 1;
  for (int j = 0; j < M; ++j) fa.comp[j] = s->ring[j].p;
  ExtractConfig cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.Q = s->prm.sos_q;
  cfg.refined = s->prm.precision == FTK2B_PRECISION_REFINED;
  const unsigned long long nv = ns * (L + 1);
  ExtCache& C = ctx->ext;
  EXT_TRY(C.words.ensure(sizeof(unsigned) * nv));
  EXT_TRY(ctx->counters.ensure(sizeof(unsigned) * kNumCounters));
  unsigned* counters = (unsigned*)ctx->counters.p;
  unsigned n_new = 0;
  for (int attempt = 0;; ++attempt) {
    if (attempt == 6) return ext_fail(ctx, FTK2B_OVERFLOW_RETRY, "stream buffers kept overflowing");
    if (s->cap < s->n + 1024) {
      rc = ensure_stream_store(s, s->n + 1024);
      if (rc) return rc;
    }
    EXT_TRY(cudaMemsetAsync(counters, 0, sizeof(unsigned) * kNumCounters, st));
    ExtSink sink;
    sink.hi = (unsigned long long*)s->hi.p + s->n;
    sink.lo = (unsigned long long*)s->lo.p + s->n;
    sink.phase = (unsigned*)s->phase.p + s->n;
    sink.lam = (double*)s->lam.p + 4 * (size_t)s->n;
    sink.bary4 = (float*)s->bary4.p + 4 * (size_t)s->n;
    sink.scalar = (float*)s->scalar.p + s->n;
    sink.count = counters + kCountFeatures;
    sink.cap = s->cap - s->n;
    EXT_TRY((enqueue_extract<T, M>(ctx, X, fa, cfg, sink, kStreamVb, nv, &nl)));
    EXT_TRY(cudaMemcpyAsync(ctx->h_counters, counters, sizeof(unsigned) * kNumCounters, cudaMemcpyDeviceToHost, st));
    EXT_TRY(ctx->sync());
    const unsigned got = ctx->h_counters[kCountFeatures];
    if (got > s->cap - s->n) {
      rc = ensure_stream_store(s, s->n + got + got / 4 + 1024);
      if (rc) return rc;
      continue;
    }
    n_new = got;
    break;
  }

  // window: spatial features of layer t-1 plus the new ones, in Simplex order
  const unsigned first_new = s->n;
  const unsigned nS = s->n_prev + n_new;
  const unsigned wcap = nS ? nS : 1;
  const unsigned wecap = kMaxOthers * wcap;
  EXT_TRY(s->s_key.ensure(8 * (size_t)wcap));
  EXT_TRY(s->s_key2.ensure(8 * (size_t)wcap));
  EXT_TRY(s->s_id.ensure(4 * (size_t)wcap));
  EXT_TRY(s->s_id2.ensure(4 * (size_t)wcap));
  EXT_TRY(s->s_hi.ensure(8 * (size_t)wcap));
  EXT_TRY(s->s_lo.ensure(8 * (size_t)wcap));
  EXT_TRY(s->s_phase.ensure(4 * (size_t)wcap));
  EXT_TRY(s->wedges.ensure(8 * (size_t)wecap));
  EXT_TRY(ctx->edge_cnt.ensure(4 * (size_t)wcap));
  EXT_TRY(ctx->hist.ensure(sizeof(unsigned) * 256 * (size_t)ctx->sort_grid(wcap > wecap ? wcap : wecap)));
  const unsigned edge_room = s->n_edges + wecap;
  if (edge_room > s->edge_cap) {
    unsigned nc = s->edge_cap ? s->edge_cap : 262144u;
    while (nc < edge_room) nc *= 2;
    EXT_TRY(grow_keep(s->edges, 8 * (size_t)s->n_edges, 8 * (size_t)nc, st));
    s->edge_cap = nc;
  }
  const int g = grid_of(wcap, 256, 4096);
  set_u32_kernel<<<1, 1, 0, st>>>(counters + kSWin, nS);
  ext_window_build_kernel<<<g, 256, 0, st>>>((const unsigned long long*)s->lo.p, (const unsigned*)s->prev_ids.p,
                                             s->n_prev, first_new, n_new, (unsigned long long*)s->s_key.p,
                                             (unsigned*)s->s_id.p);
  const int bits = kStreamVb + bits_of(ns * (tnow + 1));
  const unsigned* ids = sort_by_tuple(ctx, s, counters + kSWin, wcap, bits, &nl);
  ext_window_fill_kernel<<<g, 256, 0, st>>>(ids, counters + kSWin, wcap, (const unsigned long long*)s->hi.p,
                                            (const unsigned long long*)s->lo.p, (const unsigned*)s->phase.p,
                                            (unsigned long long*)s->s_hi.p, (unsigned long long*)s->s_lo.p,
                                            (unsigned*)s->s_phase.p);
  ExtFeatures Fs;
  Fs.hi = (const unsigned long long*)s->s_hi.p;
  Fs.lo = (const unsigned long long*)s->s_lo.p;
  Fs.phase = (const unsigned*)s->s_phase.p;
  Fs.n_ptr = counters + kSWin;
  Fs.cap = wcap;
  Fs.vb = kStreamVb;
  unsigned* err = counters + kCountErr;
  unsigned* ecnt = (unsigned*)ctx->edge_cnt.p;
  unsigned long long* ek = (unsigned long long*)s->wedges.p;
  ext_edges_kernel<M, 0><<<g, 256, 0, st>>>(X, Fs, ecnt, nullptr, ek, wecap, err);
  EXT_TRY(launch_scan(ecnt, wcap, counters + kSWinEdges, counters + kSWin, st));
  ext_edges_kernel<M, 1><<<g, 256, 0, st>>>(X, Fs, nullptr, ecnt, ek, wecap, err);
  if (n_new) uf_init_range_kernel<<<grid_of(n_new, 256, 4096), 256, 0, st>>>((unsigned*)s->parent.p, first_new, n_new);
  ext_append_edges_kernel<<<grid_of(wecap, 256, 4096), 256, 0, st>>>(ek, counters + kSWinEdges, wecap, ids,
                                                                    (unsigned*)s->parent.p, (unsigned*)s->edges.p,
                                                                    s->n_edges, s->edge_cap, err);
  if (M == 3) ext_coface_union_kernel<<<g, 256, 0, st>>>(X, Fs, ids, (unsigned*)s->parent.p, err);
  if (n_new)
    ext_collect_spatial_kernel<M><<<grid_of(n_new, 256, 4096), 256, 0, st>>>(
        (const unsigned long long*)s->hi.p, (const unsigned long long*)s->lo.p, first_new, n_new, ns, tnow,
        (unsigned*)s->prev_ids2.p, counters + kSPrev);
  nl += 9;
  EXT_TRY(cudaGetLastError());
  EXT_TRY(cudaMemcpyAsync(ctx->h_counters, counters, sizeof(unsigned) * kNumCounters, cudaMemcpyDeviceToHost, st));
  EXT_TRY(ctx->sync());
  ctx->launches += nl;
  const unsigned* h = ctx->h_counters;
  if (h[kCountErr] & kErrCofaces) return ext_fail(ctx, FTK2B_UNSUPPORTED, "a base face has more than 8 coface cells");
  if (h[kCountErr] & 1u) return ext_fail(ctx, FTK2B_TIMEOUT, "union-find retry bound reached");
  s->n_edges += h[kSWinEdges];
  s->n_prev = h[kSPrev];
  std::swap(s->prev_ids, s->prev_ids2);
  s->n += n_new;
  if (tnow == 0) s->n_first = n_new;
  s->last_new = n_new;
  return FTK2B_OK;
}

template <int M>
ftk2b_status result_extruded_t(ftk2b_stream* s, ftk2b_cp_result** out) {
  ftk2b_ctx* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  unsigned long long nl = 0;
  const unsigned n = s->n, ne = s->n_edges;
  const unsigned nc = n ? n : 1, ec = ne ? ne : 1, mc = nc > ec ? nc : ec;
  EXT_TRY(ctx->counters.ensure(sizeof(unsigned) * kNumCounters));
  unsigned* counters = (unsigned*)ctx->counters.p;
  EXT_TRY(s->s_key.ensure(8 * (size_t)mc));
  EXT_TRY(s->s_key2.ensure(8 * (size_t)mc));
  EXT_TRY(s->s_id.ensure(4 * (size_t)mc));
  EXT_TRY(s->s_id2.ensure(4 * (size_t)mc));
  EXT_TRY(ctx->perm0.ensure(4 * (size_t)nc));
  EXT_TRY(ctx->perm1.ensure(4 * (size_t)nc));
  EXT_TRY(ctx->parent.ensure(4 * (size_t)nc));
  EXT_TRY(ctx->lam_s.ensure(32 * (size_t)nc));
  EXT_TRY(ctx->bary4_s.ensure(16 * (size_t)nc));
  EXT_TRY(ctx->scalar_s.ensure(4 * (size_t)nc));
  EXT_TRY(ctx->cls.ensure(4 * (size_t)nc));
  EXT_TRY(ctx->track.ensure(8 * (size_t)nc));
  EXT_TRY(ctx->simplices.ensure(8 * (size_t)(M + 1) * nc));
  EXT_TRY(ctx->bary.ensure(4 * (size_t)(M + 1) * nc));
  EXT_TRY(ctx->edges.ensure(8 * (size_t)ec));
  EXT_TRY(ctx->hist.ensure(sizeof(unsigned) * 256 * (size_t)ctx->sort_grid(mc)));
  const int g = grid_of(mc, 256, 4096);
  EXT_TRY(cudaMemsetAsync(counters, 0, sizeof(unsigned) * kNumCounters, st));
  set_u32_kernel<<<1, 1, 0, st>>>(counters + kSWin, n);
  set_u32_kernel<<<1, 1, 0, st>>>(counters + kSWinEdges, ne);
  if (n) EXT_TRY(cudaMemcpyAsync(s->s_key.p, s->lo.p, 8 * (size_t)n, cudaMemcpyDeviceToDevice, st));
  iota_u32_kernel<<<g, 256, 0, st>>>((unsigned*)s->s_id.p, n);
  const unsigned long long ns = s->emesh.n_base_verts;
  const unsigned* perm = sort_by_tuple(ctx, s, counters + kSWin, nc, kStreamVb + bits_of(ns * (s->T + 1)), &nl);
  unsigned* inv = (unsigned*)ctx->perm0.p;
  unsigned* root = (unsigned*)ctx->perm1.p;
  unsigned* cmin = (unsigned*)ctx->parent.p;
  invert_kernel<<<g, 256, 0, st>>>(perm, n, inv);
  fill_u32_kernel<<<g, 256, 0, st>>>(cmin, n, 0xFFFFFFFFu);
  comp_min_kernel<<<g, 256, 0, st>>>((unsigned*)s->parent.p, inv, n, root, cmin, counters + kCountRoots);
  gather_result_kernel<<<g, 256, 0, st>>>(perm, n, root, cmin, (const double*)s->lam.p, (const float*)s->bary4.p,
                                          (const float*)s->scalar.p, (const unsigned*)s->cls.p, (double*)ctx->lam_s.p,
                                          (float*)ctx->bary4_s.p, (float*)ctx->scalar_s.p, (unsigned*)ctx->cls.p,
                                          (unsigned long long*)ctx->track.p);
  ext_stream_expand_kernel<M><<<g, 256, 0, st>>>(perm, n, (const unsigned long long*)s->hi.p,
                                                 (const unsigned long long*)s->lo.p, (const float*)ctx->bary4_s.p,
                                                 (unsigned long long*)ctx->simplices.p, (float*)ctx->bary.p);
  // edges in canonical ids, sorted; the id buffers are free after the gathers
  unsigned long long* ek = (unsigned long long*)(perm == (const unsigned*)s->s_id.p ? s->s_key2.p : s->s_key.p);
  unsigned long long* ek2 = (unsigned long long*)(perm == (const unsigned*)s->s_id.p ? s->s_key.p : s->s_key2.p);
  canon_edges_kernel<<<g, 256, 0, st>>>((const unsigned*)s->edges.p, ne, inv, ek);
  const bool ealt = radix_sort(ek, (unsigned*)s->s_id.p, ek2, (unsigned*)s->s_id2.p, counters + kSWinEdges, ec, 64,
                               (unsigned*)ctx->hist.p, ctx->sort_grid(mc), st, &nl);
  unpack_edges_kernel<<<g, 256, 0, st>>>(ealt ? ek2 : ek, ne, (unsigned*)ctx->edges.p);
  nl += 8;
  EXT_TRY(cudaGetLastError());
  EXT_TRY(cudaMemcpyAsync(ctx->h_counters, counters, sizeof(unsigned) * kNumCounters, cudaMemcpyDeviceToHost, st));
  EXT_TRY(ctx->sync());
  ctx->launches += nl;
  ctx->last.kind = FTK2B_MESH_EXTRUDED;
  ctx->last.m = M;
  ctx->last.f64 = s->dtype == FTK2B_F64;
  ctx->last.n = n;
  ctx->last.ne = s->prm.want_edges ? ne : 0;
  ctx->last.n_roots = ctx->h_counters[kCountRoots];
  // m-simplices of the T-timestep mesh, from the prepared base mesh's counts
  const uint64_t L = s->T ? s->T - 1 : 0;
  ctx->last.n_simplices =
      s->T ? ctx->ext.ncell * (L + 1) + (uint64_t)ctx->ext.nface * L * M + ctx->ext.ncell * L * M : 0;
  ctx->last.device_ms = 0;
  ctx->last.classify = 0;
  ctx->last.want_edges = s->prm.want_edges;
  return ftk2b_cp_fetch(ctx, out);
}

}  // namespace

uint64_t hash_base_cells(const uint64_t* p, uint64_t n) { return hash_cells(p, n); }

}  // namespace ftk2b

ftk2b_status stream_push_extruded(ftk2b_stream* s) {
  if (s->prm.classify) {
    s->ctx->err = "classification of extruded meshes is not available";
    return FTK2B_UNSUPPORTED;
  }
  const bool f64 = s->dtype == FTK2B_F64;
  if (s->m == 3) return f64 ? push_extruded_t<double, 3>(s) : push_extruded_t<float, 3>(s);
  return f64 ? push_extruded_t<double, 2>(s) : push_extruded_t<float, 2>(s);
}

ftk2b_status stream_result_extruded(ftk2b_stream* s, ftk2b_cp_result** out) {
  return s->m == 3 ? result_extruded_t<3>(s, out) : result_extruded_t<2>(s, out);
}

uint64_t extruded_simplex_count(const ftk2b_mesh_desc* mesh, int m) {
  const int cd = mesh->base_cell_dim;
  if ((cd != 2 && cd != 3) || m != cd || (mesh->n_base_cells && !mesh->base_cells)) return 0;
  // unique (cd-1)-faces of the base, counted on the host from packed keys
  // (base vertex ids below 2^21 for tets, 2^32 for triangles; wider ids are
  // not supported by the extruded path either)
  const int fbits = bits_of(mesh->n_base_verts ? mesh->n_base_verts - 1 : 0);
  if (fbits * cd > 64) return 0;
  std::vector<uint64_t> keys;
  keys.reserve(mesh->n_base_cells * (cd + 1));
  for (uint64_t c = 0; c < mesh->n_base_cells; ++c) {
    uint64_t v[4];
    for (int i = 0; i <= cd; ++i) v[i] = mesh->base_cells[c * (cd + 1) + i];
    std::sort(v, v + cd + 1);
    for (int r = 0; r <= cd; ++r) {
      uint64_t k = 0;
      for (int i = 0; i <= cd; ++i)
        if (i != r) k = (k << fbits) | v[i];
      keys.push_back(k);
    }
  }
  std::sort(keys.begin(), keys.end());
  const uint64_t nface = (uint64_t)(std::unique(keys.begin(), keys.end()) - keys.begin());
  const uint64_t L = mesh->n_layers;
  return mesh->n_base_cells * (L + 1) + nface * L * cd + mesh->n_base_cells * L * cd;
}

ftk2b_status run_extruded(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* field,
                          const ftk2b_cp_params* prm, const double* fiber_thr) {
  int fbits = 0;
  ftk2b_status st = validate_mesh(ctx, mesh, &fbits);
  if (st) return st;
  const int M = mesh->base_cell_dim;
  if (field->ncomp != M)
    return ext_fail(ctx, FTK2B_INVALID_ARG, "an extruded mesh over dimension-" + std::to_string(M) +
                                                " cells needs " + std::to_string(M) + " components");
  if (field->layout == FTK2B_LAYOUT_MULTICOMPONENT)
    return ext_fail(ctx, FTK2B_UNSUPPORTED,
                    "extruded meshes take per-vertex arrays (the reference indexes multicomponent arrays "
                    "by grid coordinates, which an unstructured mesh does not have)");
  if (field->layout == FTK2B_LAYOUT_SEPARATE && field->nd != 1)
    return ext_fail(ctx, FTK2B_INVALID_ARG, "extruded meshes take 1-D per-vertex arrays");
  const unsigned ns = (unsigned)mesh->n_base_verts;
  const unsigned L = (unsigned)mesh->n_layers;
  const unsigned long long nv = (unsigned long long)ns * (L + 1);
  FieldAccess fa;
  st = prepare_field(ctx, field, 1, nullptr, nullptr, nv, fa);
  if (st) return st;
  if (!fa.per_vertex) return ext_fail(ctx, FTK2B_INVALID_ARG, "extruded meshes take per-vertex arrays");
  if (fa.has_scalar && !fa.scalar_per_vertex)
    return ext_fail(ctx, FTK2B_INVALID_ARG, "the scalar of an extruded mesh must be a per-vertex array");

  unsigned long long nl = 0;
  st = prepare_base(ctx, mesh, fbits, &nl);
  if (st) return st;
  ExtCache& C = ctx->ext;
  ExtMeshDev X;
  X.cd = M;
  X.ns = ns;
  X.L = L;
  X.ncell = (unsigned)C.ncell;
  X.nface = C.nface;
  X.fbits = C.fbits;
  X.cells = (const unsigned*)C.cells.p;
  X.fkeys = (const unsigned long long*)C.fkeys.p;
  X.cof_start = (const unsigned*)C.cof_start.p;
  X.cof = (const unsigned*)C.cof.p;
  X.t0 = 0;
  X.tflip = 0;
  X.skip_first_spatial = 0;
  const int vb = bits_of(nv - 1);
  const uint64_t nsimp = C.ncell * (uint64_t)(L + 1) + (uint64_t)C.nface * L * M + C.ncell * (uint64_t)L * M;

  ExtractConfig cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.Q = prm->sos_q;
  cfg.refined = prm->precision == FTK2B_PRECISION_REFINED;
  if (fiber_thr) {  // FiberPredicate: every simplex tested, values minus thresholds
    cfg.fiber = 1;
    cfg.fthr[0] = fiber_thr[0];
    cfg.fthr[1] = fiber_thr[1];
    cfg.refined = 0;
  }
  const int f64 = field->dtype == FTK2B_F64;
  EXT_TRY(C.words.ensure(sizeof(unsigned) * nv));

  unsigned cap = ctx->cap_hint ? ctx->cap_hint : 65536u;
  for (int attempt = 0; attempt < 4; ++attempt) {
    const unsigned edge_cap = cap * 2;
    st = ensure_feature_buffers(ctx, cap, edge_cap, M);
    if (st) return st;
    const size_t wk = std::max<size_t>(std::max<size_t>(cap, edge_cap), C.ncell * (size_t)(M + 1));
    EXT_TRY(C.hi.ensure(sizeof(unsigned long long) * cap));
    EXT_TRY(C.lo.ensure(sizeof(unsigned long long) * cap));
    EXT_TRY(C.phase.ensure(sizeof(unsigned) * cap));
    EXT_TRY(C.hi_s.ensure(sizeof(unsigned long long) * cap));
    EXT_TRY(C.lo_s.ensure(sizeof(unsigned long long) * cap));
    EXT_TRY(C.phase_s.ensure(sizeof(unsigned) * cap));
    EXT_TRY(C.sort_k.ensure(sizeof(unsigned long long) * wk));
    EXT_TRY(C.sort_k2.ensure(sizeof(unsigned long long) * wk));
    EXT_TRY(C.sort_v.ensure(sizeof(unsigned) * wk));
    EXT_TRY(C.sort_v2.ensure(sizeof(unsigned) * wk));
    EXT_TRY(C.ekeys.ensure(sizeof(unsigned long long) * wk));
    EXT_TRY(ctx->hist.ensure(sizeof(unsigned) * 256 * (size_t)ctx->sort_grid((unsigned)wk)));
    ExtSink sink;
    sink.hi = (unsigned long long*)C.hi.p;
    sink.lo = (unsigned long long*)C.lo.p;
    sink.phase = (unsigned*)C.phase.p;
    sink.lam = (double*)ctx->lam.p;
    sink.bary4 = (float*)ctx->bary4.p;
    sink.scalar = (float*)ctx->scalar.p;
    sink.count = (unsigned*)ctx->counters.p + kCountFeatures;
    sink.cap = cap;
    cudaStream_t s = ctx->stream;
    EXT_TRY(cudaEventRecord(ctx->ev0, s));
    EXT_TRY(cudaMemsetAsync(ctx->counters.p, 0, sizeof(unsigned) * kNumCounters, s));
    cudaError_t e;
    if (M == 3)
      e = f64 ? enqueue_extract<double, 3>(ctx, X, fa, cfg, sink, vb, nv, &nl)
              : enqueue_extract<float, 3>(ctx, X, fa, cfg, sink, vb, nv, &nl);
    else
      e = f64 ? enqueue_extract<double, 2>(ctx, X, fa, cfg, sink, vb, nv, &nl)
              : enqueue_extract<float, 2>(ctx, X, fa, cfg, sink, vb, nv, &nl);
    EXT_TRY(e);
    EXT_TRY(cudaEventRecord(ctx->ev_x, s));
    e = (M == 3) ? enqueue_post<3>(ctx, X, sink, cap, edge_cap, vb, prm->want_edges, &nl)
                 : enqueue_post<2>(ctx, X, sink, cap, edge_cap, vb, prm->want_edges, &nl);
    EXT_TRY(e);
    EXT_TRY(cudaMemcpyAsync(ctx->h_counters, ctx->counters.p, sizeof(unsigned) * kNumCounters,
                            cudaMemcpyDeviceToHost, s));
    EXT_TRY(cudaEventRecord(ctx->ev1, s));
    EXT_TRY(ctx->sync());
    ctx->launches += nl;
    nl = 0;
    unsigned h[kNumCounters];
    memcpy(h, ctx->h_counters, sizeof(h));
    float ms = 0.f, xms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) != cudaSuccess) ms = 0.f;
    if (cudaEventElapsedTime(&xms, ctx->ev0, ctx->ev_x) != cudaSuccess) xms = 0.f;
    cudaGetLastError();
    ctx->last_extract_ms = xms;
    if (h[kCountErr] & kErrCofaces)
      return ext_fail(ctx, FTK2B_UNSUPPORTED, "a base face has more than 8 coface cells");
    if (h[kCountErr] & 1u) return ext_fail(ctx, FTK2B_TIMEOUT, "union-find retry bound reached");
    if (h[kCountFeatures] > cap || h[kCountEdges] > edge_cap) {
      uint64_t want = (uint64_t)h[kCountFeatures] + h[kCountFeatures] / 4 + 1024;
      const uint64_t want_e = ((uint64_t)h[kCountEdges] + 1) / 2 + 1024;
      if (want_e > want) want = want_e;
      if (want > 0x7FFFFFF0ull) return ext_fail(ctx, FTK2B_OVERFLOW_RETRY, "feature count exceeds 2^31");
      cap = (unsigned)want;
      ctx->cap_hint = cap;
      continue;
    }
    ctx->last.kind = FTK2B_MESH_EXTRUDED;
    ctx->last.m = M;
    ctx->last.f64 = field->dtype == FTK2B_F64;
    ctx->last.n = h[kCountFeatures];
    ctx->last.ne = prm->want_edges ? h[kCountEdges] : 0;
    ctx->last.n_roots = h[kCountRoots];
    ctx->last.n_simplices = nsimp;
    ctx->last.device_ms = ms;
    ctx->last.classify = 0;
    ctx->last.want_edges = prm->want_edges;
    return FTK2B_OK;
  }
  return ext_fail(ctx, FTK2B_OVERFLOW_RETRY, "feature buffer overflow persisted after retries");
}
