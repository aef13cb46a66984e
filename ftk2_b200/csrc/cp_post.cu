// Post-extraction stages of the critical-point path, all on the device and
// driven by device-resident counts (so the whole pipeline can be enqueued, and
// captured in a CUDA graph, without a host round trip):
//
//   1. canonical order: LSD radix sort of the feature keys.  Key order equals
//      the reference's Simplex::operator< order (mesh.hpp:36-42), so sorted
//      position = canonical id (engine.hpp:838-850).
//   2. star edges: for every feature, the top cells it is a face of (the two
//      Kuhn cofaces of a codimension-1 simplex), their other faces looked up by
//      binary search; the smallest active face of a cell is the star centre and
//      links to every other active face (engine.hpp:1342-1387; for regular
//      meshes encode_simplex_id order equals key order, mesh.hpp:736-749).
//   3. trajectories: lock-free union-find that always hooks the larger root
//      under the smaller one, so every component's root is its smallest
//      canonical id = the reference's track_id (engine.hpp:46-74, 965-983).
#include "cp_batch.h"
#include "cp_post.h"
#include "cp_kuhn.cuh"
#include "cp_pdl.cuh"
#include "cp_uf.cuh"

namespace ftk2b {

__constant__ ChainTable c_post_chains[2];
__constant__ signed char c_rank3[64];     // (m1 | m2 << 3) -> chain rank, d = 3
__constant__ signed char c_rank4[4096];   // (m1 | m2 << 4 | m3 << 8) -> chain rank, d = 4
// the same tables for lane-dependent indices (the constant bank would
// serialise them): chain masks of vertices 0..m, 4 bits each, and the rank
// tables [0] = c_rank3 (64 entries, then -1), [1] = c_rank4
__device__ unsigned g_star_mk[2][kMaxChains];
__device__ __align__(16) signed char g_rank[2][4096];

// ---------------------------------------------------------------------------
// radix sort (keys u64, payload u32), stable, device-resident count

constexpr int kRsThreads = 256;

__global__ void rs_hist_kernel(const unsigned long long* __restrict__ keys, const unsigned* n_ptr,
                               unsigned cap, int shift, unsigned* __restrict__ hist) {
  pdl_enter();
  __shared__ unsigned h[256];
  const unsigned n = min(*n_ptr, cap);
  const unsigned G = gridDim.x, b = blockIdx.x;
  const unsigned chunk = (n + G - 1) / G;
  const unsigned start = min(b * chunk, n), end = min(start + chunk, n);
  h[threadIdx.x] = 0;
  __syncthreads();
  for (unsigned i = start + threadIdx.x; i < end; i += kRsThreads)
    atomicAdd(&h[(keys[i] >> shift) & 255], 1u);
  __syncthreads();
  hist[threadIdx.x * G + b] = h[threadIdx.x];
}

// Exclusive scan over a block of 1024 threads, one value each; *total = sum.
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* wsum /* 33 */, unsigned* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const unsigned w = wsum[lane];
    unsigned wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= o) wi += y;
    }
    wsum[lane] = wi - w;
    if (lane == 31) wsum[32] = wi;
  }
  __syncthreads();
  *total = wsum[32];
  return wsum[warp] + incl - v;
}

// exclusive scan of `total` counters in place (clamped to *n_ptr), one block
// of 1024 threads: tiles of 4096 counters, each thread 4 consecutive ones
// (coalesced 16-byte loads), the next tile's loads issued before the current
// tile is scanned, a running carry between tiles
__global__ void scan_inplace_kernel(unsigned* __restrict__ a, unsigned total, unsigned* total_out,
                                    const unsigned* n_ptr, const unsigned* skip_small) {
  pdl_enter();
  constexpr int kPer = 4;
  constexpr unsigned kTile = 1024u * kPer;
  __shared__ unsigned wsum[33];
  const unsigned t = threadIdx.x;
  (void)skip_small;
  if (n_ptr) total = min(total, *n_ptr);
  const bool vec = (reinterpret_cast<uintptr_t>(a) & 15) == 0;  // 16-byte loads need an aligned array
  auto load = [&](unsigned base, unsigned (&v)[kPer]) {
    const unsigned i0 = base + t * kPer;
    if (vec && base + kTile <= total) {
      const uint4 q = *reinterpret_cast<const uint4*>(a + i0);
      v[0] = q.x;
      v[1] = q.y;
      v[2] = q.z;
      v[3] = q.w;
    } else {
#pragma unroll
      for (int j = 0; j < kPer; ++j) v[j] = i0 + j < total ? a[i0 + j] : 0u;
    }
  };
  unsigned nxt[kPer] = {0u, 0u, 0u, 0u};
  if (total) load(0, nxt);
  unsigned carry = 0;
  for (unsigned base = 0; base < total; base += kTile) {
    unsigned v[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) v[j] = nxt[j];
    if (base + kTile < total) load(base + kTile, nxt);
    const unsigned sum = v[0] + v[1] + v[2] + v[3];
    unsigned tile_total;
    unsigned run = carry + block_exclusive_scan(sum, wsum, &tile_total);
    const unsigned i0 = base + t * kPer;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      if (i0 + j < total) a[i0 + j] = run;
      run += v[j];
    }
    carry += tile_total;
    __syncthreads();  // wsum is rewritten by the next tile's scan
  }
  if (total_out && t == 0) *total_out = carry;
}

__global__ void rs_scatter_kernel(const unsigned long long* __restrict__ kin,
                                  const unsigned* __restrict__ vin,
                                  unsigned long long* __restrict__ kout, unsigned* __restrict__ vout,
                                  const unsigned* n_ptr, unsigned cap, int shift,
                                  const unsigned* __restrict__ hist) {
  pdl_enter();
  __shared__ unsigned base[256];
  __shared__ unsigned wcnt[kRsThreads / 32][256];
  const unsigned n = min(*n_ptr, cap);
  const unsigned G = gridDim.x, b = blockIdx.x;
  const unsigned chunk = (n + G - 1) / G;
  const unsigned start = min(b * chunk, n), end = min(start + chunk, n);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  base[tid] = hist[tid * G + b];
  for (unsigned t0 = start; t0 < end; t0 += kRsThreads) {
    const unsigned i = t0 + tid;
    const bool valid = i < end;
    const unsigned long long key = valid ? kin[i] : 0ull;
    const unsigned val = valid ? vin[i] : 0u;
    const unsigned dig = valid ? (unsigned)((key >> shift) & 255) : 256u;
#pragma unroll
    for (int w = 0; w < kRsThreads / 32; ++w) wcnt[w][tid] = 0;
    __syncthreads();
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, dig);
    const unsigned rank = __popc(peers & ((1u << lane) - 1));
    if (valid && lane == __ffs(peers) - 1) wcnt[warp][dig] = __popc(peers);
    __syncthreads();
    unsigned run = 0;
#pragma unroll
    for (int w = 0; w < kRsThreads / 32; ++w) {
      const unsigned c = wcnt[w][tid];
      wcnt[w][tid] = run;
      run += c;
    }
    __syncthreads();
    if (valid) {
      const unsigned pos = base[dig] + wcnt[warp][dig] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
    base[tid] += run;
    __syncthreads();
  }
}

__global__ void iota_kernel(unsigned* v, const unsigned* n_ptr, unsigned cap) {
  pdl_enter();
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// Sorts (keys, vals) of device count *n_ptr (clamped to cap) over the low
// `bits` bits.  Result lands in whichever buffer pair the pass parity selects;
// returns true when it is the alternate pair.
bool radix_sort(unsigned long long* k0, unsigned* v0, unsigned long long* k1, unsigned* v1,
                const unsigned* n_ptr, unsigned cap, int bits, unsigned* hist, int grid,
                cudaStream_t st, unsigned long long* launches) {
  bool alt = false;
  for (int shift = 0; shift < bits; shift += 8) {
    const unsigned long long* ki = alt ? k1 : k0;
    const unsigned* vi = alt ? v1 : v0;
    unsigned long long* ko = alt ? k0 : k1;
    unsigned* vo = alt ? v0 : v1;
    launch_pdl(rs_hist_kernel, grid, kRsThreads, 0, st, ki, n_ptr, cap, shift, hist);
    launch_pdl(scan_inplace_kernel, 1, 1024, 0, st, hist, 256u * grid, (unsigned*)nullptr, (const unsigned*)nullptr,
               n_ptr);
    launch_pdl(rs_scatter_kernel, grid, kRsThreads, 0, st, ki, vi, ko, vo, n_ptr, cap, shift, (const unsigned*)hist);
    if (launches) *launches += 3;
    alt = !alt;
  }
  return alt;
}

// ---------------------------------------------------------------------------
// gather features into canonical order

__global__ void gather_kernel(const unsigned* n_ptr, unsigned cap, const unsigned* __restrict__ perm,
                              const double* __restrict__ lam_in, const float* __restrict__ sc_in,
                              const float* __restrict__ bary_in, double* __restrict__ lam_out,
                              float* __restrict__ sc_out, float* __restrict__ bary_out) {
  pdl_enter();
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned p = perm[i];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      lam_out[4 * (size_t)i + k] = lam_in[4 * (size_t)p + k];
      bary_out[4 * (size_t)i + k] = bary_in[4 * (size_t)p + k];
    }
    sc_out[i] = sc_in[p];
  }
}

// ---------------------------------------------------------------------------
// regular-mesh geometry helpers

__device__ __forceinline__ void decode_key(const RegularMesh& mesh, int nch, unsigned long long key,
                                           Decoded& dc) {
  const ChainTable& CT = c_post_chains[mesh.d - 3];
  const int m = mesh.d - 1;
  unsigned long long vid = key / (unsigned long long)nch;
  const int ch = (int)(key % (unsigned long long)nch);
  for (int k = 0; k < mesh.d; ++k) {
    dc.g[k] = (long long)(vid % (unsigned long long)mesh.gd[k]);
    vid /= (unsigned long long)mesh.gd[k];
  }
  dc.mk[0] = 0;
  for (int i = 0; i < m; ++i) dc.mk[i + 1] = CT.mask[ch][i];
}

__device__ __forceinline__ int chain_rank(int d, const int* rel /* m masks */) {
  if (d == 3) return c_rank3[rel[0] | (rel[1] << 3)];
  return c_rank4[rel[0] | (rel[1] << 4) | (rel[2] << 8)];
}

__device__ __forceinline__ long long find_key(const unsigned long long* keys, unsigned n,
                                              unsigned long long k) {
  unsigned lo = 0, hi = n;
  while (lo < hi) {
    const unsigned mid = (lo + hi) >> 1;
    const unsigned long long v = keys[mid];
    if (v == k) return mid;
    if (v < k) lo = mid + 1;
    else hi = mid;
  }
  return -1;
}

// find_key over n sorted keys in global memory with a sample of every
// 2^slog-th key in shared memory: the sample's binary search picks the run of
// 2^slog keys that can hold k, then a binary search inside that run.
__device__ __forceinline__ long long find_key_sampled(const unsigned long long* keys, unsigned n,
                                                      const unsigned long long* sample, unsigned ns, int slog,
                                                      unsigned long long k) {
  unsigned lo = 0, hi = ns;  // the last run whose first key is <= k
  while (hi - lo > 1) {
    const unsigned mid = (lo + hi) >> 1;
    if (sample[mid] <= k) lo = mid;
    else hi = mid;
  }
  const unsigned r0 = lo << slog, r1 = min(r0 + (1u << slog), n);
  const long long j = find_key(keys + r0, r1 - r0, k);
  return j < 0 ? -1 : (long long)r0 + j;
}

// Indices of the active faces of a top cell, ascending.
__device__ int active_faces(const RegularMesh& mesh, int nch, const unsigned long long* keys,
                            unsigned n, const long long cc[4], const int cm[5], long long out[5]) {
  const int d = mesh.d, m = d - 1;
  int na = 0;
  for (int r = 0; r <= d; ++r) {
    // face without vertex r: corner = cell vertex (r == 0 ? 1 : 0)
    const int basem = (r == 0) ? cm[1] : 0;
    int rel[4];
    int w = 0;
    for (int i = 0; i <= d; ++i) {
      if (i == r || (r == 0 && i == 1) || (r != 0 && i == 0)) continue;
      rel[w++] = cm[i] & ~basem;
    }
    unsigned long long vid = 0;
    for (int k = 0; k < d; ++k)
      vid += (unsigned long long)(cc[k] + ((basem >> k) & 1)) * mesh.gstride[k];
    const int rk = chain_rank(d, rel);
    const long long idx = find_key(keys, n, vid * (unsigned long long)nch + (unsigned long long)rk);
    if (idx >= 0) out[na++] = idx;
    (void)m;
  }
  // insertion sort (at most 5)
  for (int i = 1; i < na; ++i)
    for (int j = i; j > 0 && out[j - 1] > out[j]; --j) {
      long long t = out[j];
      out[j] = out[j - 1];
      out[j - 1] = t;
    }
  return na;
}

constexpr int kEdgeSlots = 8;  // a codimension-1 simplex has 2 cofaces with <= 4 other faces each

// Index of the face of top cell (cc, cm) without vertex r, or -1.
__device__ __forceinline__ long long face_index(const RegularMesh& mesh, int nch,
                                                const unsigned long long* keys, unsigned n,
                                                const long long cc[4], const int cm[5], int r,
                                                unsigned long long kbase = 0) {
  const int d = mesh.d;
  const int basem = (r == 0) ? cm[1] : 0;
  int rel[4];
  int w = 0;
  for (int i = 0; i <= d; ++i) {
    if (i == r || (r == 0 && i == 1) || (r != 0 && i == 0)) continue;
    rel[w++] = cm[i] & ~basem;
  }
  unsigned long long vid = 0;
  for (int k = 0; k < d; ++k) vid += (unsigned long long)(cc[k] + ((basem >> k) & 1)) * mesh.gstride[k];
  return find_key(keys, n, kbase + vid * (unsigned long long)nch + (unsigned long long)chain_rank(d, rel));
}

// One warp per feature: lanes look up the faces of both cofaces in parallel;
// when the feature is the smallest active face of a cell it writes the star
// edges to its other active faces into padded slots (ascending), and its
// edge count.  Feature i has key kbase + local_key; keys of its mesh's faces
// are searched in the same key space.
__device__ __forceinline__ void edges_of_feature(const RegularMesh& mesh, int nch,
                                                 const unsigned long long* __restrict__ keys, unsigned n, unsigned i,
                                                 unsigned long long local_key, unsigned long long kbase, int lane,
                                                 unsigned* __restrict__ cnt, unsigned* __restrict__ slots) {
  const int d = mesh.d;
  Decoded dc;
  decode_key(mesh, nch, local_key, dc);
  long long cc[2][4];
  int cm[2][5];
  const int nc = top_cells(mesh, dc, cc, cm);
  long long idx = -1;
  const int q = lane / (d + 1), r = lane % (d + 1);
  if (lane < nc * (d + 1)) idx = face_index(mesh, nch, keys, n, cc[q], cm[q], r, kbase);
  const unsigned act = __ballot_sync(0xFFFFFFFFu, idx >= 0);
  unsigned others[kEdgeSlots];
  int no = 0;
  for (int qq = 0; qq < nc; ++qq) {
    const unsigned cellmask = ((1u << (d + 1)) - 1u) << (qq * (d + 1));
    const unsigned a = act & cellmask;
    const unsigned v = ((a >> lane) & 1u) ? (unsigned)idx : 0xFFFFFFFFu;
    const unsigned mn = __reduce_min_sync(0xFFFFFFFFu, v);
    if (__popc(a) < 2 || mn != i) continue;
    for (unsigned bits = a; bits; bits &= bits - 1) {
      const unsigned val = __shfl_sync(0xFFFFFFFFu, (unsigned)idx, __ffs(bits) - 1);
      if (val != i && no < kEdgeSlots) others[no++] = val;
    }
  }
  if (lane == 0) {
    for (int a2 = 1; a2 < no; ++a2)
      for (int b2 = a2; b2 > 0 && others[b2 - 1] > others[b2]; --b2) {
        const unsigned t = others[b2];
        others[b2] = others[b2 - 1];
        others[b2 - 1] = t;
      }
    cnt[i] = no;
    for (int k = 0; k < no; ++k) slots[(size_t)i * kEdgeSlots + k] = others[k];
  }
}

__global__ void edges_regular_warp_kernel(RegularMesh mesh, int nch,
                                          const unsigned long long* __restrict__ keys,
                                          const unsigned* n_ptr, unsigned cap,
                                          unsigned* __restrict__ cnt, unsigned* __restrict__ slots) {
  pdl_enter();
  const unsigned n = min(*n_ptr, cap);
  const int lane = threadIdx.x & 31;
  const unsigned gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nw = (gridDim.x * blockDim.x) >> 5;
  for (unsigned i = gw; i < n; i += nw) edges_of_feature(mesh, nch, keys, n, i, keys[i], 0ull, lane, cnt, slots);
}

// Field of a key of a batch: the last f with kb[f] <= key (kb ascending, nf entries).
__device__ __forceinline__ unsigned batch_field_of(const unsigned long long* __restrict__ kb, int nf,
                                                   unsigned long long key) {
  unsigned lo = 0, hi = (unsigned)nf;
  while (hi - lo > 1) {
    const unsigned mid = (lo + hi) >> 1;
    if (kb[mid] <= key) lo = mid;
    else hi = mid;
  }
  return lo;
}

// After the exclusive scan of the counts (in place), copy every feature's
// edges to their final positions: (centre, other) pairs, sorted and unique.
__global__ void edges_compact_kernel(const unsigned* n_ptr, unsigned cap, const unsigned* __restrict__ off,
                                     const unsigned* n_edges, const unsigned* __restrict__ slots,
                                     unsigned* __restrict__ edges, unsigned edge_cap) {
  pdl_enter();
  const unsigned n = min(*n_ptr, cap);
  const unsigned ne = *n_edges;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned o = off[i];
    const unsigned c = (i + 1 < n ? off[i + 1] : ne) - o;
    for (unsigned k = 0; k < c; ++k)
      if (o + k < edge_cap) {
        edges[2 * (size_t)(o + k)] = i;
        edges[2 * (size_t)(o + k) + 1] = slots[(size_t)i * kEdgeSlots + k];
      }
  }
}

// pass 0: count edges per feature (as star centre); pass 1: write them
template <int PASS>
__global__ void edges_regular_kernel(RegularMesh mesh, int nch, const unsigned long long* __restrict__ keys,
                                     const unsigned* n_ptr, unsigned cap, unsigned* __restrict__ cnt,
                                     const unsigned* __restrict__ off, unsigned* __restrict__ edges,
                                     unsigned edge_cap) {
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Decoded dc;
    decode_key(mesh, nch, keys[i], dc);
    long long cc[2][4];
    int cm[2][5];
    const int nc = top_cells(mesh, dc, cc, cm);
    long long others[8];
    int no = 0;
    for (int q = 0; q < nc; ++q) {
      long long act[5];
      const int na = active_faces(mesh, nch, keys, n, cc[q], cm[q], act);
      if (na >= 2 && act[0] == (long long)i)
        for (int t = 1; t < na; ++t) others[no++] = act[t];
    }
    if (PASS == 0) {
      cnt[i] = no;
    } else {
      for (int a = 1; a < no; ++a)
        for (int b = a; b > 0 && others[b - 1] > others[b]; --b) {
          long long t = others[b];
          others[b] = others[b - 1];
          others[b - 1] = t;
        }
      const unsigned o = off[i];
      for (int t = 0; t < no; ++t)
        if (o + t < edge_cap) {
          edges[2 * (size_t)(o + t)] = i;
          edges[2 * (size_t)(o + t) + 1] = (unsigned)others[t];
        }
    }
  }
}

// ---------------------------------------------------------------------------
// union-find

__global__ void uf_init_kernel(unsigned* parent, const unsigned* n_ptr, unsigned cap) {
  pdl_enter();
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    parent[i] = i;
}

__global__ void uf_hook_kernel(unsigned* parent, const unsigned* __restrict__ edges,
                               const unsigned* ne_ptr, unsigned edge_cap, unsigned* err) {
  pdl_enter();
  const unsigned ne = min(*ne_ptr, edge_cap);
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x)
    uf_unite(parent, edges[2 * (size_t)e], edges[2 * (size_t)e + 1], err);
}

__global__ void uf_label_kernel(unsigned* parent, const unsigned* n_ptr, unsigned cap,
                                unsigned long long* __restrict__ track, unsigned* n_roots) {
  pdl_enter();
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned x = uf_root(parent, i);
    track[i] = x;
    if (x == i) atomicAdd(n_roots, 1u);
  }
}

// ---------------------------------------------------------------------------
// output expansion: vertex ids and float barycentrics

// Vertex ids (and float barycentrics) of feature i with local key key, into
// rows of `stride` entries.
__device__ __forceinline__ void expand_feature(const RegularMesh& mesh, int nch, unsigned long long key, unsigned i,
                                               int stride, const float* __restrict__ bary4,
                                               unsigned long long* __restrict__ simplices, float* __restrict__ bary) {
  const int m = mesh.d - 1;
  Decoded dc;
  decode_key(mesh, nch, key, dc);
  for (int v = 0; v <= m; ++v) {
    unsigned long long vid = 0;
    for (int k = 0; k < mesh.d; ++k)
      vid += (unsigned long long)(dc.g[k] + ((dc.mk[v] >> k) & 1)) * mesh.gstride[k];
    simplices[(size_t)i * stride + v] = vid;
    if (bary) bary[(size_t)i * stride + v] = bary4[4 * (size_t)i + v];
  }
}

__global__ void expand_regular_kernel(RegularMesh mesh, int nch, const unsigned long long* __restrict__ keys,
                                      const unsigned* n_ptr, unsigned cap,
                                      const float* __restrict__ bary4,
                                      unsigned long long* __restrict__ simplices,
                                      float* __restrict__ bary) {
  pdl_enter();
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    expand_feature(mesh, nch, keys[i], i, mesh.d, bary4, simplices, bary);
}

// Batches: rows of 4 entries whatever the field's dimension.
__global__ void expand_batch_kernel(const BatchMesh* __restrict__ fm, const unsigned long long* __restrict__ kb, int nf,
                                    const unsigned long long* __restrict__ keys, const unsigned* n_ptr, unsigned cap,
                                    const float* __restrict__ bary4, unsigned long long* __restrict__ simplices,
                                    float* __restrict__ bary) {
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned long long key = keys[i];
    const unsigned f = batch_field_of(kb, nf, key);
    expand_feature(fm[f].mesh, fm[f].nch, key - kb[f], i, 4, bary4, simplices, bary);
  }
}

// fbase[f] = index of the first feature of field f in canonical order
// (f = 0 .. nf; kb[nf] is the end of the key space)
__global__ void batch_bounds_kernel(const unsigned long long* __restrict__ kb, int nf,
                                    const unsigned long long* __restrict__ keys, const unsigned* n_ptr, unsigned cap,
                                    unsigned* __restrict__ fbase) {
  const unsigned n = min(*n_ptr, cap);
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f <= nf; f += gridDim.x * blockDim.x) {
    const unsigned long long k = kb[f];
    unsigned lo = 0, hi = n;
    while (lo < hi) {
      const unsigned mid = (lo + hi) >> 1;
      if (keys[mid] < k) lo = mid + 1;
      else hi = mid;
    }
    fbase[f] = lo;
  }
}

// ---------------------------------------------------------------------------

void upload_post_tables() {
  ChainTable h[2];
  // same construction as the extraction tables (canonical chain order)
  auto build = [](ChainTable& t, int d, int m) {
    t.n = 0;
    const int full = (1 << d) - 1;
    int cur[5] = {0, 0, 0, 0, 0}, next[5] = {0, 0, 0, 0, 0};
    int depth = 1;
    while (depth > 0) {
      const int prev = cur[depth - 1];
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
  };
  build(h[0], 3, 2);
  build(h[1], 4, 3);
  cudaMemcpyToSymbol(c_post_chains, h, sizeof(h));
  signed char r3[64], r4[4096];
  for (int i = 0; i < 64; ++i) r3[i] = -1;
  for (int i = 0; i < 4096; ++i) r4[i] = -1;
  for (int c = 0; c < h[0].n; ++c) r3[h[0].mask[c][0] | (h[0].mask[c][1] << 3)] = (signed char)c;
  for (int c = 0; c < h[1].n; ++c)
    r4[h[1].mask[c][0] | (h[1].mask[c][1] << 4) | (h[1].mask[c][2] << 8)] = (signed char)c;
  cudaMemcpyToSymbol(c_rank3, r3, sizeof(r3));
  cudaMemcpyToSymbol(c_rank4, r4, sizeof(r4));
  signed char gr[2][4096];
  for (int i = 0; i < 4096; ++i) {
    gr[0][i] = i < 64 ? r3[i] : (signed char)-1;
    gr[1][i] = r4[i];
  }
  cudaMemcpyToSymbol(g_rank, gr, sizeof(gr));
  unsigned mk[2][kMaxChains] = {};
  for (int t = 0; t < 2; ++t)
    for (int c = 0; c < h[t].n; ++c)
      for (int k = 0; k < t + 2; ++k) mk[t][c] |= (unsigned)h[t].mask[c][k] << (4 * (k + 1));
  cudaMemcpyToSymbol(g_star_mk, mk, sizeof(mk));
}

static int grid_for(unsigned cap, int threads, int max_blocks) {
  long long b = ((long long)cap + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

// ---------------------------------------------------------------------------
// Post-extraction for small feature counts (capacity <= kSmallPostCap, keys
// below 2^50): the outputs of the general chain above in two launches.
//   1. sort, one block: a counting sort of the keys (each packed with its
//      feature index in the low kIdxBits bits) by their top bits in shared
//      memory, then each key's canonical position = its bucket's start + the
//      keys of its bucket below it (the keys of one extraction are
//      distinct); the packed keys land in key_alt in canonical order.
//   2. star edges, one block of 1024 threads per SM: every block copies the
//      sorted keys into shared memory, its warps find the star edges of the
//      sorted features (one warp per feature) in the sorted keys and join
//      each feature with its linked faces in a lock-free union-find (parents
//      initialised by the sort); then each block writes the outputs of its
//      contiguous share of positions, and the last block to finish runs the
//      final step: exclusive scan of the edge counts, edge compaction, and
//      every feature's root (the union-find's parents copied to shared
//      memory): track ids and root count.

constexpr int kSortThreads = 1024;
constexpr int kBucketBits = 13;
constexpr int kBuckets = 1 << kBucketBits;
constexpr int kIdxBits = 14;  // feature index bits packed under a key (kSmallPostCap = 2^14)
static_assert((1u << kIdxBits) >= kSmallPostCap, "feature indices of the short chain fit kIdxBits");

// Shared tables of the sort + edges kernel: the chain masks of the mesh's
// dimension, 4 bits each with mk[0] = 0 in the lowest nibble, and the chain
// rank by relative masks (c_rank3 / c_rank4).  Lane-dependent indices into
// the constant bank would be serialised.
struct __align__(16) StarTables {
  unsigned mk[kMaxChains];
  signed char rank[4096];
};

__device__ __forceinline__ void fill_star_tables(StarTables& T, int d) {
  for (int c = threadIdx.x; c < kMaxChains; c += blockDim.x) T.mk[c] = g_star_mk[d - 3][c];
  const unsigned* src = reinterpret_cast<const unsigned*>(g_rank[d - 3]);
  unsigned* dst = reinterpret_cast<unsigned*>(T.rank);
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) dst[i] = src[i];
}

// a / b and a % b, in 32 bits when both fit
__device__ __forceinline__ unsigned long long divmod_u64(unsigned long long a, unsigned long long b,
                                                         unsigned long long& rem) {
  if (((a | b) >> 32) == 0) {
    const unsigned q = (unsigned)a / (unsigned)b;
    rem = (unsigned)a - q * (unsigned)b;
    return q;
  }
  const unsigned long long q = a / b;
  rem = a - q * b;
  return q;
}

// Star edges of sorted feature i (one warp; key = kbase + local key): the two
// Kuhn cofaces of its simplex inside the local box (the order of top_cells),
// lane q * (d + 1) + r looks face r of coface q up in the sorted keys; when
// feature i is the smallest active face of a coface it links to that coface's
// other active faces.  Writes cnt[i] and the slots ascending, and (parent not
// null) joins i with every linked face in the union-find.  Register-only form
// of edges_of_feature.
__device__ __forceinline__ void star_edges_warp(const RegularMesh& mesh, int nch, const unsigned long long* keys,
                                                unsigned n, unsigned i, unsigned long long local_key,
                                                unsigned long long kbase, const StarTables& T, int lane,
                                                unsigned* __restrict__ cnt, unsigned* __restrict__ slots,
                                                unsigned* parent, unsigned* err,
                                                const unsigned long long* sample = nullptr, unsigned ns = 0,
                                                int slog = 0) {
  const int d = mesh.d, m = d - 1, full = (1 << d) - 1;
  unsigned long long rem;
  unsigned long long vid = divmod_u64(local_key, (unsigned long long)nch, rem);
  const int ch = (int)rem;
  long long g[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    g[k] = 0;
    if (k < d) {
      vid = divmod_u64(vid, (unsigned long long)mesh.gd[k], rem);
      g[k] = (long long)rem;
    }
  }
  const unsigned mkp = FTK2B_CHECK(ch >= 0 && ch < kMaxChains, err) ? T.mk[ch] : 0u;  // masks of vertices 0..m, 4 bits each
  const int mkm = (int)((mkp >> (4 * m)) & 15u);
  const int missing = full & ~mkm;
  const int q = lane > d ? 1 : 0, r = lane - q * (d + 1);
  long long c[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) c[k] = g[k];
  unsigned cmp = 0;  // masks of the coface's d + 1 vertices, 4 bits each
  int nc;
  if (missing) {
    // axis a never steps: prepend (corner - e_a) and / or append (full mask)
    const int a = __ffs(missing) - 1;
    long long ga = 0, la = 0;  // local coordinate and extent along a
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k == a) {
        ga = g[k] - mesh.off[k];
        la = mesh.ld[k];
      }
    const bool lo = ga >= 1, hi = ga + 1 < la;
    nc = (int)lo + (int)hi;
    if (lo && q == 0) {
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (k == a) c[k] -= 1;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j <= m) cmp |= ((((mkp >> (4 * j)) & 15u) | (1u << a)) << (4 * (j + 1)));
    } else {
      cmp = mkp | ((unsigned)full << (4 * (m + 1)));
    }
  } else {
    // the one step of two axes, split in either order
    int js = -1, ins_lo = 0, ins_hi = 0;
#pragma unroll
    for (int j = 1; j < 4; ++j)
      if (j <= m && js < 0) {
        const int step = (int)(((mkp >> (4 * j)) & 15u) & ~((mkp >> (4 * (j - 1))) & 15u));
        if (__popc(step) == 2) {
          js = j;
          ins_lo = step & -step;
          ins_hi = step & ~ins_lo;
        }
      }
    nc = js < 0 ? 0 : 2;
    if (js > 0) {
      const unsigned ins = (unsigned)(q ? ins_hi : ins_lo);
      const unsigned low = (1u << (4 * js)) - 1u;
      cmp = (mkp & low) | ((((mkp >> (4 * (js - 1))) & 15u) | ins) << (4 * js)) | ((mkp & ~low) << 4);
    }
  }
  long long idx = -1;
  if (lane < nc * (d + 1)) {
    // face without vertex r: based at vertex 1 when r == 0, else at vertex 0
    const unsigned base = r == 0 ? ((cmp >> 4) & 15u) : 0u;
    const int bits = d == 3 ? 3 : 4;
    unsigned rel = 0;
    int w = 0;
#pragma unroll
    for (int v = 1; v <= 4; ++v)
      if (v <= d && v != r && !(r == 0 && v == 1)) {
        rel |= (((cmp >> (4 * v)) & 15u) & ~base) << (bits * w);
        ++w;
      }
    unsigned long long fvid = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k < d) fvid += (unsigned long long)(c[k] + ((base >> k) & 1u)) * mesh.gstride[k];
    const int rk = FTK2B_CHECK(rel < 4096u, err) ? T.rank[rel] : -1;
    const unsigned long long fk = kbase + fvid * (unsigned long long)nch + (unsigned long long)rk;
    idx = sample ? find_key_sampled(keys, n, sample, ns, slog, fk) : find_key(keys, n, fk);
  }
  const unsigned act = __ballot_sync(0xFFFFFFFFu, idx >= 0);
  bool qual[2] = {false, false};
#pragma unroll
  for (int qq = 0; qq < 2; ++qq)
    if (qq < nc) {
      const unsigned a = act & (((1u << (d + 1)) - 1u) << (qq * (d + 1)));
      const unsigned v = ((a >> lane) & 1u) ? (unsigned)idx : 0xFFFFFFFFu;
      const unsigned mn = __reduce_min_sync(0xFFFFFFFFu, v);
      qual[qq] = __popc(a) >= 2 && mn == i;
    }
  // the other active faces of the qualifying cofaces are distinct (two top
  // cells share only the feature), so each lane's slot is its rank among them
  const bool valid = idx >= 0 && (q ? qual[1] : qual[0]) && (unsigned)idx != i;
  const unsigned vm = __ballot_sync(0xFFFFFFFFu, valid);
  unsigned rk = 0;
  for (unsigned b = vm; b; b &= b - 1) {
    const unsigned o = __shfl_sync(0xFFFFFFFFu, (unsigned)idx, __ffs(b) - 1);
    rk += o < (unsigned)idx ? 1u : 0u;
  }
  if (valid && FTK2B_CHECK(rk < (unsigned)kEdgeSlots, err)) {
    slots[(size_t)i * kEdgeSlots + rk] = (unsigned)idx;
    if (parent) uf_unite(parent, i, (unsigned)idx, err);
  }
  if (lane == 0) cnt[i] = __popc(vm);
}

// Batches: one warp per feature (the short chain's star_edges_warp with the
// feature's field, found by its key).
// The keys live in global memory; every block keeps every 2^slog-th of them
// in shared memory (dynamic, (cap >> slog) + 1 entries) for the lookups, and
// the fields' first keys after them (up to kBatchKbSmem fields): a binary
// search over global memory per feature would cost one dependent load a step.
constexpr int kBatchKbSmem = 4096;
__global__ void edges_batch_warp_kernel(const BatchMesh* __restrict__ fm, const unsigned long long* __restrict__ kb,
                                        int nf, const unsigned long long* __restrict__ keys, const unsigned* n_ptr,
                                        unsigned cap, unsigned* __restrict__ cnt, unsigned* __restrict__ slots,
                                        int slog) {
  extern __shared__ unsigned long long sample[];  // then the fields' first keys, when kb_smem
  __shared__ StarTables T[2];  // d = 3, d = 4
  fill_star_tables(T[0], 3);
  fill_star_tables(T[1], 4);
  const unsigned n = min(*n_ptr, cap);
  const unsigned ns = (n + (1u << slog) - 1) >> slog;
  const unsigned smax = (unsigned)((cap >> slog) + 1);
  for (unsigned j = threadIdx.x; j < ns; j += blockDim.x) sample[j] = keys[(size_t)j << slog];
  const bool kb_smem = nf <= kBatchKbSmem;
  unsigned long long* const skb = sample + smax;
  if (kb_smem)
    for (int f = threadIdx.x; f < nf; f += blockDim.x) skb[f] = kb[f];
  const unsigned long long* fkb = kb_smem ? skb : kb;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nw = (gridDim.x * blockDim.x) >> 5;
  for (unsigned i = gw; i < n; i += nw) {
    const unsigned long long key = keys[i];
    const unsigned f = batch_field_of(fkb, nf, key);
    const RegularMesh mesh = fm[f].mesh;
    star_edges_warp(mesh, fm[f].nch, keys, n, i, key - fkb[f], fkb[f], T[mesh.d - 3], lane, cnt, slots, nullptr,
                    nullptr, sample, ns, slog);
  }
}


__global__ void __launch_bounds__(kSortThreads, 1) small_sort_kernel(PostBuffers B) {
  extern __shared__ unsigned long long sk[];  // the n packed keys, by bucket
  __shared__ unsigned bcnt[kBuckets];
  __shared__ unsigned wsum[33];
  const unsigned t = threadIdx.x;
  for (unsigned b = t; b < kBuckets; b += kSortThreads) bcnt[b] = 0;
  pdl_enter();
  const unsigned n = min(*B.count, B.cap);
  const int shift = B.key_bits > kBucketBits ? B.key_bits - kBucketBits : 0;
  // bucket of a key: its top bits (clamped, which keeps the order)
  auto bucket = [shift](unsigned long long key) {
    return (unsigned)min(key >> shift, (unsigned long long)(kBuckets - 1));
  };
  __syncthreads();
  for (unsigned i = t; i < n; i += kSortThreads) atomicAdd(&bcnt[bucket(B.key[i])], 1u);
  __syncthreads();
  // exclusive scan of the bucket counts, kBuckets / 1024 consecutive per thread
  constexpr int kPerT = kBuckets / kSortThreads;
  unsigned cb[kPerT], sum = 0;
#pragma unroll
  for (int b = 0; b < kPerT; ++b) {
    cb[b] = bcnt[t * kPerT + b];
    sum += cb[b];
  }
  unsigned total;
  unsigned run = block_exclusive_scan(sum, wsum, &total);
#pragma unroll
  for (int b = 0; b < kPerT; ++b) {
    bcnt[t * kPerT + b] = run;
    run += cb[b];
  }
  __syncthreads();
  // scatter; afterwards bcnt[b] = end of bucket b = start of bucket b + 1
  for (unsigned i = t; i < n; i += kSortThreads) {
    const unsigned long long key = B.key[i];
    const unsigned slot = atomicAdd(&bcnt[bucket(key)], 1u);
    if (FTK2B_CHECK(slot < n, B.err)) sk[slot] = (key << kIdxBits) | i;
  }
  __syncthreads();
  // union-find parents of the canonical positions (the edge kernel hooks)
  for (unsigned p = t; p < n; p += kSortThreads) B.parent[p] = p;
  // packed keys compare like their keys (distinct keys)
  for (unsigned p = t; p < n; p += kSortThreads) {
    const unsigned long long v = sk[p];
    const unsigned b = bucket(v >> kIdxBits);
    const unsigned b0 = b ? bcnt[b - 1] : 0u, b1 = bcnt[b];
    unsigned below = 0;
    for (unsigned j = b0; j < b1; ++j) below += sk[j] < v ? 1u : 0u;
    if (FTK2B_CHECK(b0 + below < n, B.err)) B.key_alt[b0 + below] = v;
  }
}

// Outputs of feature i at its canonical position pos.
__device__ __forceinline__ void write_sorted_feature(const RegularMesh& mesh, int nch, const PostBuffers& B,
                                                     unsigned i, unsigned pos, unsigned long long key) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    B.lam_sorted[4 * (size_t)pos + c] = B.lam[4 * (size_t)i + c];
    B.bary4_sorted[4 * (size_t)pos + c] = B.bary4[4 * (size_t)i + c];
  }
  B.scalar_sorted[pos] = B.scalar[i];
  expand_feature(mesh, nch, key, pos, mesh.d, B.bary4_sorted, B.simplices, B.bary);
}

__device__ __forceinline__ void finish_block(const PostBuffers& B, unsigned* sh, unsigned* wsum, unsigned& s_roots);

__global__ void __launch_bounds__(kSortThreads, 1)
    small_edges_kernel(RegularMesh mesh, int nch, PostBuffers B, int want_edges) {
  extern __shared__ unsigned long long sk[];  // the n sorted keys
  __shared__ StarTables T;
  fill_star_tables(T, mesh.d);
  pdl_enter();
  const unsigned n = min(*B.count, B.cap);
  const unsigned G = gridDim.x;
  if (want_edges) {
    for (unsigned p = threadIdx.x; p < n; p += kSortThreads) sk[p] = B.key_alt[p] >> kIdxBits;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const unsigned gw = (blockIdx.x * kSortThreads + threadIdx.x) >> 5;
    const unsigned nw = (G * kSortThreads) >> 5;
    for (unsigned i = gw; i < n; i += nw)
      star_edges_warp(mesh, nch, sk, n, i, sk[i], 0ull, T, lane, B.edge_cnt, B.edge_slots, B.parent, B.err);
  }
  // the outputs of the block's contiguous share of positions (few warps,
  // converged)
  const unsigned share = (n + G - 1) / G, p0 = min(blockIdx.x * share, n), p1 = min(p0 + share, n);
  for (unsigned p = p0 + threadIdx.x; p < p1; p += kSortThreads) {
    const unsigned long long v = B.key_alt[p];
    write_sorted_feature(mesh, nch, B, (unsigned)(v & ((1ull << kIdxBits) - 1)), p, v >> kIdxBits);
  }
  if (!want_edges) return;
  // the last block to finish runs the final step: every block's edge
  // counts, slots and union-find hooks are visible to it (each block fences
  // its writes before counting itself done)
  __shared__ unsigned s_last, s_roots;
  __shared__ unsigned wsum[33];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(B.done, 1u) == G - 1 ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  finish_block(B, reinterpret_cast<unsigned*>(sk), wsum, s_roots);
}

// The short chain's last step, by one block of 1024 threads: exclusive scan
// of the edge counts, edge compaction, every feature's root from the union-find
// parents (copied to shared memory), track ids and root count.  sh: n words
// of shared memory.
__device__ __forceinline__ void finish_block(const PostBuffers& B, unsigned* sh, unsigned* wsum, unsigned& s_roots) {
  constexpr int kPer = (int)(kSmallPostCap / 1024);  // features per thread, at most
  const unsigned n = min(*B.count, B.cap);
  unsigned* const sp = sh;  // the union-find parents
  const unsigned t = threadIdx.x;
  // exclusive scan of the per-feature edge counts: each thread's contiguous
  // segment, its counts loaded first (independent loads)
  const unsigned seg = (n + 1023) / 1024;
  const unsigned s0 = min(t * seg, n);
  unsigned c[kPer];
  unsigned sum = 0;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    c[k] = (k < (int)seg && s0 + k < n) ? __ldcg(&B.edge_cnt[s0 + k]) : 0u;
    sum += c[k];
  }
  // the edge kernel's union-find is complete: its parents into shared memory
  for (unsigned i = t; i < n; i += 1024) sp[i] = __ldcg(&B.parent[i]);
  if (t == 0) s_roots = 0;
  unsigned total;
  unsigned run = block_exclusive_scan(sum, wsum, &total);
  if (t == 0) *B.n_edges = total;
  // the edges of each thread's contiguous run of features at their scanned
  // offsets: the counts are in registers, the slots contiguous in memory
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const unsigned i = s0 + k;
    if (k < (int)seg && i < n) {
      for (unsigned r = 0; r < c[k]; ++r) {
        const unsigned other = __ldcg(&B.edge_slots[(size_t)i * kEdgeSlots + r]);
        const unsigned e = run + r;
        if (e < B.edge_cap) {
          B.edges[2 * (size_t)e] = i;
          B.edges[2 * (size_t)e + 1] = other;
        }
      }
    }
    run += c[k];
  }
  // every feature's root (the minimum of its component) by pointer jumping:
  // each round replaces every parent by its parent's parent, halving every
  // path (reads may see this round's or the last round's values, both
  // ancestors); a path of length L needs log2(L) rounds, at most 14 here
  for (int round = 0; round < 16; ++round) {
    bool changed = false;
    for (unsigned i = t; i < n; i += 1024) {
      const unsigned p = sp[i];
      if (!FTK2B_CHECK(p < n, B.err)) continue;
      const unsigned pp = sp[p];
      if (pp != p) {
        sp[i] = pp;
        changed = true;
      }
    }
    if (!__syncthreads_or(changed)) break;
  }
  unsigned roots = 0;
  for (unsigned i = t; i < n; i += 1024) {
    const unsigned x = sp[i];
    B.track[i] = x;
    roots += x == i ? 1u : 0u;
  }
  atomicAdd(&s_roots, roots);
  __syncthreads();
  if (t == 0) *B.n_roots = s_roots;
}

static cudaError_t launch_post_small(const RegularMesh& mesh, int nch, const PostBuffers& B, int want_edges,
                                     cudaStream_t st, unsigned long long* launches) {
  const unsigned cap = B.cap;
  const size_t key_smem = sizeof(unsigned long long) * (size_t)(cap ? cap : 1);
  // the edge kernel's last block reuses the keys' shared memory for the
  // final step's 2n + 1 words
  const size_t edge_smem = key_smem + 16;
  const int g = B.num_sms > 0 ? B.num_sms : 148;
  cudaError_t e = cudaFuncSetAttribute(small_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)key_smem);
  if (!e) e = launch_pdl(small_sort_kernel, 1, kSortThreads, key_smem, st, B);
  if (!e) e = cudaFuncSetAttribute(small_edges_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)edge_smem);
  if (!e) e = launch_pdl(small_edges_kernel, g, kSortThreads, edge_smem, st, mesh, nch, B, want_edges);
  if (e) return e;
  *launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_post_regular(const RegularMesh& mesh, int nch, const PostBuffers& B,
                                int want_edges, cudaStream_t st, unsigned long long* launches) {
  const unsigned cap = B.cap;
  if (cap <= kSmallPostCap && B.key_bits <= 64 - kIdxBits)
    return launch_post_small(mesh, nch, B, want_edges, st, launches);
  const int gsort = B.sort_grid;
  const int g = grid_for(cap, 256, 4096);
  // keys in canonical order: multi-block stable LSD radix passes
  // consecutive kernels overlap their launch with the predecessor's tail
  // (programmatic dependent launch; each waits for its predecessor first)
  launch_pdl(iota_kernel, g, 256, 0, st, B.perm0, (const unsigned*)B.count, cap);
  const bool alt = radix_sort(B.key, B.perm0, B.key_alt, B.perm1, B.count, cap, B.key_bits, B.hist,
                              gsort, st, launches);
  *launches += 3;  // iota, gather, expand
  const unsigned long long* skey = alt ? B.key_alt : B.key;
  const unsigned* perm = alt ? B.perm1 : B.perm0;
  launch_pdl(gather_kernel, g, 256, 0, st, (const unsigned*)B.count, cap, perm, (const double*)B.lam,
             (const float*)B.scalar, (const float*)B.bary4, B.lam_sorted, B.scalar_sorted, B.bary4_sorted);
  launch_pdl(expand_regular_kernel, g, 256, 0, st, mesh, nch, skey, (const unsigned*)B.count, cap,
             (const float*)B.bary4_sorted, B.simplices, B.bary);
  if (!want_edges) return cudaGetLastError();
  // star edges, written in (centre, other) order: already sorted and unique
  {
    const int gw = grid_for(cap, 8, 8192);  // one warp per feature, 8 warps per block
    launch_pdl(edges_regular_warp_kernel, gw, 256, 0, st, mesh, nch, skey, (const unsigned*)B.count, cap, B.edge_cnt,
               B.edge_slots);
  }
  launch_pdl(scan_inplace_kernel, 1, 1024, 0, st, B.edge_cnt, cap, B.n_edges, (const unsigned*)B.count,
             (const unsigned*)nullptr);
  launch_pdl(edges_compact_kernel, g, 256, 0, st, (const unsigned*)B.count, cap, (const unsigned*)B.edge_cnt,
             (const unsigned*)B.n_edges, (const unsigned*)B.edge_slots, B.edges, B.edge_cap);
  // trajectories
  launch_pdl(uf_init_kernel, g, 256, 0, st, B.parent, (const unsigned*)B.count, cap);
  const int ge = grid_for(B.edge_cap, 256, 4096);
  launch_pdl(uf_hook_kernel, ge, 256, 0, st, B.parent, (const unsigned*)B.edges, (const unsigned*)B.n_edges,
             B.edge_cap, B.err);
  launch_pdl(uf_label_kernel, g, 256, 0, st, B.parent, (const unsigned*)B.count, cap, B.track, B.n_roots);
  *launches += 6;  // edge count, scan, edge write, uf init, hook, label
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// launchers shared with the extruded-mesh pipeline

cudaError_t launch_iota(unsigned* v, const unsigned* n_ptr, unsigned cap, cudaStream_t st) {
  iota_kernel<<<grid_for(cap, 256, 4096), 256, 0, st>>>(v, n_ptr, cap);
  return cudaGetLastError();
}

cudaError_t launch_scan(unsigned* a, unsigned total, unsigned* total_out, const unsigned* n_ptr,
                        cudaStream_t st) {
  scan_inplace_kernel<<<1, 1024, 0, st>>>(a, total, total_out, n_ptr, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_uf(unsigned* parent, const unsigned* n_ptr, unsigned cap, const unsigned* edges,
                      const unsigned* ne_ptr, unsigned edge_cap, unsigned* err, cudaStream_t st) {
  uf_init_kernel<<<grid_for(cap, 256, 4096), 256, 0, st>>>(parent, n_ptr, cap);
  uf_hook_kernel<<<grid_for(edge_cap, 256, 4096), 256, 0, st>>>(parent, edges, ne_ptr, edge_cap, err);
  return cudaGetLastError();
}

cudaError_t launch_uf_label(unsigned* parent, const unsigned* n_ptr, unsigned cap,
                            unsigned long long* track, unsigned* n_roots, cudaStream_t st) {
  uf_label_kernel<<<grid_for(cap, 256, 4096), 256, 0, st>>>(parent, n_ptr, cap, track, n_roots);
  return cudaGetLastError();
}

cudaError_t launch_window_edges_regular(const RegularMesh& mesh, int nch, const unsigned long long* skeys,
                                        const unsigned* n_ptr, unsigned cap, unsigned* edge_cnt,
                                        unsigned* edge_slots, unsigned* edges, unsigned* n_edges,
                                        unsigned edge_cap, cudaStream_t st) {
  const int g = grid_for(cap, 256, 4096);
  edges_regular_warp_kernel<<<grid_for(cap, 8, 8192), 256, 0, st>>>(mesh, nch, skeys, n_ptr, cap, edge_cnt,
                                                                   edge_slots);
  scan_inplace_kernel<<<1, 1024, 0, st>>>(edge_cnt, cap, n_edges, n_ptr, nullptr);
  edges_compact_kernel<<<g, 256, 0, st>>>(n_ptr, cap, edge_cnt, n_edges, edge_slots, edges, edge_cap);
  return cudaGetLastError();
}

cudaError_t launch_expand_regular(const RegularMesh& mesh, int nch, const unsigned long long* keys,
                                  const unsigned* n_ptr, unsigned cap, const float* bary4,
                                  unsigned long long* simplices, float* bary, cudaStream_t st) {
  expand_regular_kernel<<<grid_for(cap, 256, 4096), 256, 0, st>>>(mesh, nch, keys, n_ptr, cap, bary4, simplices,
                                                                  bary);
  return cudaGetLastError();
}


cudaError_t launch_post_batch(const BatchMesh* fm, const unsigned long long* kb, int nf, const PostBuffers& B,
                              unsigned* fbase, cudaStream_t st, unsigned long long* launches) {
  const unsigned cap = B.cap;
  const int g = grid_for(cap, 256, 4096);
  iota_kernel<<<g, 256, 0, st>>>(B.perm0, B.count, cap);
  const bool alt = radix_sort(B.key, B.perm0, B.key_alt, B.perm1, B.count, cap, B.key_bits, B.hist, B.sort_grid,
                              st, launches);
  const unsigned long long* skey = alt ? B.key_alt : B.key;
  const unsigned* perm = alt ? B.perm1 : B.perm0;
  gather_kernel<<<g, 256, 0, st>>>(B.count, cap, perm, B.lam, B.scalar, B.bary4, B.lam_sorted, B.scalar_sorted,
                                   B.bary4_sorted);
  expand_batch_kernel<<<g, 256, 0, st>>>(fm, kb, nf, skey, B.count, cap, B.bary4_sorted, B.simplices, B.bary);
  batch_bounds_kernel<<<(nf + 256) / 256, 256, 0, st>>>(kb, nf, skey, B.count, cap, fbase);
  // a persistent grid: every block copies the face tables and a sample of
  // the sorted keys (every 2^slog-th, at most 8192 entries) into shared memory once
  {
    int slog = 4;
    while (((unsigned long long)cap >> slog) + 1 > 8192ull) ++slog;
    const size_t smp = sizeof(unsigned long long) * (((size_t)cap >> slog) + 1 + (nf <= kBatchKbSmem ? nf : 0));
    cudaFuncSetAttribute(edges_batch_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp);
    edges_batch_warp_kernel<<<(B.num_sms > 0 ? B.num_sms : 148) * 2, 512, smp, st>>>(fm, kb, nf, skey, B.count, cap,
                                                                                      B.edge_cnt, B.edge_slots, slog);
  }
  scan_inplace_kernel<<<1, 1024, 0, st>>>(B.edge_cnt, cap, B.n_edges, B.count, nullptr);
  edges_compact_kernel<<<g, 256, 0, st>>>(B.count, cap, B.edge_cnt, B.n_edges, B.edge_slots, B.edges, B.edge_cap);
  uf_init_kernel<<<g, 256, 0, st>>>(B.parent, B.count, cap);
  uf_hook_kernel<<<grid_for(B.edge_cap, 256, 4096), 256, 0, st>>>(B.parent, B.edges, B.n_edges, B.edge_cap, B.err);
  uf_label_kernel<<<g, 256, 0, st>>>(B.parent, B.count, cap, B.track, B.n_roots);
  *launches += 11;  // iota, gather, expand, bounds, edges, scan, compact, uf init, hook, label (+ sort passes)
  return cudaGetLastError();
}
}  // namespace ftk2b
