// Small kernels shared by the stream drivers of regular and extruded meshes.
// Static: every translation unit that includes this header gets its own
// copies.
#pragma once

#include "cp_uf.cuh"

namespace ftk2b {

static __global__ void set_u32_kernel(unsigned* p, unsigned v) { *p = v; }

static __global__ void uf_init_range_kernel(unsigned* parent, unsigned lo, unsigned n) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    parent[lo + i] = lo + i;
}

// window edges (indices into the sorted window) -> stream ids, united and
// appended after the `base` edges already stored
// new features whose chain does not step in time are the spatial ones of
// the newest layer
static __global__ void iota_u32_kernel(unsigned* v, unsigned n) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

static __global__ void invert_kernel(const unsigned* __restrict__ perm, unsigned n, unsigned* __restrict__ inv) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) inv[perm[i]] = i;
}

// component minimum of the canonical ids, through the roots of the stream ids
static __global__ void comp_min_kernel(unsigned* parent, const unsigned* __restrict__ inv, unsigned n,
                                unsigned* __restrict__ root, unsigned* cmin, unsigned* n_roots) {
  for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x) {
    const unsigned r = uf_root(parent, id);
    root[id] = r;
    atomicMin(&cmin[r], inv[id]);
    if (r == id) atomicAdd(n_roots, 1u);
  }
}

static __global__ void fill_u32_kernel(unsigned* v, unsigned n, unsigned x) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = x;
}

static __global__ void canon_edges_kernel(const unsigned* __restrict__ edges, unsigned ne,
                                   const unsigned* __restrict__ inv, unsigned long long* __restrict__ out) {
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    const unsigned a = inv[edges[2 * (size_t)e]], b = inv[edges[2 * (size_t)e + 1]];
    out[e] = ((unsigned long long)min(a, b) << 32) | max(a, b);
  }
}

static __global__ void unpack_edges_kernel(const unsigned long long* __restrict__ k, unsigned ne, unsigned* __restrict__ out) {
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    out[2 * (size_t)e] = (unsigned)(k[e] >> 32);
    out[2 * (size_t)e + 1] = (unsigned)k[e];
  }
}

// canonical-order copies of the per-feature records
static __global__ void gather_result_kernel(const unsigned* __restrict__ perm, unsigned n,
                                     const unsigned* __restrict__ root, const unsigned* __restrict__ cmin,
                                     const double* __restrict__ lam, const float* __restrict__ bary4,
                                     const float* __restrict__ sc, const unsigned* __restrict__ cls,
                                     double* __restrict__ lam_o, float* __restrict__ bary4_o,
                                     float* __restrict__ sc_o, unsigned* __restrict__ cls_o,
                                     unsigned long long* __restrict__ track) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned p = perm[i];
    for (int k = 0; k < 4; ++k) {
      lam_o[4 * (size_t)i + k] = lam[4 * (size_t)p + k];
      bary4_o[4 * (size_t)i + k] = bary4[4 * (size_t)p + k];
    }
    sc_o[i] = sc[p];
    cls_o[i] = cls[p];
    track[i] = cmin[root[p]];
  }
}


}  // namespace ftk2b
