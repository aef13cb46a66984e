// Attributes at the features of the last extraction (ftk2b_cp_attributes):
// the values extract_simplex records into FeatureElement::attributes for each
// accepted simplex (engine.hpp:1143-1199), computed on the device from the
// features' vertex ids and their stored float barycentrics:
//
//   attr = sum_i float_lambda_i * value(vertex i)   accumulated in the field
//                                                   precision, then rounded
//                                                   to float
//   COMPONENT: value = a.f(component, coords...)    multicomponent source
//   MAGNITUDE: value = sqrt(sum_c a.f(c, coords...)^2)
//   VALUE:     value = a[vertex id] for 1-D arrays, else a.f(coords - offset)
//
// a.f(i0, i1, ...) is ndarray's Fortran element access with as many indices
// as given (offset = sum_k i_k * prod_{j<k} dim_j); coords are the vertex's
// grid coordinates (the regular spacetime mesh's, or the spatial grid's plus
// the timestep on an extruded regular grid); offset is the regular mesh's
// offset (zero on extruded meshes).  Multiplies and adds are rounded one by
// one (the reference is built without fused multiply-add), sqrt is the
// correctly rounded one.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/ftk2b.h"
#include "cp_api_internal.h"
#include "cp_device.cuh"

using namespace ftk2b;

namespace {

struct AttrDev {
  int kind, component, slot, nd;
  const void* data;
  unsigned long long dims[6];
};

// vertex id -> grid coordinates
struct AttrGeom {
  int n;                        // coordinates per vertex
  int extruded;                 // 1: extruded regular grid (spatial dims + time)
  unsigned long long gd[4];     // grid dims of the coordinates (spatial only when extruded)
  unsigned long long off[4];    // subtracted from VALUE lookups
  unsigned long long S;         // extruded: vertex id stride per timestep
};

// element count of an attribute array: reads at or past it give 0 (the
// reference would read past its array there)
__device__ __forceinline__ unsigned long long attr_elems(const AttrDev& a) {
  unsigned long long t = 1;
  for (int k = 0; k < a.nd; ++k) t *= a.dims[k];
  return t;
}

template <typename T>
__device__ __forceinline__ T fetch(const AttrDev& a, const unsigned long long* idx, int n) {
  unsigned long long o = 0, mul = 1;
  for (int k = 0; k < n; ++k) {
    o += idx[k] * mul;
    mul *= (k < a.nd) ? a.dims[k] : 1ull;
  }
  return o < attr_elems(a) ? static_cast<const T*>(a.data)[o] : T(0);
}

template <typename T>
__global__ void attributes_kernel(AttrGeom g, const AttrDev* __restrict__ attrs, int na,
                                  const unsigned long long* __restrict__ simplices, const float* __restrict__ bary,
                                  unsigned n, int k, float* __restrict__ out) {
  using F = fp<T>;
  const unsigned long long total = (unsigned long long)n * na;
  for (unsigned long long w = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; w < total;
       w += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned f = (unsigned)(w / na);
    const AttrDev a = attrs[w % na];
    T acc = T(0);
    for (int v = 0; v < k; ++v) {
      const unsigned long long vid = simplices[(size_t)f * k + v];
      unsigned long long c[5], idx[6];
      unsigned long long s = vid;
      if (g.extruded) s = vid % g.S;
      for (int q = 0; q < g.n - g.extruded; ++q) {
        c[q] = s % g.gd[q];
        s /= g.gd[q];
      }
      if (g.extruded) c[g.n - 1] = vid / g.S;
      T val;
      if (a.kind == FTK2B_ATTR_COMPONENT) {
        idx[0] = (unsigned long long)a.component;
        for (int q = 0; q < g.n; ++q) idx[q + 1] = c[q];
        val = fetch<T>(a, idx, g.n + 1);
      } else if (a.kind == FTK2B_ATTR_MAGNITUDE) {
        T sq = T(0);
        for (unsigned long long comp = 0; comp < a.dims[0]; ++comp) {
          idx[0] = comp;
          for (int q = 0; q < g.n; ++q) idx[q + 1] = c[q];
          const T cv = fetch<T>(a, idx, g.n + 1);
          sq = F::add(sq, F::mul(cv, cv));
        }
        if constexpr (sizeof(T) == 8) val = __dsqrt_rn(sq);
        else val = __fsqrt_rn(sq);
      } else if (a.nd == 1) {
        val = vid < a.dims[0] ? static_cast<const T*>(a.data)[vid] : T(0);
      } else {
        for (int q = 0; q < g.n; ++q) idx[q] = c[q] - g.off[q];
        val = fetch<T>(a, idx, g.n);
      }
      acc = F::add(acc, F::mul((T)bary[(size_t)f * k + v], val));
    }
    out[(size_t)f * 16 + a.slot] = (float)acc;
  }
}

ftk2b_status afail(ftk2b_ctx* ctx, ftk2b_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  ctx->err = buf;
  return st;
}

#define A_TRY(call)                                                                             \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return afail(ctx, e_ == cudaErrorMemoryAllocation ? FTK2B_OOM : FTK2B_CUDA_ERROR,          \
                   "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

}  // namespace

extern "C" ftk2b_status ftk2b_cp_attributes(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                                            const uint64_t* base_grid_dims, uint32_t n_attrs,
                                            const ftk2b_attribute_desc* attrs, float* out) {
  ftk2b::NvtxRange nvtx_range("ftk2b_cp_attributes");
  if (!ctx) return FTK2B_INVALID_ARG;
  if (!mesh || (n_attrs && !attrs) || !out) return afail(ctx, FTK2B_INVALID_ARG, "null argument");
  if (n_attrs > 16) return afail(ctx, FTK2B_INVALID_ARG, "at most 16 attributes");
  if (ctx->last.n == 0) return FTK2B_OK;  // no features: nothing to write
  if (ctx->last.kind != mesh->kind)
    return afail(ctx, FTK2B_INVALID_ARG, "the mesh kind differs from the last extraction's");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return afail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  const unsigned n = (unsigned)ctx->last.n;
  const int k = ctx->last.m + 1;
  const int f64 = ctx->last.f64;
  const size_t es = f64 ? 8 : 4;
  AttrGeom g;
  std::memset(&g, 0, sizeof(g));
  if (mesh->kind == FTK2B_MESH_REGULAR) {
    if (mesh->ndims < 3 || mesh->ndims > 4) return afail(ctx, FTK2B_INVALID_ARG, "regular meshes have 3 or 4 dims");
    g.n = mesh->ndims;
    for (int q = 0; q < g.n; ++q) {
      g.gd[q] = mesh->global_dims[q] ? mesh->global_dims[q] : 1;
      g.off[q] = mesh->offset[q];
    }
  } else {
    g.extruded = 1;
    g.S = mesh->n_base_verts ? mesh->n_base_verts : 1;
    g.n = mesh->ndims;
    for (int q = 0; q + 1 < g.n; ++q) g.gd[q] = (base_grid_dims && base_grid_dims[q]) ? base_grid_dims[q] : 1;
  }
  AttrDev h[16];
  for (uint32_t i = 0; i < n_attrs; ++i) {
    const ftk2b_attribute_desc& d = attrs[i];
    if (d.slot < 0 || d.slot >= 16) return afail(ctx, FTK2B_INVALID_ARG, "attribute %u: slot out of range", i);
    if (d.kind != FTK2B_ATTR_VALUE && d.kind != FTK2B_ATTR_COMPONENT && d.kind != FTK2B_ATTR_MAGNITUDE)
      return afail(ctx, FTK2B_INVALID_ARG, "attribute %u: unknown kind", i);
    if (d.nd < 1 || d.nd > 6 || !d.data) return afail(ctx, FTK2B_INVALID_ARG, "attribute %u: bad array", i);
    if (mesh->kind == FTK2B_MESH_EXTRUDED && !base_grid_dims && !(d.kind == FTK2B_ATTR_VALUE && d.nd == 1))
      return afail(ctx, FTK2B_UNSUPPORTED,
                   "attribute %u: grid lookups on an extruded mesh need the base grid dims", i);
    std::memset(&h[i], 0, sizeof(AttrDev));
    h[i].kind = d.kind;
    h[i].component = d.component;
    h[i].slot = d.slot;
    h[i].nd = d.nd;
    size_t ne = 1;
    for (int q = 0; q < d.nd; ++q) {
      h[i].dims[q] = d.dims[q];
      ne *= (size_t)d.dims[q];
    }
    if (d.location == FTK2B_DEVICE) {
      h[i].data = d.data;
    } else {
      A_TRY(ctx->attr_stage[i].ensure(ne * es));
      A_TRY(cudaMemcpyAsync(ctx->attr_stage[i].p, d.data, ne * es, cudaMemcpyHostToDevice, ctx->stream));
      h[i].data = ctx->attr_stage[i].p;
    }
  }
  A_TRY(ctx->attr_desc.ensure(sizeof(AttrDev) * 16));
  A_TRY(ctx->attr_out.ensure(sizeof(float) * 16 * (size_t)n));
  A_TRY(cudaMemcpyAsync(ctx->attr_desc.p, h, sizeof(AttrDev) * (n_attrs ? n_attrs : 1), cudaMemcpyHostToDevice,
                        ctx->stream));
  A_TRY(cudaMemsetAsync(ctx->attr_out.p, 0, sizeof(float) * 16 * (size_t)n, ctx->stream));
  if (n_attrs) {
    const unsigned long long work = (unsigned long long)n * n_attrs;
    const unsigned grid = (unsigned)std::min<unsigned long long>((work + 255) / 256, 8192ull);
    const auto* ad = static_cast<const AttrDev*>(ctx->attr_desc.p);
    const auto* sp = static_cast<const unsigned long long*>(ctx->simplices.p);
    const auto* bp = static_cast<const float*>(ctx->bary.p);
    float* op = static_cast<float*>(ctx->attr_out.p);
    if (f64) attributes_kernel<double><<<grid, 256, 0, ctx->stream>>>(g, ad, (int)n_attrs, sp, bp, n, k, op);
    else attributes_kernel<float><<<grid, 256, 0, ctx->stream>>>(g, ad, (int)n_attrs, sp, bp, n, k, op);
    A_TRY(cudaGetLastError());
    ctx->launches += 1;
  }
  A_TRY(cudaMemcpyAsync(out, ctx->attr_out.p, sizeof(float) * 16 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  A_TRY(ctx->sync());
  return FTK2B_OK;
}
