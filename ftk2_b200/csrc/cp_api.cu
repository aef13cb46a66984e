// C-ABI layer: contexts, device buffers and the orchestration of the
// critical-point pipeline (extraction -> canonical order -> star edges ->
// trajectories -> output expansion) on the context's stream.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ftk2b.h"
#include "cp_internal.h"
#include "cp_post.h"
#include "cp_api_internal.h"

using namespace ftk2b;

// ---------------------------------------------------------------------------
// helpers

namespace ftk2b {

cudaError_t DevBuf::ensure(size_t want) {
  if (bytes >= want && p) return cudaSuccess;
  ++generation;
  // a buffer that has to grow gets half as much again, so that sizes creeping
  // up call by call reallocate (and synchronise the device) only a few times
  const bool regrow = p != nullptr;
  if (p) {
    if (st) cudaFreeAsync(p, st);
    else cudaFree(p);
  }
  p = nullptr;
  bytes = 0;
  size_t alloc = want < 256 ? 256 : want;
  if (regrow) alloc += alloc / 2;
  auto do_alloc = [&](size_t n) { return st ? cudaMallocAsync(&p, n, st) : cudaMalloc(&p, n); };
  cudaError_t e = do_alloc(alloc);
  if (e != cudaSuccess && regrow) {  // the headroom did not fit: exact size
    cudaGetLastError();
    alloc = want < 256 ? 256 : want;
    e = do_alloc(alloc);
  }
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    return e;
  }
  bytes = alloc;
  return cudaSuccess;
}

void DevBuf::release() {
  if (p) {
    if (st) cudaFreeAsync(p, st);
    else cudaFree(p);
  }
  p = nullptr;
  bytes = 0;
}

}  // namespace ftk2b

static ftk2b_status fail(ftk2b_ctx* ctx, ftk2b_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return st;
}

#define CUDA_TRY(ctx, call)                                                                    \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? FTK2B_OOM : FTK2B_CUDA_ERROR,          \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

constexpr int kMaxDevices = 64;
static std::once_flag g_tables_once[kMaxDevices];

namespace ftk2b {
// constant tables live per device: upload them once for each device, for
// contexts and the allocation-free entry point alike
bool ensure_device_tables(int device) {
  if (device >= 0 && device < kMaxDevices) {
    std::call_once(g_tables_once[device], [] {
      upload_chain_tables();
      upload_post_tables();
    });
  } else {
    upload_chain_tables();
    upload_post_tables();
  }
  return cudaGetLastError() == cudaSuccess;
}
}  // namespace ftk2b

// ---------------------------------------------------------------------------
// context

extern "C" ftk2b_status ftk2b_ctx_create(int device, ftk2b_ctx** out) {
  if (!out) return FTK2B_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return FTK2B_NO_DEVICE;
  }
  if (device < 0 || device >= n) return FTK2B_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return FTK2B_CUDA_ERROR;
  ftk2b_ctx* ctx = new ftk2b_ctx();
  ctx->device = device;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
      cudaEventCreate(&ctx->ev_x) != cudaSuccess || cudaEventCreate(&ctx->ev_r) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_sync, cudaEventBlockingSync | cudaEventDisableTiming) != cudaSuccess) {
    delete ctx;
    return FTK2B_CUDA_ERROR;
  }
  if (cudaMallocHost((void**)&ctx->h_counters, sizeof(unsigned) * kNumCounters) != cudaSuccess) {
    delete ctx;
    return FTK2B_OOM;
  }
  for (DevBuf* b : ctx->all_bufs()) b->st = ctx->stream;
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  ctx->num_sms = prop.multiProcessorCount;
  if (!ensure_device_tables(device)) {
    delete ctx;
    return FTK2B_CUDA_ERROR;
  }
  *out = ctx;
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_ctx_last_phases(ftk2b_ctx* ctx, double* phase_ms) {
  if (!ctx || !phase_ms) return FTK2B_INVALID_ARG;
  for (int i = 0; i < 4; ++i) phase_ms[i] = ctx->phase_ms[i];
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_ctx_last_timing(ftk2b_ctx* ctx, double* extract_ms, double* total_ms,
                                              uint64_t* kernels_launched) {
  if (!ctx) return FTK2B_INVALID_ARG;
  if (extract_ms) *extract_ms = ctx->last_extract_ms;
  if (total_ms) *total_ms = ctx->last.device_ms;
  if (kernels_launched) *kernels_launched = ctx->launches;
  return FTK2B_OK;
}

extern "C" void ftk2b_ctx_destroy(ftk2b_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->release_all();
  cudaStreamSynchronize(ctx->stream);
  ctx->drop_graphs();
  if (ctx->h_counters) cudaFreeHost(ctx->h_counters);
  for (int i = 0; i < 2; ++i) {
    if (ctx->d2h_pin[i]) cudaFreeHost(ctx->d2h_pin[i]);
    if (ctx->d2h_ev[i]) cudaEventDestroy(ctx->d2h_ev[i]);
  }
  if (ctx->batch.h_tab) cudaFreeHost(ctx->batch.h_tab);
  if (ctx->batch.h_fbase) cudaFreeHost(ctx->batch.h_fbase);
  cudaEventDestroy(ctx->ev0);
  cudaEventDestroy(ctx->ev1);
  cudaEventDestroy(ctx->ev_x);
  cudaEventDestroy(ctx->ev_r);
  cudaEventDestroy(ctx->ev_sync);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
}

extern "C" const char* ftk2b_last_error(const ftk2b_ctx* ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

extern "C" void* ftk2b_ctx_stream(ftk2b_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" ftk2b_cp_params ftk2b_cp_params_default(void) {
  ftk2b_cp_params p;
  p.sos_q = 1000000.0;
  p.precision = FTK2B_PRECISION_EXACT;
  p.want_edges = 1;
  p.classify = 0;
  return p;
}

extern "C" ftk2b_status ftk2b_ctx_set_option(ftk2b_ctx* ctx, int option, int64_t value) {
  if (!ctx) return FTK2B_INVALID_ARG;
  switch (option) {
    case FTK2B_OPT_FEATURE_CAPACITY:
      if (value < 0 || value > 0xFFFFFFF0ll) return fail(ctx, FTK2B_INVALID_ARG, "capacity out of range");
      ctx->cap_hint = (unsigned)value;
      return FTK2B_OK;
    case FTK2B_OPT_TIME_CHUNK:
      if (value < 0 || value > (1 << 30)) return fail(ctx, FTK2B_INVALID_ARG, "time chunk out of range");
      ctx->tune_tchunk = (int)value;
      return FTK2B_OK;
    case FTK2B_OPT_DISABLE_TMA:
      ctx->disable_tma = value != 0;
      return FTK2B_OK;
    case FTK2B_OPT_USE_GRAPHS:
      ctx->use_graphs = value != 0;
      ctx->drop_graphs();
      return FTK2B_OK;
    case FTK2B_OPT_BLOCKING_SYNC:
      ctx->blocking_sync = value != 0;
      return FTK2B_OK;
    case FTK2B_OPT_CULL_MODE:
      if (value < 0 || value > 2) return fail(ctx, FTK2B_INVALID_ARG, "cull mode is 0, 1 or 2");
      ctx->cull_mode = (int)value;
      return FTK2B_OK;
    case FTK2B_OPT_TEST_STALL_POLLS:
      if (value < 0 || value > (1 << 22)) return fail(ctx, FTK2B_INVALID_ARG, "stall polls out of range");
      ctx->stall_polls = (int)value;
      return FTK2B_OK;
    case FTK2B_OPT_BATCH_TIME_CHUNK:
      if (value < 0 || value > 65535) return fail(ctx, FTK2B_INVALID_ARG, "batch time chunk out of range");
      ctx->batch.tchunk = (int)value;
      return FTK2B_OK;
    default:
      return fail(ctx, FTK2B_INVALID_ARG, "unknown option %d", option);
  }
}

extern "C" ftk2b_status ftk2b_ctx_get_option(ftk2b_ctx* ctx, int option, int64_t* value) {
  if (!ctx || !value) return FTK2B_INVALID_ARG;
  switch (option) {
    case FTK2B_OPT_FEATURE_CAPACITY: *value = ctx->cap_hint; return FTK2B_OK;
    case FTK2B_OPT_TIME_CHUNK: *value = ctx->tune_tchunk; return FTK2B_OK;
    case FTK2B_OPT_DISABLE_TMA: *value = ctx->disable_tma ? 1 : 0; return FTK2B_OK;
    case FTK2B_INFO_LAST_TMA: *value = ctx->last_used_tma; return FTK2B_OK;
    case FTK2B_INFO_LAST_CULL_MODE: *value = ctx->last_cull_mode; return FTK2B_OK;
    case FTK2B_INFO_LAST_CANDIDATES: *value = (int64_t)ctx->last_candidates; return FTK2B_OK;
    case FTK2B_INFO_LAST_TESTED: *value = (int64_t)ctx->last_tested; return FTK2B_OK;
    case FTK2B_INFO_LAST_BATCH_TIME_CHUNK: *value = ctx->batch.last_tchunk; return FTK2B_OK;
    case FTK2B_OPT_USE_GRAPHS: *value = ctx->use_graphs ? 1 : 0; return FTK2B_OK;
    case FTK2B_OPT_BLOCKING_SYNC: *value = ctx->blocking_sync ? 1 : 0; return FTK2B_OK;
    case FTK2B_OPT_CULL_MODE: *value = ctx->cull_mode; return FTK2B_OK;
    case FTK2B_OPT_BATCH_TIME_CHUNK: *value = ctx->batch.tchunk; return FTK2B_OK;
    case FTK2B_OPT_TEST_STALL_POLLS: *value = ctx->stall_polls; return FTK2B_OK;
    default: return fail(ctx, FTK2B_INVALID_ARG, "unknown option %d", option);
  }
}

void ftk2b_ctx::release_all() {
  // cached graphs point into these buffers
  drop_graphs();
  ext.valid = false;
  for (DevBuf* b : all_bufs()) b->release();
}

std::vector<DevBuf*> ftk2b_ctx::all_bufs() {
  std::vector<DevBuf*> v = {&stage[0], &stage[1], &stage[2], &stage_scalar, &key, &lam, &bary4,
                            &scalar, &key_alt, &perm0, &perm1, &hist, &lam_s, &bary4_s, &scalar_s,
                            &simplices, &bary, &track, &edge_cnt, &edges, &parent, &counters,
                            &cls, &cand_corner, &cand_chains, &edge_slots, &tstats, &runs, &refine_pairs};
  for (auto& b : extra) v.push_back(&b);
  for (DevBuf* b : ext.bufs()) v.push_back(b);
  for (DevBuf* b : batch.bufs()) v.push_back(b);
  v.push_back(&attr_out);
  v.push_back(&attr_desc);
  for (DevBuf& b : attr_stage) v.push_back(&b);
  for (DevBuf& b : contour) v.push_back(&b);
  return v;
}

// ---------------------------------------------------------------------------
// mesh bookkeeping

static int chains_for(int d) { return d == 3 ? 12 : 60; }

static const unsigned char* host_chain_last_masks(int d, int* n) {
  // last vertex mask of every chain, in canonical order (same construction as
  // the device tables)
  static unsigned char last3[12], last4[60];
  static std::once_flag once;
  std::call_once(once, [] {
    for (int d = 3; d <= 4; ++d) {
      const int m = d - 1, full = (1 << d) - 1;
      int cur[5] = {0, 0, 0, 0, 0}, next[5] = {0, 0, 0, 0, 0}, depth = 1, cnt = 0;
      unsigned char* out = d == 3 ? last3 : last4;
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
        if (depth == m) out[cnt++] = (unsigned char)nx;
        else {
          ++depth;
          next[depth] = 0;
        }
      }
    }
  });
  *n = chains_for(d);
  return d == 3 ? last3 : last4;
}

extern "C" uint64_t ftk2b_mesh_simplex_count(const ftk2b_mesh_desc* mesh, int m) {
  if (!mesh) return 0;
  if (mesh->kind == FTK2B_MESH_REGULAR) {
    const int d = mesh->ndims;
    if (d != m + 1 || (d != 3 && d != 4)) return 0;
    int n;
    const unsigned char* last = host_chain_last_masks(d, &n);
    uint64_t total = 0;
    for (int c = 0; c < n; ++c) {
      uint64_t cnt = 1;
      for (int k = 0; k < d; ++k) {
        const uint64_t l = mesh->local_dims[k];
        const uint64_t need = (last[c] >> k) & 1;
        cnt *= (l > need) ? l - need : 0;
      }
      total += cnt;
    }
    return total;
  }
  if (mesh->kind == FTK2B_MESH_EXTRUDED) return extruded_simplex_count(mesh, m);
  return 0;
}

static int bits_for(unsigned long long v) {
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b < 1 ? 1 : b;
}

// ---------------------------------------------------------------------------
// descriptor validation -> FieldAccess

static size_t elem_size(int dtype) { return dtype == FTK2B_F64 ? 8 : 4; }

static uint64_t prod(const uint64_t* d, int n) {
  uint64_t p = 1;
  for (int i = 0; i < n; ++i) p *= d[i];
  return p;
}

ftk2b_status ftk2b::prepare_field(ftk2b_ctx* ctx, const ftk2b_field_desc* f, int mesh_d,
                           const uint64_t* need_global_hi, const uint64_t* need_local_hi,
                           uint64_t n_vertices, FieldAccess& fa, StageArena* arena) {
  memset(&fa, 0, sizeof(fa));
  if (f->dtype != FTK2B_F32 && f->dtype != FTK2B_F64)
    return fail(ctx, FTK2B_INVALID_ARG, "dtype must be FTK2B_F32 or FTK2B_F64");
  const int M = f->ncomp;
  const size_t es = elem_size(f->dtype);
  const bool per_vertex = f->layout == FTK2B_LAYOUT_PER_VERTEX ||
                          (f->layout == FTK2B_LAYOUT_SEPARATE && f->nd == 1);
  int narr = (f->layout == FTK2B_LAYOUT_MULTICOMPONENT) ? 1 : M;
  uint64_t nelem = 0;
  if (f->layout == FTK2B_LAYOUT_MULTICOMPONENT) {
    if (f->nd != mesh_d) return fail(ctx, FTK2B_INVALID_ARG, "multicomponent field needs nd == mesh dims");
    for (int k = 0; k < mesh_d; ++k)
      if (need_global_hi && f->dims[k] < need_global_hi[k])
        return fail(ctx, FTK2B_INVALID_ARG, "field dim %d (%llu) smaller than offset+local (%llu)", k,
                    (unsigned long long)f->dims[k], (unsigned long long)need_global_hi[k]);
    nelem = prod(f->dims, f->nd) * (uint64_t)M;
    for (int k = 0; k < mesh_d; ++k) fa.adims[k] = (long long)f->dims[k];
    long long s = M;
    for (int k = 0; k < mesh_d; ++k) {
      fa.estride[k] = s;
      s *= (long long)f->dims[k];
    }
  } else if (per_vertex) {
    if (f->dims[0] < n_vertices)
      return fail(ctx, FTK2B_INVALID_ARG, "per-vertex field shorter than the vertex count (%llu < %llu)",
                  (unsigned long long)f->dims[0], (unsigned long long)n_vertices);
    nelem = f->dims[0];
    fa.per_vertex = 1;
    fa.adims[0] = (long long)f->dims[0];
  } else if (f->layout == FTK2B_LAYOUT_SEPARATE) {
    if (f->nd != mesh_d) return fail(ctx, FTK2B_INVALID_ARG, "separate arrays need nd == mesh dims");
    for (int k = 0; k < mesh_d; ++k)
      if (need_local_hi && f->dims[k] < need_local_hi[k])
        return fail(ctx, FTK2B_INVALID_ARG, "array dim %d (%llu) smaller than local dim (%llu)", k,
                    (unsigned long long)f->dims[k], (unsigned long long)need_local_hi[k]);
    nelem = prod(f->dims, f->nd);
    for (int k = 0; k < mesh_d; ++k) fa.adims[k] = (long long)f->dims[k];
    long long s = 1;
    for (int k = 0; k < mesh_d; ++k) {
      fa.estride[k] = s;
      s *= (long long)f->dims[k];
    }
  } else {
    return fail(ctx, FTK2B_INVALID_ARG, "unknown layout %d", f->layout);
  }
  for (int j = 0; j < narr; ++j)
    if (!f->comp[j]) return fail(ctx, FTK2B_INVALID_ARG, "component array %d is null", j);

  // device pointers (staging copies for host input)
  // arena: host arrays go to consecutive 256-byte aligned slots of the
  // caller's staging buffer; with a null base only the bytes are counted
  auto arena_slot = [&](size_t bytes) -> unsigned char* {
    const size_t o = arena->off;
    arena->off += (bytes + 255) & ~(size_t)255;
    return arena->base ? arena->base + o : nullptr;
  };
  const void* dev[3] = {nullptr, nullptr, nullptr};
  for (int j = 0; j < narr; ++j) {
    if (f->location == FTK2B_DEVICE) {
      dev[j] = f->comp[j];
    } else if (arena) {
      unsigned char* dst = arena_slot(nelem * es);
      if (dst) CUDA_TRY(ctx, cudaMemcpyAsync(dst, f->comp[j], nelem * es, cudaMemcpyHostToDevice, ctx->stream));
      dev[j] = dst;
    } else {
      CUDA_TRY(ctx, ctx->stage[j].ensure(nelem * es));
      CUDA_TRY(ctx, cudaMemcpyAsync(ctx->stage[j].p, f->comp[j], nelem * es, cudaMemcpyHostToDevice,
                                    ctx->stream));
      dev[j] = ctx->stage[j].p;
    }
  }
  if (f->layout == FTK2B_LAYOUT_MULTICOMPONENT) {
    for (int j = 0; j < M; ++j) fa.comp[j] = (const char*)dev[0] + j * es;
  } else {
    for (int j = 0; j < M; ++j) fa.comp[j] = dev[j];
  }
  // scalar: interpolated only for separate-array fields
  if (f->scalar && f->layout != FTK2B_LAYOUT_MULTICOMPONENT) {
    uint64_t sn;
    if (f->scalar_nd == 1) {
      fa.scalar_per_vertex = 1;
      sn = f->scalar_dims[0];
      if (sn < n_vertices)
        return fail(ctx, FTK2B_INVALID_ARG, "per-vertex scalar shorter than the vertex count (%llu < %llu)",
                    (unsigned long long)sn, (unsigned long long)n_vertices);
    } else {
      if (f->scalar_nd != mesh_d) return fail(ctx, FTK2B_INVALID_ARG, "scalar needs nd == mesh dims");
      for (int k = 0; k < mesh_d; ++k)
        if (need_global_hi && f->scalar_dims[k] < need_global_hi[k])
          return fail(ctx, FTK2B_INVALID_ARG, "scalar dim %d smaller than offset+local", k);
      sn = prod(f->scalar_dims, f->scalar_nd);
      long long s = 1;
      for (int k = 0; k < mesh_d; ++k) {
        fa.sstride[k] = s;
        s *= (long long)f->scalar_dims[k];
      }
    }
    if (f->location == FTK2B_DEVICE) {
      fa.scalar = f->scalar;
    } else if (arena) {
      unsigned char* dst = arena_slot(sn * es);
      if (dst) CUDA_TRY(ctx, cudaMemcpyAsync(dst, f->scalar, sn * es, cudaMemcpyHostToDevice, ctx->stream));
      fa.scalar = dst;
    } else {
      CUDA_TRY(ctx, ctx->stage_scalar.ensure(sn * es));
      CUDA_TRY(ctx, cudaMemcpyAsync(ctx->stage_scalar.p, f->scalar, sn * es, cudaMemcpyHostToDevice,
                                    ctx->stream));
      fa.scalar = ctx->stage_scalar.p;
    }
    fa.has_scalar = 1;
  }
  return FTK2B_OK;
}

// ---------------------------------------------------------------------------
// buffers for one run

ftk2b_status ftk2b::ensure_feature_buffers(ftk2b_ctx* ctx, unsigned cap, unsigned edge_cap, int m) {
  CUDA_TRY(ctx, ctx->key.ensure(sizeof(unsigned long long) * cap));
  CUDA_TRY(ctx, ctx->lam.ensure(sizeof(double) * 4 * (size_t)cap));
  CUDA_TRY(ctx, ctx->bary4.ensure(sizeof(float) * 4 * (size_t)cap));
  CUDA_TRY(ctx, ctx->scalar.ensure(sizeof(float) * cap));
  CUDA_TRY(ctx, ctx->key_alt.ensure(sizeof(unsigned long long) * cap));
  CUDA_TRY(ctx, ctx->perm0.ensure(sizeof(unsigned) * cap));
  CUDA_TRY(ctx, ctx->perm1.ensure(sizeof(unsigned) * cap));
  CUDA_TRY(ctx, ctx->lam_s.ensure(sizeof(double) * 4 * (size_t)cap));
  CUDA_TRY(ctx, ctx->bary4_s.ensure(sizeof(float) * 4 * (size_t)cap));
  CUDA_TRY(ctx, ctx->scalar_s.ensure(sizeof(float) * cap));
  CUDA_TRY(ctx, ctx->simplices.ensure(sizeof(unsigned long long) * (m + 1) * (size_t)cap));
  CUDA_TRY(ctx, ctx->bary.ensure(sizeof(float) * (m + 1) * (size_t)cap));
  CUDA_TRY(ctx, ctx->track.ensure(sizeof(unsigned long long) * cap));
  CUDA_TRY(ctx, ctx->edge_cnt.ensure(sizeof(unsigned) * cap));
  CUDA_TRY(ctx, ctx->parent.ensure(sizeof(unsigned) * cap));
  CUDA_TRY(ctx, ctx->cls.ensure(sizeof(unsigned) * cap));
  CUDA_TRY(ctx, ctx->edges.ensure(sizeof(unsigned) * 2 * (size_t)edge_cap));
  CUDA_TRY(ctx, ctx->edge_slots.ensure(sizeof(unsigned) * 8 * (size_t)cap));
  CUDA_TRY(ctx, ctx->counters.ensure(sizeof(unsigned) * kNumCounters));
  const int grid = ctx->sort_grid(cap);
  CUDA_TRY(ctx, ctx->hist.ensure(sizeof(unsigned) * 256 * (size_t)grid));
  return FTK2B_OK;
}

PostBuffers ftk2b_ctx::post_buffers(unsigned cap_, unsigned edge_cap_, int key_bits) {
  PostBuffers B;
  memset(&B, 0, sizeof(B));
  B.cap = cap_;
  B.edge_cap = edge_cap_;
  B.key_bits = key_bits;
  B.sort_grid = sort_grid(cap_);
  B.num_sms = num_sms;
  B.key = (unsigned long long*)key.p;
  B.lam = (double*)lam.p;
  B.bary4 = (float*)bary4.p;
  B.scalar = (float*)scalar.p;
  unsigned* c = (unsigned*)counters.p;
  B.count = c + kCountFeatures;
  B.n_edges = c + kCountEdges;
  B.n_roots = c + kCountRoots;
  B.err = c + kCountErr;
  B.done = c + kCountDone;
  B.key_alt = (unsigned long long*)key_alt.p;
  B.perm0 = (unsigned*)perm0.p;
  B.perm1 = (unsigned*)perm1.p;
  B.hist = (unsigned*)hist.p;
  B.lam_sorted = (double*)lam_s.p;
  B.bary4_sorted = (float*)bary4_s.p;
  B.scalar_sorted = (float*)scalar_s.p;
  B.simplices = (unsigned long long*)simplices.p;
  B.bary = (float*)bary.p;
  B.track = (unsigned long long*)track.p;
  B.edge_cnt = (unsigned*)edge_cnt.p;
  B.edges = (unsigned*)edges.p;
  B.edge_slots = (unsigned*)edge_slots.p;
  B.parent = (unsigned*)parent.p;
  B.cls = (unsigned*)cls.p;
  return B;
}

// ---------------------------------------------------------------------------
// regular meshes

ftk2b_status ftk2b::build_regular(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, RegularMesh& rm) {
  memset(&rm, 0, sizeof(rm));
  const int d = mesh->ndims;
  if (d != 3 && d != 4) return fail(ctx, FTK2B_UNSUPPORTED, "regular meshes need 3 or 4 dims (got %d)", d);
  rm.d = d;
  unsigned long long s = 1;
  for (int k = 0; k < d; ++k) {
    if (mesh->local_dims[k] < 1 || mesh->global_dims[k] < 1)
      return fail(ctx, FTK2B_INVALID_ARG, "mesh dim %d is zero", k);
    if (mesh->offset[k] + mesh->local_dims[k] > mesh->global_dims[k])
      return fail(ctx, FTK2B_INVALID_ARG, "offset + local exceeds global along dim %d", k);
    if (mesh->local_dims[k] >= (1ull << 16))
      return fail(ctx, FTK2B_UNSUPPORTED, "local mesh dim %d exceeds 65535", k);
    rm.ld[k] = (long long)mesh->local_dims[k];
    rm.off[k] = (long long)mesh->offset[k];
    rm.gd[k] = (long long)mesh->global_dims[k];
    rm.gstride[k] = s;
    s *= mesh->global_dims[k];
  }
  return FTK2B_OK;
}

namespace ftk2b {

cudaError_t setup_cull_scratch(ftk2b_ctx* ctx, const RegularMesh& rm, ExtractConfig& cfg) {
  size_t sb = 0;
  unsigned rc = 0;
  tile_scratch_size(rm, &sb, &rc);
  cudaError_t e = ctx->tstats.ensure(sb);
  if (!e) e = ctx->runs.ensure(16 * (size_t)rc + 16);
  if (e) return e;
  cfg.tstats = (int*)ctx->tstats.p;
  cfg.runs = (unsigned*)ctx->runs.p + 4;
  cfg.n_runs = (unsigned*)ctx->runs.p;
  cfg.runs_cap = rc;
  return cudaSuccess;
}

cudaError_t resolve_cull_mode(ftk2b_ctx* ctx, const RegularMesh& rm, const FieldAccess& fa, int f64, bool multi,
                              const std::function<cudaError_t(int)>& enqueue, int* mode) {
  if (ctx->cull_mode != 2) {
    *mode = ctx->cull_mode;
    return cudaSuccess;
  }
  CullTune k;
  memset(&k, 0, sizeof(k));
  for (int i = 0; i < rm.d; ++i) {
    k.ld[i] = rm.ld[i];
    k.off[i] = rm.off[i];
    k.adims[i] = fa.adims[i];
    k.estride[i] = fa.estride[i];
    k.shift[i] = fa.shift[i];
  }
  k.d = rm.d;
  k.f64 = f64;
  k.multi = multi ? 1 : 0;
  k.tma = ctx->disable_tma ? 0 : 1;
  auto same = [&](const CullTune& a) {
    return memcmp(a.ld, k.ld, sizeof(k.ld)) == 0 && memcmp(a.off, k.off, sizeof(k.off)) == 0 &&
           memcmp(a.adims, k.adims, sizeof(k.adims)) == 0 && memcmp(a.estride, k.estride, sizeof(k.estride)) == 0 &&
           memcmp(a.shift, k.shift, sizeof(k.shift)) == 0 && a.d == k.d && a.f64 == k.f64 && a.multi == k.multi &&
           a.tma == k.tma;
  };
  for (const CullTune& t : ctx->cull_tunes)
    if (same(t)) {
      *mode = t.mode;
      return cudaSuccess;
    }
  cudaError_t e;
  for (int m = 0; m < 2; ++m) {
    float best = 0.f;
    for (int rep = 0; rep < 4; ++rep) {
      if ((e = cudaEventRecord(ctx->ev0, ctx->stream))) return e;
      if ((e = enqueue(m))) return e;
      if ((e = cudaEventRecord(ctx->ev_x, ctx->stream))) return e;
      if ((e = ctx->sync())) return e;
      float ms = 0.f;
      if ((e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev_x))) return e;
      if (rep == 1 || (rep > 1 && ms < best)) best = ms;  // rep 0 warms up
    }
    k.ms[m] = best;
  }
  k.mode = k.ms[1] < k.ms[0] ? 1 : 0;
  if (ctx->cull_tunes.size() >= kMaxCullTunes) ctx->cull_tunes.erase(ctx->cull_tunes.begin());
  ctx->cull_tunes.push_back(k);
  *mode = k.mode;
  return cudaSuccess;
}

}  // namespace ftk2b

// fiber_thr: null for CriticalPointPredicate; the two thresholds for
// FiberPredicate (2D+t meshes)
static ftk2b_status run_regular(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                                const ftk2b_field_desc* field, const ftk2b_cp_params* prm,
                                const double* fiber_thr = nullptr) {
  using Clk = std::chrono::steady_clock;
  auto msd = [](Clk::time_point a, Clk::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
  };
  const Clk::time_point p0 = Clk::now();
  for (double& x : ctx->phase_ms) x = 0;
  RegularMesh rm;
  ftk2b_status st = ftk2b::build_regular(ctx, mesh, rm);
  if (st) return st;
  const int d = rm.d, m = d - 1;
  if (field->ncomp != m)
    return fail(ctx, FTK2B_INVALID_ARG, "a %dD spacetime mesh needs %d components (got %d)", d, m, field->ncomp);
  uint64_t ghi[4], lhi[4];
  uint64_t nv = 1;
  for (int k = 0; k < d; ++k) {
    ghi[k] = mesh->offset[k] + mesh->local_dims[k];
    lhi[k] = mesh->local_dims[k];
    nv *= mesh->global_dims[k];
  }
  FieldAccess fa;
  st = prepare_field(ctx, field, d, ghi, lhi, nv, fa);
  if (st) return st;
  for (int k = 0; k < d; ++k) fa.shift[k] = (field->layout == FTK2B_LAYOUT_SEPARATE) ? rm.off[k] : 0;

  const int nch = chains_for(d);
  const uint64_t nsimp = ftk2b_mesh_simplex_count(mesh, m);
  const int key_bits = bits_for((unsigned long long)nv * (unsigned long long)nch);
  ExtractConfig cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.Q = prm->sos_q;
  cfg.refined = prm->precision == FTK2B_PRECISION_REFINED;
  cfg.cull_mode = ctx->cull_mode;  // 2 is resolved below, once the buffers exist
  if (ctx->stall_polls > 0) {  // the failure-path check runs in the fused cull
    cfg.stall_polls = ctx->stall_polls;
    cfg.cull_mode = 0;
  }
  if (fiber_thr) {
    cfg.fiber = 1;
    cfg.fthr[0] = fiber_thr[0];
    cfg.fthr[1] = fiber_thr[1];
    cfg.cull_mode = 0;
    cfg.refined = 0;
  }
  cfg.tchunk = (int)rm.ld[d - 1];
  if (cfg.cull_mode != 0) CUDA_TRY(ctx, setup_cull_scratch(ctx, rm, cfg));
  if (ctx->tune_tchunk > 0) cfg.tchunk = ctx->tune_tchunk;
  int TX, TY, TZ;
  regular_tile(d, &TX, &TY, &TZ);
  cfg.tiles[0] = (int)((rm.ld[0] + TX - 1) / TX);
  cfg.tiles[1] = (int)((rm.ld[1] + TY - 1) / TY);
  cfg.tiles[2] = (d == 4) ? (int)((rm.ld[2] + TZ - 1) / TZ) : 1;

  // feature capacity: starts small (sorting cost scales with it; up to
  // kSmallPostCap the short post-extraction chain runs) and grows on
  // overflow; the context remembers the grown value
  unsigned cap = ctx->cap_hint ? ctx->cap_hint : kSmallPostCap;
  unsigned ccap = ctx->cand_cap_hint ? ctx->cand_cap_hint : 65536u;
  if (fiber_thr) {  // every local vertex is a candidate corner
    uint64_t nloc = 1;
    for (int k = 0; k < d; ++k) nloc *= rm.ld[k];
    if (nloc > 0xFFFFFFF0ull) return fail(ctx, FTK2B_UNSUPPORTED, "mesh too large for fiber extraction");
    ccap = std::max<unsigned>(ccap, (unsigned)nloc);
  }
  for (int attempt = 0; attempt < 4; ++attempt) {
    const unsigned edge_cap = cap * 2;
    st = ensure_feature_buffers(ctx, cap, edge_cap, m);
    if (st) return st;
    CUDA_TRY(ctx, ctx->cand_corner.ensure(sizeof(unsigned long long) * (size_t)ccap));
    CUDA_TRY(ctx, ctx->cand_chains.ensure(sizeof(unsigned long long) * (size_t)ccap));
    CUDA_TRY(ctx, ctx->refine_pairs.ensure(refine_mask_bytes(ccap, cap)));
    PostBuffers B = ctx->post_buffers(cap, edge_cap, key_bits);
    FeatureSink sink;
    sink.key = B.key;
    sink.lam = B.lam;
    sink.bary4 = B.bary4;
    sink.scalar = B.scalar;
    sink.count = B.count;
    sink.cap = cap;
    CandidateQueue cq{};
    cq.corner = (unsigned long long*)ctx->cand_corner.p;
    cq.chains = (unsigned long long*)ctx->cand_chains.p;
    cq.count = (unsigned*)ctx->counters.p + kCountCand;
    cq.cap = ccap;
    RefineStage rs;
    // the single-field test keeps values and quantised values in shared
    // memory and reads the field again for the solve: no staging block
    refine_stage_bind(rs, ctx->refine_pairs.p, ccap, cap);
    rs.count = (unsigned*)ctx->counters.p + kCountPairs;
    rs.err = (unsigned*)ctx->counters.p + kCountErr;
    rs.big_count = (unsigned*)ctx->counters.p + kCountBig;
    rs.acc_count = (unsigned*)ctx->counters.p + kCountAcc;
    const int f64 = field->dtype == FTK2B_F64;
    // the device pipeline after the counters' reset in two parts, so that the
    // fused cull kernel can be timed on its own: [cull] and [exact tests,
    // canonical order, star edges, trajectories, counters readback]
    auto enqueue0 = [&]() -> cudaError_t {
      return cudaMemsetAsync(ctx->counters.p, 0, sizeof(unsigned) * kNumCounters, ctx->stream);
    };
    auto enqueue1 = [&](unsigned long long* nl) -> cudaError_t {
      cudaError_t e;
      int nk = 1;
      if (cfg.fiber) {
        if ((e = launch_fiber_candidates(rm, cq, ctx->num_sms, ctx->stream))) return e;
      } else if ((e = launch_extract_regular(f64, rm, fa, cfg, cq, B.err, ctx->stream, !ctx->disable_tma,
                                             &ctx->last_used_tma, &nk))) {
        return e;
      }
      *nl += (unsigned long long)nk;
      return cudaSuccess;
    };
    auto enqueue2 = [&](unsigned long long* nl) -> cudaError_t {
      cudaError_t e;
      if ((e = launch_refine_staged(f64, rm, fa, cfg, cq, rs, sink, ctx->num_sms, ctx->stream))) return e;
      *nl += 2;
      if ((e = launch_post_regular(rm, nch, B, prm->want_edges, ctx->stream, nl))) return e;
      if (prm->classify && !cfg.fiber) {
        if ((e = launch_classify_regular(f64, rm, fa, nch, B, ctx->stream))) return e;
        *nl += 1;
      }
      return cudaMemcpyAsync(ctx->h_counters, ctx->counters.p, sizeof(unsigned) * kNumCounters,
                             cudaMemcpyDeviceToHost, ctx->stream);
    };
    if (cfg.cull_mode == 2) {
      int mode = 0;
      NvtxRange tune_range("ftk2b_tune_cull_mode");
      CUDA_TRY(ctx, resolve_cull_mode(ctx, rm, fa, f64, field->layout == FTK2B_LAYOUT_MULTICOMPONENT,
                                      [&](int md) -> cudaError_t {
                                        ExtractConfig c = cfg;
                                        c.cull_mode = md;
                                        cudaError_t e = cudaMemsetAsync(ctx->counters.p, 0,
                                                                        sizeof(unsigned) * kNumCounters, ctx->stream);
                                        int nk = 1;
                                        if (!e)
                                          e = launch_extract_regular(f64, rm, fa, c, cq, B.err, ctx->stream,
                                                                     !ctx->disable_tma, &ctx->last_used_tma, &nk);
                                        ctx->launches += (unsigned long long)nk;
                                        return e;
                                      },
                                      &mode));
      cfg.cull_mode = mode;
    }
    ctx->last_cull_mode = cfg.cull_mode;
    const Clk::time_point p1 = Clk::now();
    ctx->phase_ms[0] += msd(p0, p1);
    Clk::time_point p2 = p1;
    if (ctx->use_graphs) {
      RegularGraphKey key;
      memset(&key, 0, sizeof(key));
      key.rm = rm;
      key.fa = fa;
      key.cfg = cfg;
      key.cap = cap;
      key.ccap = ccap;
      key.edge_cap = edge_cap;
      key.f64 = f64;
      key.want_edges = prm->want_edges;
      key.classify = prm->classify;
      key.allow_tma = !ctx->disable_tma;
      key.key_bits = key_bits;
      key.nch = nch;
      const unsigned long long gen = ctx->buffer_generation();
      GraphEntry* ent = nullptr;
      for (auto it = ctx->graphs.begin(); it != ctx->graphs.end();) {
        if (it->gen != gen) {  // captured over buffers that have been reallocated since
          if (it->g1) cudaGraphExecDestroy(it->g1);
          if (it->g2) cudaGraphExecDestroy(it->g2);
          it = ctx->graphs.erase(it);
          continue;
        }
        if (memcmp(&it->key, &key, sizeof(key)) == 0) ent = &*it;
        ++it;
      }
      if (!ent) {
        NvtxRange capture_range("ftk2b_capture_pipeline");
        if (ctx->graphs.size() >= kMaxGraphs) {
          auto lru = ctx->graphs.begin();
          for (auto it = ctx->graphs.begin(); it != ctx->graphs.end(); ++it)
            if (it->last_use < lru->last_use) lru = it;
          if (lru->g1) cudaGraphExecDestroy(lru->g1);
          if (lru->g2) cudaGraphExecDestroy(lru->g2);
          ctx->graphs.erase(lru);
        }
        GraphEntry e;
        e.key = key;
        e.gen = gen;
        unsigned long long nl = 0;
        // one graph for the whole pipeline, the call's three timing events
        // captured as event-record nodes; two graphs with the events recorded
        // between their launches when that capture fails
        {
          cudaGraph_t graph = nullptr;
          CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
          cudaError_t ce = enqueue0();
          if (!ce) ce = cudaEventRecordWithFlags(ctx->ev0, ctx->stream, cudaEventRecordExternal);
          if (!ce) ce = enqueue1(&nl);
          if (!ce) ce = cudaEventRecordWithFlags(ctx->ev_x, ctx->stream, cudaEventRecordExternal);
          if (!ce) ce = enqueue2(&nl);
          if (!ce) ce = cudaEventRecordWithFlags(ctx->ev1, ctx->stream, cudaEventRecordExternal);
          const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &graph);
          if (!ce && !ee && cudaGraphInstantiate(&e.g1, graph, 0) == cudaSuccess) {
            cudaGraphDestroy(graph);
          } else {
            if (graph) cudaGraphDestroy(graph);
            e.g1 = nullptr;
            nl = 0;
            cudaGetLastError();
          }
        }
        cudaGraphExec_t* slots[2] = {&e.g1, &e.g2};
        for (int part = 0; part < 2 && !(part == 0 && e.g1); ++part) {
          cudaGraph_t graph = nullptr;
          CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
          cudaError_t ce = part == 0 ? enqueue1(&nl) : enqueue2(&nl);
          cudaError_t ee = cudaStreamEndCapture(ctx->stream, &graph);
          if (ce || ee) {
            if (graph) cudaGraphDestroy(graph);
            if (e.g1) cudaGraphExecDestroy(e.g1);
            cudaGetLastError();
            return fail(ctx, FTK2B_CUDA_ERROR, "graph capture failed: %s",
                        cudaGetErrorString(ce ? ce : ee));
          }
          cudaError_t ie = cudaGraphInstantiate(slots[part], graph, 0);
          cudaGraphDestroy(graph);
          if (ie) {
            if (e.g1 && part == 1) cudaGraphExecDestroy(e.g1);
            return fail(ctx, FTK2B_CUDA_ERROR, "graph instantiate failed: %s", cudaGetErrorString(ie));
          }
        }
        e.launches = nl;
        e.used_tma = ctx->last_used_tma;
        ctx->graphs.push_back(e);
        ent = &ctx->graphs.back();
      }
      ent->last_use = ++ctx->graph_clock;
      ctx->last_used_tma = ent->used_tma;
      p2 = Clk::now();
      ctx->phase_ms[1] += msd(p1, p2);
      if (ent->g2) {
        CUDA_TRY(ctx, enqueue0());
        CUDA_TRY(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
        CUDA_TRY(ctx, cudaGraphLaunch(ent->g1, ctx->stream));
        CUDA_TRY(ctx, cudaEventRecord(ctx->ev_x, ctx->stream));
        CUDA_TRY(ctx, cudaGraphLaunch(ent->g2, ctx->stream));
        CUDA_TRY(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
      } else {
        CUDA_TRY(ctx, cudaGraphLaunch(ent->g1, ctx->stream));  // the event records are nodes of the graph
      }
      ctx->launches += ent->launches;
    } else {
      unsigned long long nl = 0;
      CUDA_TRY(ctx, enqueue0());
      CUDA_TRY(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
      CUDA_TRY(ctx, enqueue1(&nl));
      CUDA_TRY(ctx, cudaEventRecord(ctx->ev_x, ctx->stream));
      CUDA_TRY(ctx, enqueue2(&nl));
      CUDA_TRY(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
      ctx->launches += nl;
    }
    {
      NvtxRange wait_range("ftk2b_pipeline_wait");
      CUDA_TRY(ctx, ctx->sync());
    }
    ctx->phase_ms[2] += msd(p2, Clk::now());
    unsigned h[kNumCounters];
    memcpy(h, ctx->h_counters, sizeof(h));
    float ms = 0.f, xms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) != cudaSuccess) ms = 0.f;
    if (cudaEventElapsedTime(&xms, ctx->ev0, ctx->ev_x) != cudaSuccess) xms = 0.f;
    cudaGetLastError();  // a failed timing query must not linger in the error slot
    ctx->last_extract_ms = xms;
    ctx->last_candidates = h[kCountCand];
    ctx->last_tested = h[kCountPairs];
    if (h[kCountErr] & kErrBounds) return fail(ctx, FTK2B_INTERNAL, "a device bounds check failed (checked build)");
    if (h[kCountErr] & 2u) return fail(ctx, FTK2B_TIMEOUT, "a TMA slice copy did not complete in time");
    if (h[kCountErr]) return fail(ctx, FTK2B_TIMEOUT, "union-find retry bound reached");
    if (h[kCountCand] > ccap) {
      const uint64_t want = (uint64_t)h[kCountCand] + h[kCountCand] / 4 + 1024;
      if (want > 0xFFFFFFF0ull) return fail(ctx, FTK2B_OVERFLOW_RETRY, "candidate count exceeds 2^32");
      ccap = (unsigned)want;
      ctx->cand_cap_hint = ccap;
      continue;
    }
    if (h[kCountFeatures] > cap || h[kCountEdges] > edge_cap) {
      uint64_t want = (uint64_t)h[kCountFeatures] + h[kCountFeatures] / 4 + 1024;
      const uint64_t want_e = ((uint64_t)h[kCountEdges] + 1) / 2 + 1024;
      if (want_e > want) want = want_e;
      if (want > 0xFFFFFFF0ull) return fail(ctx, FTK2B_OVERFLOW_RETRY, "feature count exceeds 2^32");
      cap = (unsigned)want;
      ctx->cap_hint = cap;
      continue;
    }
    ctx->last.kind = FTK2B_MESH_REGULAR;
    ctx->last.m = m;
    ctx->last.f64 = field->dtype == FTK2B_F64;
    ctx->last.n = h[kCountFeatures];
    ctx->last.ne = prm->want_edges ? h[kCountEdges] : 0;
    ctx->last.n_roots = h[kCountRoots];
    ctx->last.n_simplices = nsimp;
    ctx->last.device_ms = ms;
    ctx->last.classify = prm->classify && !cfg.fiber;
    ctx->last.want_edges = prm->want_edges;
    return FTK2B_OK;
  }
  return fail(ctx, FTK2B_OVERFLOW_RETRY, "feature buffer overflow persisted after retries");
}

// ---------------------------------------------------------------------------

extern "C" ftk2b_status ftk2b_cp_run(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                                     const ftk2b_field_desc* field, const ftk2b_cp_params* params,
                                     uint64_t* n_features, uint64_t* n_edges) {
  ftk2b::NvtxRange nvtx_range("ftk2b_cp_run");
  if (!ctx) return FTK2B_INVALID_ARG;
  if (!mesh || !field) return fail(ctx, FTK2B_INVALID_ARG, "null descriptor");
  ftk2b_cp_params prm = params ? *params : ftk2b_cp_params_default();
  if (!(prm.sos_q > 0)) return fail(ctx, FTK2B_INVALID_ARG, "sos_q must be positive");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  ftk2b_status st;
  if (mesh->kind == FTK2B_MESH_REGULAR) st = run_regular(ctx, mesh, field, &prm);
  else if (mesh->kind == FTK2B_MESH_EXTRUDED) st = run_extruded(ctx, mesh, field, &prm);
  else st = fail(ctx, FTK2B_INVALID_ARG, "unknown mesh kind %d", mesh->kind);
  if (st == FTK2B_OK) {
    if (n_features) *n_features = ctx->last.n;
    if (n_edges) *n_edges = ctx->last.ne;
  }
  return st;
}

extern "C" ftk2b_status ftk2b_cp_fetch(ftk2b_ctx* ctx, ftk2b_cp_result** out) {
  ftk2b::NvtxRange nvtx_range("ftk2b_cp_fetch");
  if (!ctx || !out) return FTK2B_INVALID_ARG;
  const auto f0 = std::chrono::steady_clock::now();
  struct PhaseTimer {
    ftk2b_ctx* c;
    std::chrono::steady_clock::time_point t;
    ~PhaseTimer() {
      c->phase_ms[3] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
    }
  } phase_timer{ctx, f0};
  *out = nullptr;
  const uint64_t n = ctx->last.n, ne = ctx->last.ne;
  const int m = ctx->last.m;
  ftk2b_cp_result* r = (ftk2b_cp_result*)calloc(1, sizeof(ftk2b_cp_result));
  if (!r) return fail(ctx, FTK2B_OOM, "host allocation failed");
  r->m = m;
  r->n_features = n;
  r->n_edges = ne;
  r->n_tracks = ctx->last.want_edges ? ctx->last.n_roots : 0;
  r->n_simplices = ctx->last.n_simplices;
  r->device_ms = ctx->last.device_ms;
  const size_t k = (size_t)(m + 1);
  r->simplices = (uint64_t*)malloc(sizeof(uint64_t) * (n * k + 1));
  r->lambda = (double*)malloc(sizeof(double) * (n * k + 1));
  r->barycentric = (float*)malloc(sizeof(float) * (n * k + 1));
  r->track_id = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  r->type = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
  r->cp_class = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
  r->scalar = (float*)malloc(sizeof(float) * (n + 1));
  r->edges = (uint32_t*)malloc(sizeof(uint32_t) * (2 * ne + 2));
  std::vector<double> lam4((size_t)n * 4 + 4);
  if (!r->simplices || !r->lambda || !r->barycentric || !r->track_id || !r->type || !r->cp_class ||
      !r->scalar || !r->edges) {
    ftk2b_cp_result_free(r);
    return fail(ctx, FTK2B_OOM, "host allocation failed");
  }
  cudaStream_t s = ctx->stream;
  auto d2h = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    if (!bytes) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
  };
  cudaError_t e = cudaSuccess;
  if (!e) e = d2h(r->simplices, ctx->simplices.p, sizeof(uint64_t) * n * k);
  if (!e) e = d2h(r->barycentric, ctx->bary.p, sizeof(float) * n * k);
  if (!e) e = d2h(lam4.data(), ctx->lam_s.p, sizeof(double) * n * 4);
  if (!e) e = d2h(r->scalar, ctx->scalar_s.p, sizeof(float) * n);
  if (!e && ctx->last.want_edges) e = d2h(r->track_id, ctx->track.p, sizeof(uint64_t) * n);
  if (!e && ctx->last.classify) e = d2h(r->cp_class, ctx->cls.p, sizeof(uint32_t) * n);
  if (!e) e = d2h(r->edges, ctx->edges.p, sizeof(uint32_t) * 2 * ne);
  if (!e) e = ctx->sync();
  if (e) {
    ftk2b_cp_result_free(r);
    return fail(ctx, FTK2B_CUDA_ERROR, "result copy failed: %s", cudaGetErrorString(e));
  }
  for (uint64_t i = 0; i < n; ++i)
    for (size_t v = 0; v < k; ++v) r->lambda[i * k + v] = lam4[i * 4 + v];
  if (!ctx->last.want_edges)
    for (uint64_t i = 0; i < n; ++i) r->track_id[i] = i;
  *out = r;
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_fiber_extract(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                                            const ftk2b_field_desc* field, const double thresholds[2],
                                            double sos_q, ftk2b_cp_result** out) {
  ftk2b::NvtxRange nvtx_range("ftk2b_fiber_extract");
  if (!ctx) return FTK2B_INVALID_ARG;
  if (!mesh || !field || !thresholds || !out) return fail(ctx, FTK2B_INVALID_ARG, "null argument");
  *out = nullptr;
  if (mesh->ndims != 3 || (mesh->kind != FTK2B_MESH_REGULAR && mesh->kind != FTK2B_MESH_EXTRUDED))
    return fail(ctx, FTK2B_UNSUPPORTED, "fibers run on 2D+t meshes (regular, or extruded over triangles)");
  if (field->ncomp != 2) return fail(ctx, FTK2B_INVALID_ARG, "fibers read two scalar fields (ncomp 2)");
  if (field->scalar) return fail(ctx, FTK2B_INVALID_ARG, "fibers interpolate no scalar");
  if (!(sos_q > 0)) return fail(ctx, FTK2B_INVALID_ARG, "sos_q must be positive");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  ftk2b_cp_params prm = ftk2b_cp_params_default();
  prm.sos_q = sos_q;
  prm.precision = FTK2B_PRECISION_EXACT;
  prm.classify = 0;
  prm.want_edges = 1;
  const ftk2b_status st = mesh->kind == FTK2B_MESH_REGULAR ? run_regular(ctx, mesh, field, &prm, thresholds)
                                                          : run_extruded(ctx, mesh, field, &prm, thresholds);
  if (st) return st;
  return ftk2b_cp_fetch(ctx, out);
}

extern "C" ftk2b_status ftk2b_cp_extract(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                                         const ftk2b_field_desc* field, const ftk2b_cp_params* params,
                                         ftk2b_cp_result** out) {
  ftk2b::NvtxRange nvtx_range("ftk2b_cp_extract");
  if (!out) return ctx ? fail(ctx, FTK2B_INVALID_ARG, "null output") : FTK2B_INVALID_ARG;
  *out = nullptr;
  ftk2b_status st = ftk2b_cp_run(ctx, mesh, field, params, nullptr, nullptr);
  if (st) return st;
  return ftk2b_cp_fetch(ctx, out);
}

extern "C" void ftk2b_cp_result_free(ftk2b_cp_result* r) {
  if (!r) return;
  free(r->simplices);
  free(r->lambda);
  free(r->barycentric);
  free(r->track_id);
  free(r->type);
  free(r->cp_class);
  free(r->scalar);
  free(r->edges);
  free(r);
}
