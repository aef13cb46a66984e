// Time streams over a fixed spatial mesh: timesteps are pushed one at a time
// and only a two-timestep window of the field is kept on the device.
//
// Replaces the reference's streaming drivers (execute_stream and
// execute_cuda_streaming_regular, engine.hpp:214-270, 601-819) with one-shot
// semantics: after T pushes, ftk2b_stream_result returns exactly what
// ftk2b_cp_extract (execute() + get_complex(), engine.hpp:96-99, 822-996)
// returns for the T-timestep spacetime mesh.
//
// Push of timestep t (t >= 1), window = layers [t-1, t]:
//   1. the step is copied into ring slot t & 1;
//   2. the fused extraction runs on the window with the purely spatial
//      simplices of layer t-1 skipped (the previous push found them), so the
//      new features are exactly the simplices whose last layer is t;
//   3. the window's features (new ones plus the spatial features of layer
//      t-1) are sorted, and the star edges of every top cell of slab
//      [t-1, t] are emitted -- every top cell belongs to exactly one slab, and
//      its centre (smallest face in Simplex order) is decided inside it;
//   4. the resident union-find over stream ids takes the new edges.
// The result sorts the store (canonical ids = rank in Simplex order) and
// labels every component with its smallest canonical id (engine.hpp:46-74).
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "cp_post.h"
#include "cp_stream.h"
#include "cp_stream_kernels.cuh"
#include "cp_uf.cuh"

using namespace ftk2b;

namespace {

enum { kSWin = 5, kSWinEdges = 6, kSPrev = 7 };

ftk2b_status sfail(ftk2b_ctx* ctx, ftk2b_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return st;
}

#define S_TRY(ctx, call)                                                                        \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return sfail(ctx, e_ == cudaErrorMemoryAllocation ? FTK2B_OOM : FTK2B_CUDA_ERROR,          \
                   "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

int bits_for(unsigned long long v) {
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

__global__ void window_build_kernel(const unsigned long long* __restrict__ key, const unsigned* __restrict__ prev,
                                    unsigned n_prev, unsigned first_new, unsigned n_new,
                                    unsigned long long* __restrict__ s_key, unsigned* __restrict__ s_id) {
  const unsigned nS = n_prev + n_new;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < nS; i += gridDim.x * blockDim.x) {
    const unsigned id = i < n_prev ? prev[i] : first_new + (i - n_prev);
    s_key[i] = key[id];
    s_id[i] = id;
  }
}

__global__ void append_edges_kernel(const unsigned* __restrict__ wedges, const unsigned* wn_ptr, unsigned wcap,
                                    const unsigned* __restrict__ s_id, unsigned* parent, unsigned* __restrict__ out,
                                    unsigned base, unsigned out_cap, unsigned* err) {
  const unsigned wn = min(*wn_ptr, wcap);
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < wn; e += gridDim.x * blockDim.x) {
    const unsigned a = s_id[wedges[2 * (size_t)e]], b = s_id[wedges[2 * (size_t)e + 1]];
    uf_unite(parent, a, b, err);
    if (base + e < out_cap) {
      out[2 * (size_t)(base + e)] = a;
      out[2 * (size_t)(base + e) + 1] = b;
    }
  }
}

__global__ void collect_spatial_kernel(const unsigned long long* __restrict__ key, unsigned first_new,
                                       unsigned n_new, int nch, unsigned long long time_chains,
                                       unsigned* __restrict__ prev, unsigned* prev_n) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += gridDim.x * blockDim.x) {
    const unsigned id = first_new + i;
    const unsigned ch = (unsigned)(key[id] % (unsigned long long)nch);
    if (!((time_chains >> ch) & 1ull)) prev[atomicAdd(prev_n, 1u)] = id;
  }
}

unsigned long long time_chain_mask(int d) {
  // chains (canonical order) whose last vertex mask has the time bit
  const int m = d - 1, full = (1 << d) - 1, tbit = 1 << (d - 1);
  unsigned long long mask = 0;
  int cur[5] = {0, 0, 0, 0, 0}, next[5] = {0, 0, 0, 0, 0}, depth = 1, cnt = 0;
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
      if (nx & tbit) mask |= 1ull << cnt;
      ++cnt;
    } else {
      ++depth;
      next[depth] = 0;
    }
  }
  return mask;
}

RegularMesh window_mesh(const ftk2b_stream* s, uint64_t t_start, uint64_t lt) {
  RegularMesh rm;
  memset(&rm, 0, sizeof(rm));
  rm.d = s->d;
  unsigned long long st = 1;
  for (int k = 0; k < s->d; ++k) {
    const bool tm = k == s->d - 1;
    rm.ld[k] = tm ? (long long)lt : (long long)s->ld[k];
    rm.off[k] = tm ? (long long)t_start : (long long)s->off[k];
    rm.gd[k] = tm ? (1ll << 30) : (long long)s->gd[k];
    rm.gstride[k] = st;
    st *= (unsigned long long)rm.gd[k];
  }
  return rm;
}

FieldAccess window_field(const ftk2b_stream* s, uint64_t t_start) {
  FieldAccess fa;
  memset(&fa, 0, sizeof(fa));
  const int d = s->d, M = s->m;
  const bool multi = s->layout == FTK2B_LAYOUT_MULTICOMPONENT;
  long long st = multi ? M : 1;
  for (int k = 0; k < d; ++k) {
    const bool tm = k == d - 1;
    fa.adims[k] = tm ? 2 : (long long)s->adims[k];
    fa.estride[k] = st;
    st *= fa.adims[k];
    fa.shift[k] = tm ? (long long)t_start : (multi ? 0 : (long long)s->off[k]);
  }
  for (int j = 0; j < M; ++j)
    fa.comp[j] = multi ? (const void*)((const char*)s->ring[0].p + j * s->es) : s->ring[j].p;
  fa.tflip = (int)(t_start & 1);
  return fa;
}

ftk2b_status push_regular(ftk2b_stream* s) {
  ftk2b_ctx* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  const int d = s->d, M = s->m;
  const int nch = d == 3 ? 12 : 60;
  const uint64_t T = s->T;
  const uint64_t t_start = T ? T - 1 : 0, lt = T ? 2 : 1;
  const RegularMesh rm = window_mesh(s, t_start, lt);
  const FieldAccess fa = window_field(s, t_start);
  ExtractConfig cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.Q = s->prm.sos_q;
  cfg.refined = s->prm.precision == FTK2B_PRECISION_REFINED;
  cfg.tchunk = (int)lt;
  cfg.skip_first_spatial = T > 0;
  cfg.cull_mode = ctx->cull_mode;  // 2 is resolved below, once the buffers exist
  if (cfg.cull_mode != 0) S_TRY(ctx, setup_cull_scratch(ctx, rm, cfg));
  int TX, TY, TZ;
  regular_tile(d, &TX, &TY, &TZ);
  cfg.tiles[0] = (int)((rm.ld[0] + TX - 1) / TX);
  cfg.tiles[1] = (int)((rm.ld[1] + TY - 1) / TY);
  cfg.tiles[2] = (d == 4) ? (int)((rm.ld[2] + TZ - 1) / TZ) : 1;
  const int f64 = s->dtype == FTK2B_F64;

  S_TRY(ctx, ctx->counters.ensure(sizeof(unsigned) * kNumCounters));
  unsigned* counters = (unsigned*)ctx->counters.p;
  ftk2b_status rc = ensure_stream_store(s, s->n + 1024);
  if (rc) return rc;
  unsigned ccap = ctx->cand_cap_hint ? ctx->cand_cap_hint : 65536u;
  unsigned n_new = 0;
  for (int attempt = 0;; ++attempt) {
    if (attempt == 6) return sfail(ctx, FTK2B_OVERFLOW_RETRY, "stream buffers kept overflowing");
    S_TRY(ctx, ctx->cand_corner.ensure(8 * (size_t)ccap));
    S_TRY(ctx, ctx->cand_chains.ensure(8 * (size_t)ccap));
    S_TRY(ctx, cudaMemsetAsync(counters, 0, sizeof(unsigned) * kNumCounters, st));
    FeatureSink sink;
    sink.key = (unsigned long long*)s->key.p + s->n;
    sink.lam = (double*)s->lam.p + 4 * (size_t)s->n;
    sink.bary4 = (float*)s->bary4.p + 4 * (size_t)s->n;
    sink.scalar = (float*)s->scalar.p + s->n;
    sink.count = counters + kCountFeatures;
    sink.cap = s->cap - s->n;
    CandidateQueue cq{};
    cq.corner = (unsigned long long*)ctx->cand_corner.p;
    cq.chains = (unsigned long long*)ctx->cand_chains.p;
    cq.count = counters + kCountCand;
    cq.cap = ccap;
    if (cfg.cull_mode == 2) {
      int mode = 0;
      S_TRY(ctx, resolve_cull_mode(ctx, rm, fa, f64, s->layout == FTK2B_LAYOUT_MULTICOMPONENT,
                                   [&](int md) -> cudaError_t {
                                     ExtractConfig c = cfg;
                                     c.cull_mode = md;
                                     cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned) * kNumCounters, st);
                                     int n = 1;
                                     if (!e)
                                       e = launch_extract_regular(f64, rm, fa, c, cq, counters + kCountErr, st,
                                                                  !ctx->disable_tma, &ctx->last_used_tma, &n);
                                     ctx->launches += (unsigned long long)n;
                                     return e;
                                   },
                                   &mode));
      cfg.cull_mode = mode;
      S_TRY(ctx, cudaMemsetAsync(counters, 0, sizeof(unsigned) * kNumCounters, st));
    }
    ctx->last_cull_mode = cfg.cull_mode;
    int nk = 1;
    S_TRY(ctx, launch_extract_regular(f64, rm, fa, cfg, cq, counters + kCountErr, st, !ctx->disable_tma,
                                      &ctx->last_used_tma, &nk));
    S_TRY(ctx, launch_refine_regular(f64, rm, fa, cfg, cq, sink, ctx->num_sms, st));
    ctx->launches += 1 + nk;
    S_TRY(ctx, cudaMemcpyAsync(ctx->h_counters, counters, sizeof(unsigned) * kNumCounters, cudaMemcpyDeviceToHost,
                               st));
    S_TRY(ctx, ctx->sync());
    const unsigned* h = ctx->h_counters;
    if (h[kCountErr] & 2u) return sfail(ctx, FTK2B_TIMEOUT, "a TMA slice copy did not complete in time");
    if (h[kCountCand] > ccap) {
      ccap = h[kCountCand] + h[kCountCand] / 4 + 1024;
      ctx->cand_cap_hint = ccap;
      continue;
    }
    if (h[kCountFeatures] > s->cap - s->n) {
      rc = ensure_stream_store(s, s->n + h[kCountFeatures] + h[kCountFeatures] / 4 + 1024);
      if (rc) return rc;
      continue;
    }
    n_new = h[kCountFeatures];
    break;
  }

  // window: spatial features of layer t-1 plus the new ones, in key order
  const unsigned first_new = s->n;
  const unsigned nS = s->n_prev + n_new;
  const unsigned wcap = nS ? nS : 1;
  S_TRY(ctx, s->s_key.ensure(8 * (size_t)wcap));
  S_TRY(ctx, s->s_key2.ensure(8 * (size_t)wcap));
  S_TRY(ctx, s->s_id.ensure(4 * (size_t)wcap));
  S_TRY(ctx, s->s_id2.ensure(4 * (size_t)wcap));
  S_TRY(ctx, s->wedges.ensure(8 * 8 * (size_t)wcap));
  S_TRY(ctx, ctx->edge_cnt.ensure(4 * (size_t)wcap));
  S_TRY(ctx, ctx->edge_slots.ensure(4 * 8 * (size_t)wcap));
  const int sgrid = ctx->sort_grid(wcap);
  S_TRY(ctx, ctx->hist.ensure(sizeof(unsigned) * 256 * (size_t)sgrid));
  const unsigned edge_room = s->n_edges + 8 * nS;
  if (edge_room > s->edge_cap) {
    unsigned nc = s->edge_cap ? s->edge_cap : 262144u;
    while (nc < edge_room) nc *= 2;
    S_TRY(ctx, grow_keep(s->edges, 8 * (size_t)s->n_edges, 8 * (size_t)nc, st));
    s->edge_cap = nc;
  }
  const int g = grid_of(wcap, 256, 4096);
  set_u32_kernel<<<1, 1, 0, st>>>(counters + kSWin, nS);
  window_build_kernel<<<g, 256, 0, st>>>((const unsigned long long*)s->key.p, (const unsigned*)s->prev_ids.p,
                                         s->n_prev, first_new, n_new, (unsigned long long*)s->s_key.p,
                                         (unsigned*)s->s_id.p);
  const unsigned long long nv_hi = (unsigned long long)rm.gstride[d - 1] * (T + 1);
  const int key_bits = bits_for(nv_hi * (unsigned long long)nch);
  const bool alt = radix_sort((unsigned long long*)s->s_key.p, (unsigned*)s->s_id.p,
                              (unsigned long long*)s->s_key2.p, (unsigned*)s->s_id2.p, counters + kSWin, wcap,
                              key_bits, (unsigned*)ctx->hist.p, sgrid, st, &ctx->launches);
  const unsigned long long* skeys = (const unsigned long long*)(alt ? s->s_key2.p : s->s_key.p);
  const unsigned* sids = (const unsigned*)(alt ? s->s_id2.p : s->s_id.p);
  S_TRY(ctx, launch_window_edges_regular(rm, nch, skeys, counters + kSWin, wcap, (unsigned*)ctx->edge_cnt.p,
                                         (unsigned*)ctx->edge_slots.p, (unsigned*)s->wedges.p,
                                         counters + kSWinEdges, 8 * wcap, st));
  if (n_new) uf_init_range_kernel<<<grid_of(n_new, 256, 4096), 256, 0, st>>>((unsigned*)s->parent.p, first_new, n_new);
  append_edges_kernel<<<grid_of(8ull * wcap, 256, 4096), 256, 0, st>>>(
      (const unsigned*)s->wedges.p, counters + kSWinEdges, 8 * wcap, sids, (unsigned*)s->parent.p,
      (unsigned*)s->edges.p, s->n_edges, s->edge_cap, counters + kCountErr);
  if (n_new)
    collect_spatial_kernel<<<grid_of(n_new, 256, 4096), 256, 0, st>>>(
        (const unsigned long long*)s->key.p, first_new, n_new, nch, time_chain_mask(d), (unsigned*)s->prev_ids2.p,
        counters + kSPrev);
  ctx->launches += 8;

  // classification while the window's values are resident: the new features,
  // and at the second push the first layer's (their coface lies in slab [0, 1])
  if (s->prm.classify) {
    S_TRY(ctx, s->tmp_simp.ensure(8 * (size_t)(M + 1) * (wcap > s->n_first ? wcap : s->n_first + 1)));
    auto classify = [&](unsigned first, unsigned cnt, unsigned* count_slot) -> cudaError_t {
      if (!cnt) return cudaSuccess;
      set_u32_kernel<<<1, 1, 0, st>>>(count_slot, cnt);
      cudaError_t e = launch_expand_regular(rm, nch, (const unsigned long long*)s->key.p + first, count_slot, cnt,
                                            nullptr, (unsigned long long*)s->tmp_simp.p, nullptr, st);
      if (e) return e;
      PostBuffers B;
      memset(&B, 0, sizeof(B));
      B.cap = cnt;
      B.count = count_slot;
      B.simplices = (unsigned long long*)s->tmp_simp.p;
      B.cls = (unsigned*)s->cls.p + first;
      ctx->launches += 3;
      return launch_classify_regular(f64, rm, fa, nch, B, st);
    };
    S_TRY(ctx, classify(first_new, n_new, counters + kCountRoots));
    if (T == 1) S_TRY(ctx, classify(0, s->n_first, counters + kCountRoots));
  }
  S_TRY(ctx, cudaMemcpyAsync(ctx->h_counters, counters, sizeof(unsigned) * kNumCounters, cudaMemcpyDeviceToHost, st));
  S_TRY(ctx, ctx->sync());
  const unsigned* h = ctx->h_counters;
  if (h[kCountErr] & 1u) return sfail(ctx, FTK2B_TIMEOUT, "union-find retry bound reached");
  s->n_edges += h[kSWinEdges];
  s->n_prev = h[kSPrev];
  std::swap(s->prev_ids, s->prev_ids2);
  s->n += n_new;
  if (T == 0) s->n_first = n_new;
  s->last_new = n_new;
  return FTK2B_OK;
}

ftk2b_status result_regular(ftk2b_stream* s, ftk2b_cp_result** out) {
  ftk2b_ctx* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  const int d = s->d, M = s->m, nch = d == 3 ? 12 : 60;
  const unsigned n = s->n, ne = s->n_edges;
  const unsigned nc = n ? n : 1, ec = ne ? ne : 1;
  S_TRY(ctx, ctx->counters.ensure(sizeof(unsigned) * kNumCounters));
  unsigned* counters = (unsigned*)ctx->counters.p;
  // canonical order of the whole store
  S_TRY(ctx, s->s_key.ensure(8 * (size_t)(nc > ec ? nc : ec)));
  S_TRY(ctx, s->s_key2.ensure(8 * (size_t)(nc > ec ? nc : ec)));
  S_TRY(ctx, s->s_id.ensure(4 * (size_t)(nc > ec ? nc : ec)));
  S_TRY(ctx, s->s_id2.ensure(4 * (size_t)(nc > ec ? nc : ec)));
  S_TRY(ctx, ctx->perm0.ensure(4 * (size_t)nc));  // inverse permutation
  S_TRY(ctx, ctx->perm1.ensure(4 * (size_t)nc));  // roots
  S_TRY(ctx, ctx->parent.ensure(4 * (size_t)nc)); // component minimum
  S_TRY(ctx, ctx->lam_s.ensure(32 * (size_t)nc));
  S_TRY(ctx, ctx->bary4_s.ensure(16 * (size_t)nc));
  S_TRY(ctx, ctx->scalar_s.ensure(4 * (size_t)nc));
  S_TRY(ctx, ctx->cls.ensure(4 * (size_t)nc));
  S_TRY(ctx, ctx->track.ensure(8 * (size_t)nc));
  S_TRY(ctx, ctx->simplices.ensure(8 * (size_t)(M + 1) * nc));
  S_TRY(ctx, ctx->bary.ensure(4 * (size_t)(M + 1) * nc));
  S_TRY(ctx, ctx->edges.ensure(8 * (size_t)ec));
  const int sgrid = ctx->sort_grid(nc > ec ? nc : ec);
  S_TRY(ctx, ctx->hist.ensure(sizeof(unsigned) * 256 * (size_t)sgrid));
  const int g = grid_of(nc > ec ? nc : ec, 256, 4096);
  S_TRY(ctx, cudaMemsetAsync(counters, 0, sizeof(unsigned) * kNumCounters, st));
  set_u32_kernel<<<1, 1, 0, st>>>(counters + kSWin, n);
  set_u32_kernel<<<1, 1, 0, st>>>(counters + kSWinEdges, ne);
  if (n) S_TRY(ctx, cudaMemcpyAsync(s->s_key.p, s->key.p, 8 * (size_t)n, cudaMemcpyDeviceToDevice, st));
  iota_u32_kernel<<<g, 256, 0, st>>>((unsigned*)s->s_id.p, n);
  const RegularMesh full = window_mesh(s, 0, s->T);
  const unsigned long long nv_hi = (unsigned long long)full.gstride[d - 1] * (s->T + 1);
  const bool alt = radix_sort((unsigned long long*)s->s_key.p, (unsigned*)s->s_id.p, (unsigned long long*)s->s_key2.p,
                              (unsigned*)s->s_id2.p, counters + kSWin, nc, bits_for(nv_hi * (unsigned long long)nch),
                              (unsigned*)ctx->hist.p, sgrid, st, &ctx->launches);
  const unsigned long long* skeys = (const unsigned long long*)(alt ? s->s_key2.p : s->s_key.p);
  const unsigned* perm = (const unsigned*)(alt ? s->s_id2.p : s->s_id.p);
  unsigned* inv = (unsigned*)ctx->perm0.p;
  unsigned* root = (unsigned*)ctx->perm1.p;
  unsigned* cmin = (unsigned*)ctx->parent.p;
  invert_kernel<<<g, 256, 0, st>>>(perm, n, inv);
  fill_u32_kernel<<<g, 256, 0, st>>>(cmin, n, 0xFFFFFFFFu);
  comp_min_kernel<<<g, 256, 0, st>>>((unsigned*)s->parent.p, inv, n, root, cmin, counters + kCountRoots);
  gather_result_kernel<<<g, 256, 0, st>>>(perm, n, root, cmin, (const double*)s->lam.p, (const float*)s->bary4.p,
                                          (const float*)s->scalar.p, (const unsigned*)s->cls.p,
                                          (double*)ctx->lam_s.p, (float*)ctx->bary4_s.p, (float*)ctx->scalar_s.p,
                                          (unsigned*)ctx->cls.p, (unsigned long long*)ctx->track.p);
  S_TRY(ctx, launch_expand_regular(full, nch, skeys, counters + kSWin, nc, (const float*)ctx->bary4_s.p,
                                   (unsigned long long*)ctx->simplices.p, (float*)ctx->bary.p, st));
  // edges in canonical ids, sorted (each pair spans one top cell: no duplicates)
  unsigned long long* ek = (unsigned long long*)s->s_key.p;  // free again after the gathers
  canon_edges_kernel<<<g, 256, 0, st>>>((const unsigned*)s->edges.p, ne, inv, ek);
  const bool ealt = radix_sort(ek, (unsigned*)s->s_id.p, (unsigned long long*)s->s_key2.p, (unsigned*)s->s_id2.p,
                               counters + kSWinEdges, ec, 2 * 32, (unsigned*)ctx->hist.p, sgrid, st, &ctx->launches);
  unpack_edges_kernel<<<g, 256, 0, st>>>(ealt ? (const unsigned long long*)s->s_key2.p : ek, ne,
                                         (unsigned*)ctx->edges.p);
  ctx->launches += 7;
  S_TRY(ctx, cudaMemcpyAsync(ctx->h_counters, counters, sizeof(unsigned) * kNumCounters, cudaMemcpyDeviceToHost, st));
  S_TRY(ctx, ctx->sync());
  // hand the canonical buffers to the context's fetch
  ctx->last.kind = FTK2B_MESH_REGULAR;
  ctx->last.m = M;
  ctx->last.f64 = s->dtype == FTK2B_F64;
  ctx->last.n = n;
  ctx->last.ne = s->prm.want_edges ? ne : 0;
  ctx->last.n_roots = ctx->h_counters[kCountRoots];
  ftk2b_mesh_desc md;
  memset(&md, 0, sizeof(md));
  md.kind = FTK2B_MESH_REGULAR;
  md.ndims = d;
  for (int k = 0; k < d - 1; ++k) md.local_dims[k] = s->ld[k];
  md.local_dims[d - 1] = s->T;
  ctx->last.n_simplices = ftk2b_mesh_simplex_count(&md, M);
  ctx->last.device_ms = 0;
  ctx->last.classify = s->prm.classify;
  ctx->last.want_edges = s->prm.want_edges;
  return ftk2b_cp_fetch(ctx, out);
}

}  // namespace

namespace ftk2b {

cudaError_t grow_keep(DevBuf& b, size_t used, size_t want, cudaStream_t st) {
  if (b.p && b.bytes >= want) return cudaSuccess;
  // stream-ordered: allocate, copy and free the old block after the work
  // already queued on the stream, without synchronising the device
  void* p = nullptr;
  const size_t n = want < 256 ? 256 : want;
  cudaError_t e = cudaMallocAsync(&p, n, st);
  if (e) {
    cudaGetLastError();
    return e;
  }
  if (b.p && used) {
    e = cudaMemcpyAsync(p, b.p, used, cudaMemcpyDeviceToDevice, st);
    if (e) {
      cudaFreeAsync(p, st);
      return e;
    }
  }
  if (b.p) cudaFreeAsync(b.p, st);
  b.p = p;
  b.bytes = n;
  b.st = st;
  ++b.generation;
  return cudaSuccess;
}

ftk2b_status ensure_stream_store(ftk2b_stream* s, unsigned want) {
  ftk2b_ctx* ctx = s->ctx;
  if (want <= s->cap) return FTK2B_OK;
  unsigned nc = s->cap ? s->cap : 262144u;
  while (nc < want) nc = nc * 2u > nc ? nc * 2u : 0xFFFFFFF0u;
  cudaStream_t st = ctx->stream;
  const size_t n = s->n;
  if (s->kind == FTK2B_MESH_REGULAR) {
    S_TRY(ctx, grow_keep(s->key, 8 * n, 8 * (size_t)nc, st));
  } else {
    S_TRY(ctx, grow_keep(s->hi, 8 * n, 8 * (size_t)nc, st));
    S_TRY(ctx, grow_keep(s->lo, 8 * n, 8 * (size_t)nc, st));
    S_TRY(ctx, grow_keep(s->phase, 4 * n, 4 * (size_t)nc, st));
  }
  S_TRY(ctx, grow_keep(s->lam, 32 * n, 32 * (size_t)nc, st));
  S_TRY(ctx, grow_keep(s->bary4, 16 * n, 16 * (size_t)nc, st));
  S_TRY(ctx, grow_keep(s->scalar, 4 * n, 4 * (size_t)nc, st));
  S_TRY(ctx, grow_keep(s->cls, 4 * n, 4 * (size_t)nc, st));
  S_TRY(ctx, grow_keep(s->parent, 4 * n, 4 * (size_t)nc, st));
  S_TRY(ctx, grow_keep(s->prev_ids, 4 * (size_t)s->n_prev, 4 * (size_t)nc, st));
  S_TRY(ctx, s->prev_ids2.ensure(4 * (size_t)nc));
  s->cap = nc;
  return FTK2B_OK;
}

}  // namespace ftk2b

// ---------------------------------------------------------------------------
// C ABI

extern "C" ftk2b_status ftk2b_stream_open(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* tmpl,
                                          const ftk2b_cp_params* params, ftk2b_stream** out) {
  if (!ctx || !out) return FTK2B_INVALID_ARG;
  *out = nullptr;
  if (!mesh || !tmpl) return sfail(ctx, FTK2B_INVALID_ARG, "null descriptor");
  ftk2b_cp_params prm = params ? *params : ftk2b_cp_params_default();
  if (!(prm.sos_q > 0)) return sfail(ctx, FTK2B_INVALID_ARG, "sos_q must be positive");
  if (tmpl->dtype != FTK2B_F32 && tmpl->dtype != FTK2B_F64)
    return sfail(ctx, FTK2B_INVALID_ARG, "dtype must be FTK2B_F32 or FTK2B_F64");
  if (tmpl->scalar) return sfail(ctx, FTK2B_UNSUPPORTED, "streams do not interpolate a scalar");
  ftk2b_stream* s = new ftk2b_stream();
  s->ctx = ctx;
  s->kind = mesh->kind;
  s->prm = prm;
  s->dtype = tmpl->dtype;
  s->layout = tmpl->layout;
  s->ncomp = tmpl->ncomp;
  s->location = tmpl->location;
  s->es = tmpl->dtype == FTK2B_F64 ? 8 : 4;
  if (mesh->kind == FTK2B_MESH_REGULAR) {
    const int d = mesh->ndims;
    if (d != 3 && d != 4) {
      delete s;
      return sfail(ctx, FTK2B_UNSUPPORTED, "regular streams need 3 or 4 dims including time");
    }
    s->d = d;
    s->m = d - 1;
    if (tmpl->ncomp != s->m) {
      delete s;
      return sfail(ctx, FTK2B_INVALID_ARG, "a %dD spacetime mesh needs %d components", d, d - 1);
    }
    if (tmpl->layout != FTK2B_LAYOUT_MULTICOMPONENT && tmpl->layout != FTK2B_LAYOUT_SEPARATE) {
      delete s;
      return sfail(ctx, FTK2B_UNSUPPORTED, "regular streams take multicomponent or separate arrays");
    }
    if (tmpl->nd != d - 1) {
      delete s;
      return sfail(ctx, FTK2B_INVALID_ARG, "a timestep has %d spatial dims", d - 1);
    }
    s->slice_elems = 1;
    for (int k = 0; k < d - 1; ++k) {
      s->ld[k] = mesh->local_dims[k];
      s->off[k] = mesh->offset[k];
      s->gd[k] = mesh->global_dims[k];
      s->adims[k] = tmpl->dims[k];
      const uint64_t need = tmpl->layout == FTK2B_LAYOUT_SEPARATE ? s->ld[k] : s->off[k] + s->ld[k];
      if (s->ld[k] < 1 || s->off[k] + s->ld[k] > s->gd[k] || s->adims[k] < need || s->ld[k] >= 65536) {
        delete s;
        return sfail(ctx, FTK2B_INVALID_ARG, "inconsistent stream mesh / array dims along axis %d", k);
      }
      s->slice_elems *= s->adims[k];
    }
    if (tmpl->layout == FTK2B_LAYOUT_MULTICOMPONENT) s->slice_elems *= s->m;
  } else if (mesh->kind == FTK2B_MESH_EXTRUDED) {
    const int cd = mesh->base_cell_dim;
    if ((cd != 2 && cd != 3) || tmpl->ncomp != cd || !mesh->base_cells || !mesh->n_base_cells) {
      delete s;
      return sfail(ctx, FTK2B_INVALID_ARG, "extruded streams need triangle or tet cells and ncomp = cell dim");
    }
    if (tmpl->layout == FTK2B_LAYOUT_MULTICOMPONENT) {
      delete s;
      return sfail(ctx, FTK2B_UNSUPPORTED, "extruded streams take per-vertex arrays");
    }
    s->d = cd + 1;
    s->m = cd;
    s->emesh = *mesh;
    s->ecells.assign(mesh->base_cells, mesh->base_cells + mesh->n_base_cells * (cd + 1));
    s->emesh.base_cells = s->ecells.data();
    s->ebase_hash = ftk2b::hash_base_cells(s->ecells.data(), (uint64_t)s->ecells.size());
    s->slice_elems = mesh->n_base_verts;
  } else {
    delete s;
    return sfail(ctx, FTK2B_INVALID_ARG, "unknown mesh kind %d", mesh->kind);
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    delete s;
    return sfail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  }
  for (DevBuf* b : {&s->ring[0], &s->ring[1], &s->ring[2], &s->key, &s->hi, &s->lo, &s->phase, &s->lam,
                    &s->bary4, &s->scalar, &s->cls, &s->parent, &s->edges, &s->prev_ids, &s->prev_ids2, &s->s_key,
                    &s->s_key2, &s->s_id, &s->s_id2, &s->s_hi, &s->s_lo, &s->s_phase, &s->wedges, &s->tmp_simp,
                    &s->dummy})
    b->st = ctx->stream;
  const int narr = s->layout == FTK2B_LAYOUT_MULTICOMPONENT ? 1 : s->m;
  for (int j = 0; j < narr; ++j)
    if (s->ring[j].ensure(2 * s->slice_elems * s->es) != cudaSuccess) {
      for (auto& b : s->ring) b.release();
      delete s;
      return sfail(ctx, FTK2B_OOM, "stream ring allocation failed");
    }
  *out = s;
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_stream_push(ftk2b_stream* s, const ftk2b_field_desc* step, uint64_t* n_new) {
  ftk2b::NvtxRange nvtx_range("ftk2b_stream_push");
  if (!s) return FTK2B_INVALID_ARG;
  ftk2b_ctx* ctx = s->ctx;
  if (!step) return sfail(ctx, FTK2B_INVALID_ARG, "null timestep");
  if (step->dtype != s->dtype || step->ncomp != s->ncomp || step->layout != s->layout)
    return sfail(ctx, FTK2B_INVALID_ARG, "timestep dtype / ncomp / layout differ from the stream's");
  if (s->kind == FTK2B_MESH_REGULAR) {
    if (step->nd != s->d - 1) return sfail(ctx, FTK2B_INVALID_ARG, "a timestep has %d spatial dims", s->d - 1);
    for (int k = 0; k < s->d - 1; ++k)
      if (step->dims[k] != s->adims[k]) return sfail(ctx, FTK2B_INVALID_ARG, "timestep dims differ along axis %d", k);
  } else {
    if (step->dims[0] < s->emesh.n_base_verts)
      return sfail(ctx, FTK2B_INVALID_ARG, "per-vertex timestep shorter than the base vertex count");
  }
  if (s->T + 2 >= (1ull << 30)) return sfail(ctx, FTK2B_UNSUPPORTED, "a stream holds fewer than 2^30 timesteps");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return sfail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  cudaStream_t st = ctx->stream;
  S_TRY(ctx, cudaEventRecord(ctx->ev0, st));
  const int narr = s->layout == FTK2B_LAYOUT_MULTICOMPONENT ? 1 : s->m;
  const size_t bytes = s->slice_elems * s->es;
  const size_t slot = (size_t)(s->T & 1);
  for (int j = 0; j < narr; ++j) {
    if (!step->comp[j]) return sfail(ctx, FTK2B_INVALID_ARG, "component array %d is null", j);
    S_TRY(ctx, cudaMemcpyAsync((char*)s->ring[j].p + slot * bytes, step->comp[j], bytes,
                               step->location == FTK2B_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                               st));
  }
  ftk2b_status rc = s->kind == FTK2B_MESH_REGULAR ? push_regular(s) : stream_push_extruded(s);
  if (rc) return rc;
  S_TRY(ctx, cudaEventRecord(ctx->ev1, st));
  S_TRY(ctx, ctx->sync());
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) != cudaSuccess) ms = 0.f;
  cudaGetLastError();
  s->last_ms = ms;
  s->T += 1;
  if (n_new) *n_new = s->last_new;
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_stream_result(ftk2b_stream* s, ftk2b_cp_result** out) {
  ftk2b::NvtxRange nvtx_range("ftk2b_stream_result");
  if (!s || !out) return FTK2B_INVALID_ARG;
  *out = nullptr;
  if (cudaSetDevice(s->ctx->device) != cudaSuccess) return sfail(s->ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  return s->kind == FTK2B_MESH_REGULAR ? result_regular(s, out) : stream_result_extruded(s, out);
}

extern "C" ftk2b_status ftk2b_stream_info(ftk2b_stream* s, uint64_t* timesteps, uint64_t* n_features,
                                          double* last_push_ms) {
  if (!s) return FTK2B_INVALID_ARG;
  if (timesteps) *timesteps = s->T;
  if (n_features) *n_features = s->n;
  if (last_push_ms) *last_push_ms = s->last_ms;
  return FTK2B_OK;
}

extern "C" void ftk2b_stream_close(ftk2b_stream* s) {
  if (!s) return;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  for (DevBuf* b : {&s->ring[0], &s->ring[1], &s->ring[2], &s->key, &s->hi, &s->lo, &s->phase, &s->lam, &s->bary4,
                    &s->scalar, &s->cls, &s->parent, &s->edges, &s->prev_ids, &s->prev_ids2, &s->s_key, &s->s_key2,
                    &s->s_id, &s->s_id2, &s->s_hi, &s->s_lo, &s->s_phase, &s->wedges, &s->tmp_simp, &s->dummy})
    b->release();
  delete s;
}

// ---------------------------------------------------------------------------
// Checkpoint / resume: everything a later push or result reads -- the
// configuration, the ring's timesteps, the feature store, the star edges,
// the union-find parents and the newest layer's ids -- as one host blob.
// Per-push scratch and the context's caches are rebuilt on demand.

namespace {

constexpr char kCkptMagic[8] = {'F', 'T', 'K', '2', 'B', 'S', 'T', 'R'};
constexpr uint32_t kCkptVersion = 1;

struct StreamCkpt {
  char magic[8];
  uint32_t version, header_bytes;
  int32_t kind, d, m, dtype, layout, ncomp, location, pad;
  uint64_t es;
  ftk2b_cp_params prm;
  uint64_t ld[3], off[3], gd[3], adims[3];
  ftk2b_mesh_desc emesh;  // base_cells stored as null; the cells follow the header
  uint64_t n_ecells, ebase_hash;
  uint64_t T, slice_elems;
  uint32_t n, n_edges, n_prev, n_first;
};

// the device sections of a stream's state, in blob order
std::vector<std::pair<ftk2b::DevBuf*, size_t>> ckpt_sections(ftk2b_stream* s) {
  std::vector<std::pair<ftk2b::DevBuf*, size_t>> v;
  const int narr = s->layout == FTK2B_LAYOUT_MULTICOMPONENT ? 1 : s->m;
  for (int j = 0; j < narr; ++j) v.push_back({&s->ring[j], 2 * s->slice_elems * s->es});
  const size_t n = s->n;
  if (s->kind == FTK2B_MESH_REGULAR) {
    v.push_back({&s->key, 8 * n});
  } else {
    v.push_back({&s->hi, 8 * n});
    v.push_back({&s->lo, 8 * n});
    v.push_back({&s->phase, 4 * n});
  }
  v.push_back({&s->lam, 32 * n});
  v.push_back({&s->bary4, 16 * n});
  v.push_back({&s->scalar, 4 * n});
  v.push_back({&s->cls, 4 * n});
  v.push_back({&s->parent, 4 * n});
  v.push_back({&s->edges, 8 * (size_t)s->n_edges});
  v.push_back({&s->prev_ids, 4 * (size_t)s->n_prev});
  return v;
}

}  // namespace

extern "C" ftk2b_status ftk2b_stream_checkpoint(ftk2b_stream* s, void* buf, uint64_t* bytes) {
  ftk2b::NvtxRange nvtx_range("ftk2b_stream_checkpoint");
  if (!s || !bytes) return FTK2B_INVALID_ARG;
  ftk2b_ctx* ctx = s->ctx;
  const auto sec = ckpt_sections(s);
  uint64_t total = sizeof(StreamCkpt) + 8 * (uint64_t)s->ecells.size();
  for (const auto& x : sec) total += x.second;
  if (!buf) {
    *bytes = total;
    return FTK2B_OK;
  }
  if (*bytes < total) {
    *bytes = total;
    return sfail(ctx, FTK2B_INVALID_ARG, "checkpoint buffer too small (%llu bytes needed)",
                 (unsigned long long)total);
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) return sfail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  StreamCkpt h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, kCkptMagic, 8);
  h.version = kCkptVersion;
  h.header_bytes = (uint32_t)sizeof(StreamCkpt);
  h.kind = s->kind;
  h.d = s->d;
  h.m = s->m;
  h.dtype = s->dtype;
  h.layout = s->layout;
  h.ncomp = s->ncomp;
  h.location = s->location;
  h.es = s->es;
  h.prm = s->prm;
  for (int k = 0; k < 3; ++k) {
    h.ld[k] = s->ld[k];
    h.off[k] = s->off[k];
    h.gd[k] = s->gd[k];
    h.adims[k] = s->adims[k];
  }
  h.emesh = s->emesh;
  h.emesh.base_cells = nullptr;
  h.n_ecells = s->ecells.size();
  h.ebase_hash = s->ebase_hash;
  h.T = s->T;
  h.slice_elems = s->slice_elems;
  h.n = s->n;
  h.n_edges = s->n_edges;
  h.n_prev = s->n_prev;
  h.n_first = s->n_first;
  char* p = static_cast<char*>(buf);
  memcpy(p, &h, sizeof(h));
  p += sizeof(h);
  if (!s->ecells.empty()) memcpy(p, s->ecells.data(), 8 * s->ecells.size());
  p += 8 * s->ecells.size();
  for (const auto& x : sec) {
    if (x.second) S_TRY(ctx, cudaMemcpyAsync(p, x.first->p, x.second, cudaMemcpyDeviceToHost, ctx->stream));
    p += x.second;
  }
  S_TRY(ctx, ctx->sync());
  *bytes = total;
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_stream_restore(ftk2b_ctx* ctx, const void* buf, uint64_t bytes, ftk2b_stream** out) {
  ftk2b::NvtxRange nvtx_range("ftk2b_stream_restore");
  if (!ctx || !out) return FTK2B_INVALID_ARG;
  *out = nullptr;
  if (!buf || bytes < sizeof(StreamCkpt)) return sfail(ctx, FTK2B_INVALID_ARG, "not a stream checkpoint (too short)");
  StreamCkpt h;
  memcpy(&h, buf, sizeof(h));
  if (memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != kCkptVersion || h.header_bytes != sizeof(StreamCkpt))
    return sfail(ctx, FTK2B_INVALID_ARG, "not a stream checkpoint of this library version");
  // the configuration must be one that ftk2b_stream_open accepts
  const bool regular = h.kind == FTK2B_MESH_REGULAR;
  bool ok = (regular || h.kind == FTK2B_MESH_EXTRUDED) && (h.d == 3 || h.d == 4) && h.m == h.d - 1 &&
            h.ncomp == h.m && (h.dtype == FTK2B_F32 || h.dtype == FTK2B_F64) &&
            h.es == (h.dtype == FTK2B_F64 ? 8u : 4u) && (h.location == FTK2B_HOST || h.location == FTK2B_DEVICE) &&
            h.prm.sos_q > 0 && h.T < (1ull << 30);
  if (ok && regular) {
    ok = (h.layout == FTK2B_LAYOUT_MULTICOMPONENT || h.layout == FTK2B_LAYOUT_SEPARATE) && h.n_ecells == 0;
    uint64_t se = 1;
    for (int k = 0; k < h.d - 1 && ok; ++k) {
      const uint64_t need = h.layout == FTK2B_LAYOUT_SEPARATE ? h.ld[k] : h.off[k] + h.ld[k];
      ok = h.ld[k] >= 1 && h.ld[k] < 65536 && h.off[k] + h.ld[k] <= h.gd[k] && h.adims[k] >= need &&
           h.adims[k] < (1ull << 32);
      se *= h.adims[k];
    }
    if (h.layout == FTK2B_LAYOUT_MULTICOMPONENT) se *= (uint64_t)h.m;
    ok = ok && se == h.slice_elems;
  } else if (ok) {
    const int cd = h.emesh.base_cell_dim;
    ok = cd == h.m && h.layout != FTK2B_LAYOUT_MULTICOMPONENT && h.emesh.n_base_cells > 0 &&
         h.emesh.n_base_cells < (1ull << 40) && h.n_ecells == h.emesh.n_base_cells * (uint64_t)(cd + 1) &&
         h.slice_elems == h.emesh.n_base_verts && h.slice_elems > 0;
  }
  if (!ok) return sfail(ctx, FTK2B_INVALID_ARG, "stream checkpoint holds an invalid configuration");

  ftk2b_stream* s = new ftk2b_stream();
  s->ctx = ctx;
  s->kind = h.kind;
  s->d = h.d;
  s->m = h.m;
  s->prm = h.prm;
  s->dtype = h.dtype;
  s->layout = h.layout;
  s->ncomp = h.ncomp;
  s->location = h.location;
  s->es = h.es;
  for (int k = 0; k < 3; ++k) {
    s->ld[k] = h.ld[k];
    s->off[k] = h.off[k];
    s->gd[k] = h.gd[k];
    s->adims[k] = h.adims[k];
  }
  s->slice_elems = h.slice_elems;
  s->T = h.T;
  const char* p = static_cast<const char*>(buf) + sizeof(h);
  // the blob's size must be exactly what its counts say
  s->n = h.n;
  s->n_edges = h.n_edges;
  s->n_prev = h.n_prev;
  uint64_t total = sizeof(h) + 8 * h.n_ecells;
  for (const auto& x : ckpt_sections(s)) total += x.second;
  if (total != bytes || h.n_prev > h.n || (h.n && h.n_first > h.n)) {
    delete s;
    return sfail(ctx, FTK2B_INVALID_ARG, "stream checkpoint size does not match its contents");
  }
  if (!regular) {
    s->emesh = h.emesh;
    s->ecells.resize(h.n_ecells);  // the caller's blob need not be 8-byte aligned
    memcpy(s->ecells.data(), p, 8 * h.n_ecells);
    s->emesh.base_cells = s->ecells.data();
    s->ebase_hash = ftk2b::hash_base_cells(s->ecells.data(), (uint64_t)s->ecells.size());
    if (s->ebase_hash != h.ebase_hash) {
      delete s;
      return sfail(ctx, FTK2B_INVALID_ARG, "stream checkpoint's base cells are damaged");
    }
  }
  p += 8 * h.n_ecells;
  auto release_all = [&]() {
    for (DevBuf* b : {&s->ring[0], &s->ring[1], &s->ring[2], &s->key, &s->hi, &s->lo, &s->phase, &s->lam, &s->bary4,
                      &s->scalar, &s->cls, &s->parent, &s->edges, &s->prev_ids, &s->prev_ids2})
      b->release();
  };
  ftk2b_status st = FTK2B_OK;
  if (cudaSetDevice(ctx->device) != cudaSuccess) st = FTK2B_CUDA_ERROR;
  for (DevBuf* b : {&s->ring[0], &s->ring[1], &s->ring[2], &s->key, &s->hi, &s->lo, &s->phase, &s->lam,
                    &s->bary4, &s->scalar, &s->cls, &s->parent, &s->edges, &s->prev_ids, &s->prev_ids2, &s->s_key,
                    &s->s_key2, &s->s_id, &s->s_id2, &s->s_hi, &s->s_lo, &s->s_phase, &s->wedges, &s->tmp_simp,
                    &s->dummy})
    b->st = ctx->stream;
  const int narr = s->layout == FTK2B_LAYOUT_MULTICOMPONENT ? 1 : s->m;
  for (int j = 0; j < narr && !st; ++j)
    if (s->ring[j].ensure(2 * s->slice_elems * s->es) != cudaSuccess) st = FTK2B_OOM;
  // an empty store grows to hold the checkpoint's features (nothing to keep)
  if (!st) {
    s->n = 0;
    s->n_prev = 0;
    st = ftk2b::ensure_stream_store(s, h.n > 0 ? h.n : 1);
    s->n = h.n;
    s->n_prev = h.n_prev;
  }
  if (!st && h.n_edges) {
    unsigned nc = 262144u;
    while (nc < h.n_edges) nc = nc * 2u > nc ? nc * 2u : 0xFFFFFFF0u;
    if (s->edges.ensure(8 * (size_t)nc) != cudaSuccess) st = FTK2B_OOM;
    else s->edge_cap = nc;
  }
  if (!st) {
    s->n_edges = h.n_edges;
    s->n_first = h.n_first;
    for (const auto& x : ckpt_sections(s)) {
      if (x.second &&
          cudaMemcpyAsync(x.first->p, p, x.second, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
        st = FTK2B_CUDA_ERROR;
        break;
      }
      p += x.second;
    }
  }
  if (!st && ctx->sync() != cudaSuccess) st = FTK2B_CUDA_ERROR;
  if (st) {
    cudaGetLastError();
    cudaStreamSynchronize(ctx->stream);
    release_all();
    delete s;
    return sfail(ctx, st, "stream restore failed (device allocation or copy)");
  }
  *out = s;
  return FTK2B_OK;
}
