// Batched extraction: many independent regular-mesh fields in one pass.
//
// The fields' canonical keys are laid end to end (field f's keys start at
// kb[f] = sum over earlier fields of vertices x chains), so one sort puts the
// batch in (field, Simplex order) order, star-edge searches stay inside a
// field's key range, and union-find components never cross fields.  Every
// per-field computation runs the single-field device code with that field's
// record, so field f's features, edges and track ids are those of
// ftk2b_cp_extract on field f alone (track ids and edge endpoints are rebased
// to the field's first feature when the results are split).

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/ftk2b.h"
#include "cp_api_internal.h"
#include "cp_batch.h"
#include "cp_post.h"

using namespace ftk2b;

namespace {

ftk2b_status bfail(ftk2b_ctx* ctx, ftk2b_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return st;
}

#define B_TRY(ctx, call)                                                                        \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return bfail(ctx, e_ == cudaErrorMemoryAllocation ? FTK2B_OOM : FTK2B_CUDA_ERROR,          \
                   "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

int bits_for(unsigned long long v) {
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b < 1 ? 1 : b;
}

// grow-only pinned host buffer (contents not kept)
cudaError_t ensure_pinned(void** p, size_t* have, size_t want) {
  if (*have >= want && *p) return cudaSuccess;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *have = 0;
  const size_t sz = want + want / 2 + 4096;
  cudaError_t e = cudaMallocHost(p, sz);
  if (!e) *have = sz;
  return e;
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

ftk2b_status run_batch(ftk2b_ctx* ctx, uint32_t n, const ftk2b_mesh_desc* meshes, const ftk2b_field_desc* fields,
                       const ftk2b_cp_params* params) {
  BatchCtx& bc = ctx->batch;
  if (n == 0) return bfail(ctx, FTK2B_INVALID_ARG, "empty batch");
  if (!meshes || !fields) return bfail(ctx, FTK2B_INVALID_ARG, "null descriptor array");
  const int f64 = fields[0].dtype == FTK2B_F64;
  const int multi = fields[0].layout == FTK2B_LAYOUT_MULTICOMPONENT ? 1 : 0;
  std::vector<RegularMesh> rms(n);
  std::vector<ftk2b_cp_params> prm(n);
  for (uint32_t i = 0; i < n; ++i) {
    prm[i] = params ? params[i] : ftk2b_cp_params_default();
    if (!(prm[i].sos_q > 0)) return bfail(ctx, FTK2B_INVALID_ARG, "field %u: sos_q must be positive", i);
    if (prm[i].classify) return bfail(ctx, FTK2B_UNSUPPORTED, "field %u: classification is not batched", i);
    if (meshes[i].kind != FTK2B_MESH_REGULAR)
      return bfail(ctx, FTK2B_UNSUPPORTED, "field %u: batches take regular meshes", i);
    if (fields[i].dtype != fields[0].dtype) return bfail(ctx, FTK2B_INVALID_ARG, "field %u: mixed dtypes", i);
    if ((fields[i].layout == FTK2B_LAYOUT_MULTICOMPONENT ? 1 : 0) != multi)
      return bfail(ctx, FTK2B_INVALID_ARG, "field %u: multicomponent and separate layouts mixed", i);
    ftk2b_status st = build_regular(ctx, &meshes[i], rms[i]);
    if (st) return st;
    if (fields[i].ncomp != rms[i].d - 1)
      return bfail(ctx, FTK2B_INVALID_ARG, "field %u: a %dD spacetime mesh needs %d components", i, rms[i].d,
                   rms[i].d - 1);
  }

  // field access; host arrays staged into one buffer (a counting pass first)
  std::vector<FieldAccess> fas(n);
  auto prepare_all = [&](StageArena* ar) -> ftk2b_status {
    for (uint32_t i = 0; i < n; ++i) {
      const RegularMesh& rm = rms[i];
      uint64_t ghi[4], lhi[4], nv = 1;
      for (int k = 0; k < rm.d; ++k) {
        ghi[k] = meshes[i].offset[k] + meshes[i].local_dims[k];
        lhi[k] = meshes[i].local_dims[k];
        nv *= meshes[i].global_dims[k];
      }
      ftk2b_status st = prepare_field(ctx, &fields[i], rm.d, ghi, lhi, nv, fas[i], ar);
      if (st) return st;
      for (int k = 0; k < rm.d; ++k) fas[i].shift[k] = (fields[i].layout == FTK2B_LAYOUT_SEPARATE) ? rm.off[k] : 0;
    }
    return FTK2B_OK;
  };
  StageArena count{nullptr, 0};
  ftk2b_status st = prepare_all(&count);
  if (st) return st;
  B_TRY(ctx, bc.stage.ensure(count.off ? count.off : 256));
  StageArena arena{static_cast<unsigned char*>(bc.stage.p), 0};
  st = prepare_all(&arena);
  if (st) return st;

  // per-field records and key bases
  std::vector<BatchField> hf(n);
  std::vector<BatchMesh> hm(n);
  std::vector<unsigned long long> hkb(n + 1);
  bc.info.assign(n, BatchFieldInfo{});
  unsigned long long kb = 0;
  uint64_t sig = 1469598103934665603ull;  // FNV-1a over the batch's shape
  auto mix = [&](const void* p, size_t bytes) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t b = 0; b < bytes; ++b) sig = (sig ^ c[b]) * 1099511628211ull;
  };
  for (uint32_t i = 0; i < n; ++i) {
    const RegularMesh& rm = rms[i];
    const int d = rm.d, nch = d == 3 ? 12 : 60;
    BatchField& F = hf[i];
    memset(&F, 0, sizeof(F));
    F.mesh = rm;
    F.fa = fas[i];
    ExtractConfig& cfg = F.cfg;
    cfg.Q = prm[i].sos_q;
    cfg.refined = prm[i].precision == FTK2B_PRECISION_REFINED;
    cfg.cull_mode = 0;
    int TX, TY, TZ;
    regular_tile(d, &TX, &TY, &TZ);
    cfg.tiles[0] = (int)((rm.ld[0] + TX - 1) / TX);
    cfg.tiles[1] = (int)((rm.ld[1] + TY - 1) / TY);
    cfg.tiles[2] = (d == 4) ? (int)((rm.ld[2] + TZ - 1) / TZ) : 1;
    F.tma = regular_tma_maps(f64, rm, F.fa, !ctx->disable_tma, F.maps) ? 1 : 0;
    F.key_base = kb;
    hkb[i] = kb;
    unsigned long long nvg = 1;
    for (int k = 0; k < d; ++k) nvg *= (unsigned long long)rm.gd[k];
    if (nvg > (~0ull - kb) / (unsigned long long)nch)
      return bfail(ctx, FTK2B_UNSUPPORTED, "the batch's key space exceeds 64 bits");
    kb += nvg * (unsigned long long)nch;
    hm[i].mesh = rm;
    hm[i].nch = nch;
    bc.info[i].m = d - 1;
    bc.info[i].want_edges = prm[i].want_edges;
    bc.info[i].nsimp = ftk2b_mesh_simplex_count(&meshes[i], d - 1);
    mix(&rm, sizeof(rm));
    mix(F.fa.adims, sizeof(F.fa.adims));
    mix(F.fa.estride, sizeof(F.fa.estride));
    mix(&F.fa.per_vertex, sizeof(int));
    mix(&F.tma, sizeof(int));
  }
  hkb[n] = kb;
  const int key_bits = bits_for(kb);
  mix(&f64, sizeof(f64));
  mix(&multi, sizeof(multi));

  // cull items: (tile, time chunk) of every field, for a time-chunk choice
  // (steps per item; 0xFFFF = the whole time range)
  auto assign_items = [&](int pick) -> unsigned long long {
    unsigned long long items = 0;
    for (uint32_t i = 0; i < n; ++i) {
      ExtractConfig& cfg = hf[i].cfg;
      const long long lt = rms[i].ld[rms[i].d - 1];
      cfg.tchunk = batch_time_chunk(lt, pick);
      hf[i].item_base = (unsigned)items;
      items += (unsigned long long)cfg.tiles[0] * cfg.tiles[1] * cfg.tiles[2] *
               (unsigned long long)((lt + cfg.tchunk - 1) / cfg.tchunk);
      if (items >= 0xFFFFFFF0ull) return ~0ull;
    }
    return items;
  };

  // tables to the device through pinned staging
  const size_t o_f = 0, o_m = align_up(sizeof(BatchField) * n, 256);
  const size_t o_k = o_m + align_up(sizeof(BatchMesh) * n, 256);
  const size_t o_i = o_k + align_up(sizeof(unsigned long long) * (n + 1), 256);
  const size_t tab_bytes = o_i + sizeof(unsigned) * n;
  B_TRY(ctx, ensure_pinned(&bc.h_tab, &bc.h_tab_bytes, tab_bytes));
  unsigned char* ht = static_cast<unsigned char*>(bc.h_tab);
  B_TRY(ctx, bc.fields.ensure(sizeof(BatchField) * n));
  B_TRY(ctx, bc.meshes.ensure(sizeof(BatchMesh) * n));
  B_TRY(ctx, bc.kb.ensure(sizeof(unsigned long long) * (n + 1)));
  B_TRY(ctx, bc.fbase.ensure(sizeof(unsigned) * (n + 1)));
  B_TRY(ctx, bc.item_base.ensure(sizeof(unsigned) * n));
  auto upload_fields = [&]() -> cudaError_t {
    memcpy(ht + o_f, hf.data(), sizeof(BatchField) * n);
    unsigned* ib = reinterpret_cast<unsigned*>(ht + o_i);
    for (uint32_t i = 0; i < n; ++i) ib[i] = hf[i].item_base;
    cudaError_t e =
        cudaMemcpyAsync(bc.fields.p, ht + o_f, sizeof(BatchField) * n, cudaMemcpyHostToDevice, ctx->stream);
    if (!e) e = cudaMemcpyAsync(bc.item_base.p, ht + o_i, sizeof(unsigned) * n, cudaMemcpyHostToDevice, ctx->stream);
    return e;
  };
  memcpy(ht + o_m, hm.data(), sizeof(BatchMesh) * n);
  memcpy(ht + o_k, hkb.data(), sizeof(unsigned long long) * (n + 1));
  B_TRY(ctx, cudaMemcpyAsync(bc.meshes.p, ht + o_m, sizeof(BatchMesh) * n, cudaMemcpyHostToDevice, ctx->stream));
  B_TRY(ctx, cudaMemcpyAsync(bc.kb.p, ht + o_k, sizeof(unsigned long long) * (n + 1), cudaMemcpyHostToDevice,
                             ctx->stream));
  unsigned cap = bc.cap_hint ? bc.cap_hint : 65536u;
  unsigned ccap = bc.ccap_hint ? bc.ccap_hint : 65536u;
  const BatchField* dfields = static_cast<const BatchField*>(bc.fields.p);
  const unsigned* ditems = static_cast<const unsigned*>(bc.item_base.p);

  // time chunk: as set, else the autotuner's choice for this batch shape,
  // timed once over the cull launch alone (results never depend on it)
  int pick = bc.tchunk;
  if (pick == 0) {
    for (const auto& t : bc.tunes)
      if (t.first == sig) pick = t.second;
  }
  if (pick == 0) {
    B_TRY(ctx, ctx->cand_corner.ensure(sizeof(unsigned long long) * (size_t)ccap));
    B_TRY(ctx, ctx->cand_chains.ensure(sizeof(unsigned long long) * (size_t)ccap));
    B_TRY(ctx, bc.cand_field.ensure(sizeof(unsigned) * (size_t)ccap));
    B_TRY(ctx, ctx->counters.ensure(sizeof(unsigned) * kNumCounters));
    CandidateQueue cq{};
    cq.corner = static_cast<unsigned long long*>(ctx->cand_corner.p);
    cq.chains = static_cast<unsigned long long*>(ctx->cand_chains.p);
    cq.count = static_cast<unsigned*>(ctx->counters.p) + kCountCand;
    cq.cap = ccap;
    cq.field = static_cast<unsigned*>(bc.cand_field.p);
    unsigned* const counters = static_cast<unsigned*>(ctx->counters.p);
    float best = 0.f;
    const int picks[3] = {0xFFFF, 4, 2};
    for (int c = 0; c < 3; ++c) {
      const unsigned long long it = assign_items(picks[c]);
      if (it == ~0ull) continue;
      B_TRY(ctx, upload_fields());
      float tbest = 0.f;
      for (int rep = 0; rep < 3; ++rep) {
        B_TRY(ctx, cudaMemsetAsync(counters, 0, sizeof(unsigned) * kNumCounters, ctx->stream));
        B_TRY(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
        B_TRY(ctx, launch_batch_cull(f64, multi, dfields, ditems, (int)n, (unsigned)it, counters + kCountItems, cq,
                                     counters + kCountErr, ctx->stream));
        B_TRY(ctx, cudaEventRecord(ctx->ev_x, ctx->stream));
        B_TRY(ctx, ctx->sync());
        ctx->launches += 1;
        float ms = 0.f;
        B_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev_x));
        if (rep == 1 || (rep > 1 && ms < tbest)) tbest = ms;  // rep 0 warms up
      }
      if (pick == 0 || tbest < best) {
        pick = picks[c];
        best = tbest;
      }
    }
    if (pick == 0) pick = 0xFFFF;
    if (bc.tunes.size() >= 64) bc.tunes.erase(bc.tunes.begin());
    bc.tunes.push_back({sig, pick});
  }
  const unsigned long long items = assign_items(pick);
  if (items == ~0ull) return bfail(ctx, FTK2B_UNSUPPORTED, "the batch has more than 2^32 tiles");
  bc.last_tchunk = pick;
  B_TRY(ctx, upload_fields());
  if (bc.h_fbase_n < n + 1) {
    void* p = bc.h_fbase;
    size_t have = bc.h_fbase_n * sizeof(unsigned);
    B_TRY(ctx, ensure_pinned(&p, &have, sizeof(unsigned) * (n + 1)));
    bc.h_fbase = static_cast<unsigned*>(p);
    bc.h_fbase_n = have / sizeof(unsigned);
  }

  const BatchMesh* dmeshes = static_cast<const BatchMesh*>(bc.meshes.p);
  const unsigned long long* dkb = static_cast<const unsigned long long*>(bc.kb.p);
  for (int attempt = 0; attempt < 5; ++attempt) {
    const unsigned edge_cap = cap * 2;
    st = ensure_feature_buffers(ctx, cap, edge_cap, 3);  // rows of 4 vertex ids
    if (st) return st;
    B_TRY(ctx, ctx->cand_corner.ensure(sizeof(unsigned long long) * (size_t)ccap));
    B_TRY(ctx, ctx->cand_chains.ensure(sizeof(unsigned long long) * (size_t)ccap));
    B_TRY(ctx, bc.cand_field.ensure(sizeof(unsigned) * (size_t)ccap));
    B_TRY(ctx, ctx->refine_pairs.ensure(refine_mask_bytes(ccap, cap)));
    PostBuffers B = ctx->post_buffers(cap, edge_cap, key_bits);
    FeatureSink sink;
    sink.key = B.key;
    sink.lam = B.lam;
    sink.bary4 = B.bary4;
    sink.scalar = B.scalar;
    sink.count = B.count;
    sink.cap = cap;
    CandidateQueue cq{};
    cq.corner = static_cast<unsigned long long*>(ctx->cand_corner.p);
    cq.chains = static_cast<unsigned long long*>(ctx->cand_chains.p);
    cq.count = static_cast<unsigned*>(ctx->counters.p) + kCountCand;
    cq.cap = ccap;
    cq.field = static_cast<unsigned*>(bc.cand_field.p);
    unsigned* const counters = static_cast<unsigned*>(ctx->counters.p);
    unsigned* const dfbase = static_cast<unsigned*>(bc.fbase.p);
    RefineStage rs;
    refine_stage_bind(rs, ctx->refine_pairs.p, ccap, cap);
    rs.count = counters + kCountPairs;
    rs.err = counters + kCountErr;
    rs.big_count = counters + kCountBig;
    rs.acc_count = counters + kCountAcc;
    auto enqueue1 = [&](unsigned long long* nl) -> cudaError_t {
      cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned) * kNumCounters, ctx->stream);
      if (!e)
        e = launch_batch_cull(f64, multi, dfields, ditems, (int)n, (unsigned)items, counters + kCountItems, cq, B.err,
                              ctx->stream);
      *nl += 1;
      return e;
    };
    auto enqueue2 = [&](unsigned long long* nl) -> cudaError_t {
      cudaError_t e = launch_batch_refine_staged(f64, dfields, cq, rs, sink, ctx->num_sms, ctx->stream);
      *nl += 3;
      if (!e) e = launch_post_batch(dmeshes, dkb, (int)n, B, dfbase, ctx->stream, nl);
      if (!e)
        e = cudaMemcpyAsync(ctx->h_counters, counters, sizeof(unsigned) * kNumCounters, cudaMemcpyDeviceToHost,
                            ctx->stream);
      if (!e)
        e = cudaMemcpyAsync(bc.h_fbase, dfbase, sizeof(unsigned) * (n + 1), cudaMemcpyDeviceToHost, ctx->stream);
      return e;
    };
    if (ctx->use_graphs) {
      BatchGraphKey key;
      memset(&key, 0, sizeof(key));
      key.nf = (int)n;
      key.n_items = (unsigned)items;
      key.cap = cap;
      key.ccap = ccap;
      key.edge_cap = edge_cap;
      key.key_bits = key_bits;
      key.f64 = f64;
      key.multi = multi;
      key.h_fbase = bc.h_fbase;
      const unsigned long long gen = ctx->buffer_generation();
      if (!bc.g1 || bc.ggen != gen || memcmp(&bc.gkey, &key, sizeof(key)) != 0) {
        bc.drop_graph();
        unsigned long long nl = 0;
        cudaGraphExec_t* slots[2] = {&bc.g1, &bc.g2};
        for (int part = 0; part < 2; ++part) {
          cudaGraph_t graph = nullptr;
          B_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
          const cudaError_t ce = part == 0 ? enqueue1(&nl) : enqueue2(&nl);
          const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &graph);
          if (ce || ee) {
            if (graph) cudaGraphDestroy(graph);
            bc.drop_graph();
            cudaGetLastError();
            return bfail(ctx, FTK2B_CUDA_ERROR, "batch graph capture failed: %s", cudaGetErrorString(ce ? ce : ee));
          }
          const cudaError_t ie = cudaGraphInstantiate(slots[part], graph, 0);
          cudaGraphDestroy(graph);
          if (ie) {
            bc.drop_graph();
            return bfail(ctx, FTK2B_CUDA_ERROR, "batch graph instantiate failed: %s", cudaGetErrorString(ie));
          }
        }
        bc.gkey = key;
        bc.ggen = gen;
        bc.glaunches = nl;
      }
      B_TRY(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
      B_TRY(ctx, cudaGraphLaunch(bc.g1, ctx->stream));
      B_TRY(ctx, cudaEventRecord(ctx->ev_x, ctx->stream));
      B_TRY(ctx, cudaGraphLaunch(bc.g2, ctx->stream));
      B_TRY(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
      ctx->launches += bc.glaunches;
    } else {
      unsigned long long nl = 0;
      B_TRY(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
      B_TRY(ctx, enqueue1(&nl));
      B_TRY(ctx, cudaEventRecord(ctx->ev_x, ctx->stream));
      B_TRY(ctx, enqueue2(&nl));
      B_TRY(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
      ctx->launches += nl;
    }
    B_TRY(ctx, ctx->sync());
    unsigned h[kNumCounters];
    memcpy(h, ctx->h_counters, sizeof(h));
    float ms = 0.f, xms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) != cudaSuccess) ms = 0.f;
    if (cudaEventElapsedTime(&xms, ctx->ev0, ctx->ev_x) != cudaSuccess) xms = 0.f;
    cudaGetLastError();
    ctx->last_extract_ms = xms;
    ctx->last_candidates = h[kCountCand];
    ctx->last_tested = h[kCountPairs];
    if (h[kCountErr] & kErrBounds) return bfail(ctx, FTK2B_INTERNAL, "a device bounds check failed (checked build)");
    if (h[kCountErr] & 2u) return bfail(ctx, FTK2B_TIMEOUT, "a TMA slice copy did not complete in time");
    if (h[kCountErr]) return bfail(ctx, FTK2B_TIMEOUT, "union-find retry bound reached");
    if (h[kCountCand] > ccap) {
      const uint64_t want = (uint64_t)h[kCountCand] + h[kCountCand] / 4 + 1024;
      if (want > 0xFFFFFFF0ull) return bfail(ctx, FTK2B_OVERFLOW_RETRY, "candidate count exceeds 2^32");
      ccap = (unsigned)want;
      bc.ccap_hint = ccap;
      continue;
    }
    if (h[kCountFeatures] > cap || h[kCountEdges] > edge_cap) {
      uint64_t want = (uint64_t)h[kCountFeatures] + h[kCountFeatures] / 4 + 1024;
      const uint64_t want_e = ((uint64_t)h[kCountEdges] + 1) / 2 + 1024;
      if (want_e > want) want = want_e;
      if (want > 0x7FFFFFF0ull) return bfail(ctx, FTK2B_OVERFLOW_RETRY, "feature count exceeds 2^31");
      cap = (unsigned)want;
      bc.cap_hint = cap;
      continue;
    }
    bc.nf = (int)n;
    bc.n = h[kCountFeatures];
    bc.ne = h[kCountEdges];
    bc.device_ms = ms;
    bc.fb.assign(bc.h_fbase, bc.h_fbase + n + 1);
    ctx->last.device_ms = ms;
    return FTK2B_OK;
  }
  return bfail(ctx, FTK2B_OVERFLOW_RETRY, "batch buffers kept overflowing");
}

}  // namespace

extern "C" ftk2b_status ftk2b_cp_run_batch(ftk2b_ctx* ctx, uint32_t n, const ftk2b_mesh_desc* meshes,
                                           const ftk2b_field_desc* fields, const ftk2b_cp_params* params,
                                           uint64_t* n_features) {
  ftk2b::NvtxRange nvtx_range("ftk2b_cp_run_batch");
  if (!ctx) return FTK2B_INVALID_ARG;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return bfail(ctx, FTK2B_CUDA_ERROR, "cudaSetDevice failed");
  ctx->batch.nf = 0;
  const ftk2b_status st = run_batch(ctx, n, meshes, fields, params);
  if (st == FTK2B_OK && n_features) *n_features = ctx->batch.n;
  return st;
}

extern "C" ftk2b_status ftk2b_cp_fetch_batch(ftk2b_ctx* ctx, ftk2b_cp_result** out) {
  ftk2b::NvtxRange nvtx_range("ftk2b_cp_fetch_batch");
  if (!ctx || !out) return FTK2B_INVALID_ARG;
  BatchCtx& bc = ctx->batch;
  if (bc.nf <= 0) return bfail(ctx, FTK2B_INVALID_ARG, "no batch has run on this context");
  const uint64_t n = bc.n, ne = bc.ne;
  std::vector<unsigned long long> simp(4 * n + 4), track(n + 1);
  std::vector<float> bary(4 * n + 4), sc(n + 1);
  std::vector<double> lam(4 * n + 4);
  std::vector<unsigned> edges(2 * ne + 2);
  cudaStream_t s = ctx->stream;
  auto d2h = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s) : cudaSuccess;
  };
  B_TRY(ctx, d2h(simp.data(), ctx->simplices.p, sizeof(unsigned long long) * 4 * n));
  B_TRY(ctx, d2h(bary.data(), ctx->bary.p, sizeof(float) * 4 * n));
  B_TRY(ctx, d2h(lam.data(), ctx->lam_s.p, sizeof(double) * 4 * n));
  B_TRY(ctx, d2h(sc.data(), ctx->scalar_s.p, sizeof(float) * n));
  B_TRY(ctx, d2h(track.data(), ctx->track.p, sizeof(unsigned long long) * n));
  B_TRY(ctx, d2h(edges.data(), ctx->edges.p, sizeof(unsigned) * 2 * ne));
  B_TRY(ctx, ctx->sync());
  const int nf = bc.nf;
  for (int f = 0; f < nf; ++f) out[f] = nullptr;
  for (int f = 0; f < nf; ++f) {
    const unsigned b = bc.fb[f], e = bc.fb[f + 1];
    const uint64_t cnt = e - b;
    const BatchFieldInfo& inf = bc.info[f];
    const size_t k = (size_t)inf.m + 1;
    ftk2b_cp_result* r = (ftk2b_cp_result*)calloc(1, sizeof(ftk2b_cp_result));
    if (r) {
      r->simplices = (uint64_t*)malloc(sizeof(uint64_t) * (cnt * k + 1));
      r->lambda = (double*)malloc(sizeof(double) * (cnt * k + 1));
      r->barycentric = (float*)malloc(sizeof(float) * (cnt * k + 1));
      r->track_id = (uint64_t*)malloc(sizeof(uint64_t) * (cnt + 1));
      r->type = (uint32_t*)calloc(cnt + 1, sizeof(uint32_t));
      r->cp_class = (uint32_t*)calloc(cnt + 1, sizeof(uint32_t));
      r->scalar = (float*)malloc(sizeof(float) * (cnt + 1));
    }
    // this field's star edges: their centres lie in [b, e) and the global
    // list is sorted by centre
    auto centre_lb = [&](unsigned v) {
      uint64_t lo = 0, hi = ne;
      while (lo < hi) {
        const uint64_t mid = (lo + hi) / 2;
        if (edges[2 * mid] < v) lo = mid + 1;
        else hi = mid;
      }
      return lo;
    };
    const uint64_t eb = inf.want_edges ? centre_lb(b) : 0, ee = inf.want_edges ? centre_lb(e) : 0;
    if (r) r->edges = (uint32_t*)malloc(sizeof(uint32_t) * (2 * (ee - eb) + 2));
    if (!r || !r->simplices || !r->lambda || !r->barycentric || !r->track_id || !r->type || !r->cp_class ||
        !r->scalar || !r->edges) {
      ftk2b_cp_result_free(r);
      for (int g = 0; g < f; ++g) {
        ftk2b_cp_result_free(out[g]);
        out[g] = nullptr;
      }
      return bfail(ctx, FTK2B_OOM, "host allocation failed");
    }
    r->m = inf.m;
    r->n_features = cnt;
    r->n_simplices = inf.nsimp;
    r->device_ms = bc.device_ms;
    uint64_t roots = 0;
    for (uint64_t i = 0; i < cnt; ++i) {
      const uint64_t g = b + i;
      for (size_t v = 0; v < k; ++v) {
        r->simplices[i * k + v] = simp[4 * g + v];
        r->barycentric[i * k + v] = bary[4 * g + v];
        r->lambda[i * k + v] = lam[4 * g + v];
      }
      r->scalar[i] = sc[g];
      if (inf.want_edges) {
        r->track_id[i] = track[g] - b;
        roots += track[g] == g;
      } else {
        r->track_id[i] = i;
      }
    }
    r->n_tracks = inf.want_edges ? roots : 0;
    r->n_edges = ee - eb;
    for (uint64_t j = eb; j < ee; ++j) {
      r->edges[2 * (j - eb)] = edges[2 * j] - b;
      r->edges[2 * (j - eb) + 1] = edges[2 * j + 1] - b;
    }
    out[f] = r;
  }
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_cp_extract_batch(ftk2b_ctx* ctx, uint32_t n, const ftk2b_mesh_desc* meshes,
                                               const ftk2b_field_desc* fields, const ftk2b_cp_params* params,
                                               ftk2b_cp_result** out) {
  if (!out) return ctx ? bfail(ctx, FTK2B_INVALID_ARG, "null output") : FTK2B_INVALID_ARG;
  ftk2b_status st = ftk2b_cp_run_batch(ctx, n, meshes, fields, params, nullptr);
  if (st) return st;
  return ftk2b_cp_fetch_batch(ctx, out);
}
