// Context object and cross-file declarations of the C-ABI layer.
#pragma once

#include <chrono>
#include <functional>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/ftk2b.h"
#include "cp_internal.h"
#include "cp_post.h"

namespace ftk2b {

// NVTX range over a scope (a profiler such as Nsight Systems shows the
// library's stages on the host timeline; without one attached the calls do
// nothing)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// grow-only device allocation owned by a context.  With `st` set, memory is
// allocated and freed in stream order on that stream (the only stream that
// uses the buffer), so growing a buffer does not synchronise the device.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  unsigned long long generation = 0;  // bumped on every reallocation
  cudaStream_t st = nullptr;
  cudaError_t ensure(size_t want);
  void release();
};

enum {
  kCountFeatures = 0,
  kCountEdges = 1,
  kCountRoots = 2,
  kCountErr = 3,
  kCountCand = 4,
  kCountItems = 5,  // batches: next cull item
  kCountPairs = 6,  // simplices the exact test ran on
  kCountBig = 7,    // candidates listed for the 128-bit inside test
  kCountAcc = 8,    // simplices inside by the fast path (listed for the solve)
  kCountDone = 9,   // blocks of the short chain's edge kernel that finished
  kNumCounters = 10
};

// Everything a regular-mesh run bakes into its kernel launches; a cached CUDA
// graph is replayed only when the next run's key is byte-identical.
struct RegularGraphKey {
  RegularMesh rm;
  FieldAccess fa;
  ExtractConfig cfg;
  unsigned cap, ccap, edge_cap;
  int f64, want_edges, classify, allow_tma, key_bits, nch;
};

// Extruded meshes: the prepared base mesh (sorted cells, unique sorted
// (cd-1)-faces with their coface cells), kept while the base cells' content
// is unchanged, plus the work buffers of the extruded pipeline.
struct ExtCache {
  bool valid = false;
  uint64_t hash = 0, ncell = 0, ns = 0;
  int cd = 0;
  unsigned nface = 0;
  int fbits = 0;
  DevBuf cells, fkeys, cof_start, cof;
  DevBuf words, hi, lo, phase, hi_s, lo_s, phase_s, sort_k, sort_v, sort_k2, sort_v2, ekeys;
  std::vector<DevBuf*> bufs() {
    return {&cells, &fkeys, &cof_start, &cof, &words, &hi, &lo, &phase, &hi_s, &lo_s, &phase_s,
            &sort_k, &sort_v, &sort_k2, &sort_v2, &ekeys};
  }
};

// One cached pair of instantiated graphs of the regular-mesh pipeline.
struct GraphEntry {
  RegularGraphKey key;
  unsigned long long gen = 0;      // buffer generation at capture
  cudaGraphExec_t g1 = nullptr;    // counters reset + fused cull kernel
  cudaGraphExec_t g2 = nullptr;    // exact tests + canonical order + trajectories
  unsigned long long launches = 0;
  unsigned long long last_use = 0;
  int used_tma = 0;                // whether the captured cull kernel stages with TMA
};
constexpr size_t kMaxGraphs = 16;

// One workload shape decided by the cull-mode autotuner: the regular mesh
// (local dims, offsets), the field's array shape and strides, dtype, layout
// and whether TMA staging was allowed, with the extraction time measured for
// each mode and the faster one.
struct CullTune {
  long long ld[4], off[4], adims[4], estride[4], shift[4];
  int d, f64, multi, tma;
  int mode;
  float ms[2];
};
constexpr size_t kMaxCullTunes = 256;

// Batched extraction state of a context: device tables of the last batch,
// its per-field bookkeeping for the fetch, and its cached graph pair.
struct BatchFieldInfo {
  int m, want_edges;
  uint64_t nsimp;
};
struct BatchGraphKey {
  int nf;
  unsigned n_items, cap, ccap, edge_cap;
  int key_bits, f64, multi;
  const void* h_fbase;
};
struct BatchCtx {
  DevBuf fields, meshes, kb, fbase, cand_field, stage, item_base;
  void* h_tab = nullptr;          // pinned staging of the tables
  size_t h_tab_bytes = 0;
  unsigned* h_fbase = nullptr;    // pinned: first feature of every field
  size_t h_fbase_n = 0;
  unsigned cap_hint = 0, ccap_hint = 0;
  int tchunk = 0;                 // FTK2B_OPT_BATCH_TIME_CHUNK (0: tuned per batch shape)
  int last_tchunk = 0;            // the time chunk the last batch ran (0xFFFF: whole range)
  std::vector<std::pair<uint64_t, int>> tunes;  // batch shape hash -> time chunk
  int nf = 0;
  uint64_t n = 0, ne = 0;
  double device_ms = 0;
  std::vector<BatchFieldInfo> info;
  std::vector<unsigned> fb;       // fbase of the last batch (nf + 1)
  BatchGraphKey gkey;
  unsigned long long ggen = 0, glaunches = 0;
  cudaGraphExec_t g1 = nullptr, g2 = nullptr;
  void drop_graph() {
    if (g1) cudaGraphExecDestroy(g1);
    if (g2) cudaGraphExecDestroy(g2);
    g1 = g2 = nullptr;
  }
  std::vector<DevBuf*> bufs() { return {&fields, &meshes, &kb, &fbase, &cand_field, &stage, &item_base}; }
};

struct LastRun {
  int kind = 0, m = 0, f64 = 0;
  uint64_t n = 0, ne = 0, n_roots = 0, n_simplices = 0;
  double device_ms = 0;
  int classify = 0, want_edges = 1;
};

}  // namespace ftk2b

struct ftk2b_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_x = nullptr;
  unsigned long long launches = 0;
  double last_extract_ms = 0;
  double last_refine_ms = 0;
  cudaEvent_t ev_r = nullptr;
  std::string err;
  unsigned cap_hint = 0;
  unsigned cand_cap_hint = 0;
  int tune_tchunk = 0;
  int cull_mode = 2;  // FTK2B_OPT_CULL_MODE (2: chosen per workload shape)
  int last_cull_mode = 0;  // the mode the last regular-mesh extraction ran
  unsigned long long last_candidates = 0;  // hypercubes the last regular-mesh cull kept
  unsigned long long last_tested = 0;      // simplices the last exact test ran on
  int stall_polls = 0;                     // FTK2B_OPT_TEST_STALL_POLLS
  std::vector<ftk2b::CullTune> cull_tunes;
  bool disable_tma = false;
  int last_used_tma = 0;
  ftk2b::DevBuf stage[3], stage_scalar;
  ftk2b::DevBuf key, lam, bary4, scalar, key_alt, perm0, perm1, hist, lam_s, bary4_s, scalar_s,
      simplices, bary, track, edge_cnt, edges, parent, counters, cls, cand_corner, cand_chains, edge_slots,
      refine_pairs;
  ftk2b::DevBuf tstats, runs;  // cull mode 1 scratch (tile statistics, run list + count)
  std::vector<ftk2b::DevBuf> extra;
  ftk2b::DevBuf attr_out, attr_desc, attr_stage[16];  // ftk2b_cp_attributes
  ftk2b::DevBuf contour[40];  // level-set and fiber-surface scratch and outputs
  unsigned fe_cap = 0;        // extruded fiber surfaces: accepted-triangle capacity (grows)
  // two pinned host chunks for large result copies (allocated on first use)
  void* d2h_pin[2] = {nullptr, nullptr};
  cudaEvent_t d2h_ev[2] = {nullptr, nullptr};
  ftk2b::ExtCache ext;
  ftk2b::BatchCtx batch;
  ftk2b::LastRun last;
  // CUDA graph of the last regular-mesh pipeline
  bool use_graphs = true;
  // least-recently-used cache of the pipeline graphs of recent workloads
  // (descriptor shapes and buffers), so that alternating requests replay
  // instead of capturing again
  std::vector<ftk2b::GraphEntry> graphs;
  unsigned long long graph_clock = 0;
  void drop_graphs() {
    batch.drop_graph();
    for (auto& g : graphs) {
      if (g.g1) cudaGraphExecDestroy(g.g1);
      if (g.g2) cudaGraphExecDestroy(g.g2);
    }
    graphs.clear();
  }
  unsigned* h_counters = nullptr;  // pinned
  // waits for the context's stream: spinning by default, or by blocking on an
  // event (FTK2B_OPT_BLOCKING_SYNC), which frees the host core while waiting
  // host time of the phases of the last call: [0] descriptors, staging and
  // buffers, [1] CUDA-graph capture and instantiation, [2] launch to device
  // completion, [3] result copy-back (ms)
  double phase_ms[4] = {0, 0, 0, 0};
  bool blocking_sync = false;
  cudaEvent_t ev_sync = nullptr;
  cudaError_t sync() {
    if (!blocking_sync) return cudaStreamSynchronize(stream);
    cudaError_t e = cudaEventRecord(ev_sync, stream);
    return e ? e : cudaEventSynchronize(ev_sync);
  }
  unsigned long long buffer_generation() {
    unsigned long long g = 0;
    for (ftk2b::DevBuf* b : all_bufs()) g += b->generation;
    return g;
  }

  // blocks of the radix sort: enough to stream the feature capacity, few
  // enough that the per-pass digit-histogram scan stays short
  int sort_grid(unsigned cap) const {
    int g = (int)(cap / 4096u);
    if (g < 1) g = 1;
    if (g > 2 * num_sms) g = 2 * num_sms;
    return g;
  }
  void release_all();
  std::vector<ftk2b::DevBuf*> all_bufs();
  ftk2b::PostBuffers post_buffers(unsigned cap, unsigned edge_cap, int key_bits);
};

namespace ftk2b {

// Staging of host arrays into one device buffer: consecutive 256-byte
// aligned slots from `off`; a null base only counts the bytes.
struct StageArena {
  unsigned char* base;
  size_t off;
};
// Validates a field descriptor and fills fa (device pointers; host arrays are
// copied to the context's staging buffers, or into the arena when given).
ftk2b_status prepare_field(ftk2b_ctx* ctx, const ftk2b_field_desc* f, int mesh_d,
                           const uint64_t* need_global_hi, const uint64_t* need_local_hi,
                           uint64_t n_vertices, FieldAccess& fa, StageArena* arena = nullptr);
// RegularSimplicialMesh(local, offset, global) of a descriptor, validated.
ftk2b_status build_regular(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, RegularMesh& rm);
ftk2b_status ensure_feature_buffers(ftk2b_ctx* ctx, unsigned cap, unsigned edge_cap, int m);

// Sizes the tile-statistics scratch of cull mode 1 for this mesh and points
// cfg at it.
cudaError_t setup_cull_scratch(ftk2b_ctx* ctx, const RegularMesh& rm, ExtractConfig& cfg);

// The cull mode of a regular-mesh extraction: modes 0 and 1 as the context
// sets them; in mode 2 the mode decided for this workload shape, or, for a new
// shape, the faster of 0 and 1 as timed with `enqueue(mode)` (counters reset
// plus the extraction, on the context's stream): one warm-up pass, then the
// best of three per mode.  Results never depend on the mode.
cudaError_t resolve_cull_mode(ftk2b_ctx* ctx, const RegularMesh& rm, const FieldAccess& fa, int f64, bool multi,
                              const std::function<cudaError_t(int)>& enqueue, int* mode);

}  // namespace ftk2b

// extruded meshes (cp_extruded.cu)
// fiber_thr: null for CriticalPointPredicate; the two thresholds for
// FiberPredicate (triangle bases)
ftk2b_status run_extruded(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* field,
                          const ftk2b_cp_params* prm, const double* fiber_thr = nullptr);
uint64_t extruded_simplex_count(const ftk2b_mesh_desc* mesh, int m);
