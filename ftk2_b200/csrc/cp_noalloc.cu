// Allocation-free variant of the regular-mesh feature extraction.
//
// Who needs it: callers that may not allocate device memory while they run.
// An in-situ analysis step inside a simulation whose memory manager already
// owns the whole device cannot get memory from cudaMalloc without evicting
// the simulation's own pool; a serving loop held to a fixed memory budget
// cannot afford cudaMalloc's implicit device synchronisation in the middle of
// its latency budget.  They get one entry point that uses no cudaMalloc or
// cudaFree (and no allocating library routine): its scratch is the file-scope
// array below, which every GPU that loads this library keeps until the
// process exits.  Inputs and outputs stay the caller's.
//
// Limits: at most kMaxCandidates surviving hypercubes and kMaxFeatures
// accepted simplices per call (scratch: ~9.3 MiB per device).  More surviving
// hypercubes than the scratch holds returns FTK2B_UNSUPPORTED: the same call
// can never succeed, so the caller splits the box into sub-boxes
// (RegularSimplicialMesh offsets).  Every call shares the array; the entry
// point clears the counters it needs at the start of each call, and calls
// whose device work overlaps (on different streams or host threads at the
// same time) race on the shared array.
#include <cstring>
#include <mutex>

#include "../../include/ftk2b.h"
#include "cp_internal.h"

namespace ftk2b {

constexpr unsigned kMaxCandidates = 1u << 18;
constexpr unsigned kMaxFeatures = 1u << 18;

// layout (64-bit words): candidate corners | candidate chain masks |
// float barycentrics (4 per feature, 2 per word) | scalars (2 per word) | counters
constexpr size_t kOffCorner = 0;
constexpr size_t kOffChains = kOffCorner + kMaxCandidates;
constexpr size_t kOffBary = kOffChains + kMaxCandidates;
constexpr size_t kOffScalar = kOffBary + 2 * (size_t)kMaxFeatures;
constexpr size_t kOffCounters = kOffScalar + kMaxFeatures / 2;
constexpr size_t kScratchWords = kOffCounters + 4;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kScratchWords];

// per-device set-up: the array's device address (host code must not use the
// symbol itself as a device pointer) and the constant tables of the kernels
static std::mutex g_setup_mu;
static void* g_scratch_ptr[64];
static bool g_setup_done[64];

static ftk2b_status noalloc_setup(int dev, void** ptr) {
  if (dev < 0 || dev >= 64) return FTK2B_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_setup_done[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return FTK2B_CUDA_ERROR;
    }
    if (!ensure_device_tables(dev)) return FTK2B_CUDA_ERROR;
    g_scratch_ptr[dev] = p;
    g_setup_done[dev] = true;
  }
  *ptr = g_scratch_ptr[dev];
  return FTK2B_OK;
}

}  // namespace ftk2b

using namespace ftk2b;

extern "C" ftk2b_status ftk2b_cp_features_noalloc(const ftk2b_mesh_desc* mesh,
                                                  const ftk2b_field_desc* field, double sos_q,
                                                  void* stream, uint64_t* keys, double* lambda,
                                                  uint32_t capacity, uint32_t* count,
                                                  uint64_t* n_features) {
  if (!mesh || !field || !keys || !lambda || !count || !n_features) return FTK2B_INVALID_ARG;
  if (!(sos_q > 0)) return FTK2B_INVALID_ARG;
  if (mesh->kind != FTK2B_MESH_REGULAR) return FTK2B_UNSUPPORTED;
  if (field->location != FTK2B_DEVICE) return FTK2B_INVALID_ARG;  // staging would allocate
  if (capacity > kMaxFeatures) return FTK2B_INVALID_ARG;          // beyond the static scratch
  const int d = mesh->ndims;
  if (d != 3 && d != 4) return FTK2B_UNSUPPORTED;
  const int M = d - 1;
  if (field->ncomp != M) return FTK2B_INVALID_ARG;
  if (field->dtype != FTK2B_F32 && field->dtype != FTK2B_F64) return FTK2B_INVALID_ARG;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FTK2B_NO_DEVICE;
  void* scratch = nullptr;
  ftk2b_status st = noalloc_setup(dev, &scratch);
  if (st != FTK2B_OK) return st;

  // mesh and field descriptors (device pointers used in place)
  RegularMesh rm;
  memset(&rm, 0, sizeof(rm));
  rm.d = d;
  unsigned long long s = 1;
  for (int k = 0; k < d; ++k) {
    if (mesh->local_dims[k] < 1 || mesh->local_dims[k] >= (1ull << 16) ||
        mesh->offset[k] + mesh->local_dims[k] > mesh->global_dims[k])
      return FTK2B_INVALID_ARG;
    rm.ld[k] = (long long)mesh->local_dims[k];
    rm.off[k] = (long long)mesh->offset[k];
    rm.gd[k] = (long long)mesh->global_dims[k];
    rm.gstride[k] = s;
    s *= mesh->global_dims[k];
  }
  FieldAccess fa;
  memset(&fa, 0, sizeof(fa));
  const size_t es = field->dtype == FTK2B_F64 ? 8 : 4;
  if (field->layout == FTK2B_LAYOUT_MULTICOMPONENT) {
    if (field->nd != d || !field->comp[0]) return FTK2B_INVALID_ARG;
    long long st2 = M;
    for (int k = 0; k < d; ++k) {
      if (field->dims[k] < mesh->offset[k] + mesh->local_dims[k]) return FTK2B_INVALID_ARG;
      fa.adims[k] = (long long)field->dims[k];
      fa.estride[k] = st2;
      st2 *= (long long)field->dims[k];
    }
    for (int j = 0; j < M; ++j) fa.comp[j] = (const char*)field->comp[0] + j * es;
  } else if (field->layout == FTK2B_LAYOUT_SEPARATE && field->nd == d) {
    long long st2 = 1;
    for (int k = 0; k < d; ++k) {
      if (field->dims[k] < mesh->local_dims[k]) return FTK2B_INVALID_ARG;
      fa.adims[k] = (long long)field->dims[k];
      fa.estride[k] = st2;
      fa.shift[k] = rm.off[k];
      st2 *= (long long)field->dims[k];
    }
    for (int j = 0; j < M; ++j) {
      if (!field->comp[j]) return FTK2B_INVALID_ARG;
      fa.comp[j] = field->comp[j];
    }
  } else {
    return FTK2B_UNSUPPORTED;
  }

  int TX, TY, TZ;
  regular_tile(d, &TX, &TY, &TZ);
  ExtractConfig cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.Q = sos_q;
  cfg.tchunk = (int)rm.ld[d - 1];
  cfg.tiles[0] = (int)((rm.ld[0] + TX - 1) / TX);
  cfg.tiles[1] = (int)((rm.ld[1] + TY - 1) / TY);
  cfg.tiles[2] = (d == 4) ? (int)((rm.ld[2] + TZ - 1) / TZ) : 1;

  unsigned long long* sw = static_cast<unsigned long long*>(scratch);
  unsigned* counters = reinterpret_cast<unsigned*>(sw + kOffCounters);  // [0] candidates, [1] error
  CandidateQueue cq{};
  cq.corner = sw + kOffCorner;
  cq.chains = sw + kOffChains;
  cq.count = counters;
  cq.cap = kMaxCandidates;
  FeatureSink sink;
  sink.key = reinterpret_cast<unsigned long long*>(keys);
  sink.lam = lambda;
  sink.bary4 = reinterpret_cast<float*>(sw + kOffBary);
  sink.scalar = reinterpret_cast<float*>(sw + kOffScalar);
  sink.count = count;
  sink.cap = capacity;

  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  int num_sms = 148;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  // the shared scratch keeps the last call's contents: clear the counters
  if (cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned), cs) != cudaSuccess ||
      cudaMemsetAsync(count, 0, sizeof(uint32_t), cs) != cudaSuccess) {
    cudaGetLastError();
    return FTK2B_CUDA_ERROR;
  }
  const int f64 = field->dtype == FTK2B_F64;
  if (launch_extract_regular(f64, rm, fa, cfg, cq, counters + 1, cs, true, nullptr) != cudaSuccess ||
      launch_refine_regular(f64, rm, fa, cfg, cq, sink, num_sms, cs) != cudaSuccess) {
    cudaGetLastError();
    return FTK2B_CUDA_ERROR;
  }
  unsigned h[4] = {0, 0, 0, 0};
  unsigned nf = 0;
  if (cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
      cudaMemcpyAsync(&nf, count, sizeof(nf), cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
      cudaStreamSynchronize(cs) != cudaSuccess) {
    cudaGetLastError();
    return FTK2B_CUDA_ERROR;
  }
  *n_features = nf;
  if (h[1]) return FTK2B_TIMEOUT;                      // a bounded TMA wait gave up
  // more survivors than the static scratch holds: no retry of this call can
  // succeed, the box has to be split
  if (h[0] > kMaxCandidates) return FTK2B_UNSUPPORTED;
  if (nf > capacity) return FTK2B_OVERFLOW_RETRY;     // caller's output too small
  return FTK2B_OK;
}
