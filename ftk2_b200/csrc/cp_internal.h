// Internal launch descriptors shared by the kernel translation units and the
// C-ABI layer.  Plain structs passed to kernels by value.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ftk2b {

// Device bounds checks of the checked build (compiled with -DFTK2B_CHECKED):
// FTK2B_CHECK(cond, err) is `cond`, and a failed check sets bit 3 of the
// call's error word (the call then reports FTK2B_INTERNAL) so that the
// caller can skip the access; never a trap.  In the normal build it is
// `true` and the compiler drops the test.
constexpr unsigned kErrBounds = 8u;
#ifdef FTK2B_CHECKED
__device__ __forceinline__ bool checked_bound(bool ok, unsigned* err) {
  if (!ok && err) atomicOr(err, kErrBounds);
  return ok;
}
#define FTK2B_CHECK(cond, err) (::ftk2b::checked_bound((cond), (err)))
#else
#define FTK2B_CHECK(cond, err) (true)
#endif

constexpr int kMaxChains = 64;

// Value access for a field sampled on a regular grid or per vertex.
//   multicomponent [M, d0, d1, ...] (Fortran):  comp[j] = base + j,
//       estride = {M, M*d0, M*d0*d1, ...}, shift = 0 (global coordinates,
//       engine.hpp:1101-1124)
//   separate arrays [d0, d1, ...]:             comp[j] = array j,
//       estride = {1, d0, d0*d1, ...}, shift = mesh offset (engine.hpp:999-1009)
//   per-vertex 1D arrays:                      index = vertex id
struct FieldAccess {
  const void* comp[3];
  long long estride[4];
  long long shift[4];
  long long adims[4];          // array dims (Fortran, excluding the component dim)
  int per_vertex;
  // optional scalar (interpolated only for separate-array fields,
  // predicate.hpp:81-92 with the arrays the engine passes, engine.hpp:1125-1139)
  const void* scalar;
  long long sstride[4];
  int scalar_per_vertex;
  int has_scalar;
  // time-axis index of the component arrays = (g - shift) xor tflip: a
  // stream's two-slot ring keeps timestep t in slot t & 1 (0 otherwise)
  int tflip;
};

// Regular spacetime mesh: RegularSimplicialMesh(local, offset, global)
// (mesh.hpp:256-265).  Corners range over the local box; vertex ids use the
// global dims (mesh.hpp:439-451).
struct RegularMesh {
  int d;                       // 3 (2D + t) or 4 (3D + t)
  long long ld[4];             // local dims
  long long off[4];            // offset of the local box in global coordinates
  long long gd[4];             // global dims
  unsigned long long gstride[4];
};

// Output of the extraction stage (unsorted, capacity-bounded)
struct FeatureSink {
  unsigned long long* key;     // canonical key: corner vertex id * n_chains + chain rank
  double* lam;                 // 4 per feature: reported barycentrics
  float* bary4;                // 4 per feature: (float) of the exact-path barycentrics
  float* scalar;
  unsigned int* count;         // number found (may exceed cap: overflow)
  unsigned int cap;
};

// Hypercubes that survive the cull, with the chains (simplex types) whose
// vertices also survive it; consumed by the exact-test kernel.
struct CandidateQueue {
  unsigned long long* corner;  // local corner coords, 16 bits each: x | y << 16 | z << 32 | t << 48
  unsigned long long* chains;  // bit c: chain c still needs the exact test
  unsigned* count;             // number queued (may exceed cap: overflow)
  unsigned cap;
  unsigned* field;             // batches: field index of every candidate (null otherwise)
  unsigned field_id;           // the index written by the current tile
};

struct ExtractConfig {
  double Q;                    // sos_q
  int refined;                 // 1: report FP32 + one FP64 refinement step
  int tchunk;                  // corner time steps per block
  int tiles[3];                // tiles along x, y, z (z = 1 for 2D)
  int skip_first_spatial;      // 1: no purely spatial simplices at local time 0
  int cull_mode;               // 0: per-vertex cull words only; 1: tile statistics first
  // > 0: failure-path check of the fused cull: after its first slice every
  // block waits, at most this many polls, on an mbarrier nothing completes,
  // and leaves through the timeout path (the call reports FTK2B_TIMEOUT)
  int stall_polls;
  // FiberPredicate<T> (predicate.hpp:341-362): every hypercube is a candidate
  // (the cull words assume the solve must succeed), values are taken minus
  // fthr[j], and a simplex whose solve fails is kept at the centroid
  int fiber;
  double fthr[2];
  // scratch of cull mode 1 (device): 8 ints per (slice, tile), and the runs
  // of surviving tile-steps (4 words each: tile, first step, end step, pad)
  int* tstats;
  unsigned* runs;
  unsigned* n_runs;
  unsigned runs_cap;
};

// chain tables: masks of vertices 1..m of every m-simplex type of a
// d-hypercube, in canonical (vertex-id) order
struct ChainTable {
  int n;
  unsigned char mask[kMaxChains][4];
};

void upload_chain_tables();
// Uploads the chain and post-processing constant tables to the current
// device once per device for the life of the process (a second upload while
// kernels of another caller read them would be a race).  Returns false when a
// CUDA call failed.
bool ensure_device_tables(int device);

// Launches the fused extraction; uses TMA tensor-tile staging when allowed
// and the array satisfies the 16-byte alignment rules (reported in used_tma);
// *launches (optional) receives the number of kernels it launched.
cudaError_t launch_extract_regular(int f64, const RegularMesh& mesh, const FieldAccess& fa,
                                   const ExtractConfig& cfg, const CandidateQueue& cq, unsigned* err,
                                   cudaStream_t st, bool allow_tma, int* used_tma, int* launches = nullptr);
// Scratch of cull mode 1 for a mesh: tile-slice statistics and run list sizes.
void tile_scratch_size(const RegularMesh& mesh, size_t* stats_bytes, unsigned* runs_cap);
// Exact SoS + solve of the queued candidates, compacted into the sink.
// FiberPredicate: queue every local vertex as a corner with all its in-mesh
// chains (no cull)
cudaError_t launch_fiber_candidates(const RegularMesh& mesh, const CandidateQueue& cq, int num_sms,
                                    cudaStream_t st);
// The exact test of the queued candidates: the fast-path inside test of
// every surviving simplex of the candidates whose quantised values all stay
// below 2^31, listing the simplices it accepts; the solve of the listed
// simplices; and the whole test of the other candidates' simplices (listed)
// with the 128-bit path.  Values and their quantised form stay in shared
// memory; the solve and the 128-bit path read values from the field.
struct RefineStage {
  unsigned long long* big_live;  // per listed candidate: chains to test on the 128-bit path
  unsigned* big_list;            // candidates listed for the 128-bit path
  unsigned* big_count;
  unsigned long long* acc;       // simplices inside by the fast path: candidate << 8 | chain
  unsigned* acc_count;           // may exceed acc_cap (then the call reports overflow)
  unsigned acc_cap;
  unsigned* count;   // simplices tested (reported after the run)
  unsigned* err;     // the call's error word (bounds checks of the checked build)
};
// bytes of the 128-bit list for `ccap` candidates (chain masks and
// candidates) and of the inside list (acc_cap entries)
inline size_t refine_mask_bytes(size_t ccap, size_t acc_cap) { return ccap * (8 + 4) + acc_cap * 8; }
inline void refine_stage_bind(RefineStage& rs, void* masks, size_t ccap, unsigned acc_cap) {
  rs.big_live = static_cast<unsigned long long*>(masks);
  rs.acc = rs.big_live + ccap;
  rs.acc_cap = acc_cap;
  rs.big_list = reinterpret_cast<unsigned*>(rs.acc + acc_cap);
}
cudaError_t launch_refine_staged(int f64, const RegularMesh& mesh, const FieldAccess& fa, const ExtractConfig& cfg,
                                 const CandidateQueue& cq, const RefineStage& rs, const FeatureSink& sink, int num_sms,
                                 cudaStream_t st);
cudaError_t launch_refine_regular(int f64, const RegularMesh& mesh, const FieldAccess& fa,
                                  const ExtractConfig& cfg, const CandidateQueue& cq,
                                  const FeatureSink& sink, int num_sms, cudaStream_t st);
void regular_tile(int d, int* tx, int* ty, int* tz);

}  // namespace ftk2b
