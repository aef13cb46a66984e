// Batched extraction over many regular-mesh fields: the per-field records the
// batched kernels read from device memory, and their launchers.
#pragma once

#include <cuda.h>

#include "cp_internal.h"

namespace ftk2b {

// One field of a batch.  The tensor maps come first so that each is 64-byte
// aligned in a device array of records (TMA reads them from global memory).
struct alignas(64) BatchField {
  CUtensorMap maps[3];
  RegularMesh mesh;
  FieldAccess fa;
  ExtractConfig cfg;
  unsigned long long key_base;  // first canonical key of the field in the batch's key space
  unsigned item_base;           // first cull item (tile, time chunk) of the field
  int tma;                      // 1: slices staged by TMA through maps
};

// What the post-extraction kernels need of a batch field.
struct BatchMesh {
  RegularMesh mesh;
  int nch;
};

// Tensor maps of a regular-mesh field for the fused cull kernel's slice boxes
// (false: the field's alignment does not allow TMA staging).
bool regular_tma_maps(int f64, const RegularMesh& mesh, const FieldAccess& fa, bool allow, CUtensorMap maps[3]);

// One persistent launch culling every (field, tile, time chunk) item of the
// batch; blocks take items from *item_next (zeroed by the caller);
// item_base[f] = fields[f].item_base (ascending, nf entries).
cudaError_t launch_batch_cull(int f64, int multi, const BatchField* fields, const unsigned* item_base, int nf,
                              unsigned n_items, unsigned* item_next, const CandidateQueue& cq, unsigned* err,
                              cudaStream_t st);
// Exact tests of every queued candidate of the batch (cq.field names its
// field) in three launches: the fast-path inside test (values gathered and
// quantised in shared memory), the solve of the accepted simplices, and the
// 128-bit path; the last two read values from the fields.
cudaError_t launch_batch_refine_staged(int f64, const BatchField* fields, const CandidateQueue& cq,
                                       const RefineStage& rs, const FeatureSink& sink, int num_sms, cudaStream_t st);
// Time chunk of a field of a batch: corner time steps per cull item.
int batch_time_chunk(long long lt, int pick);

}  // namespace ftk2b
