// Time streams: a spatial mesh whose timesteps arrive one at a time.
#pragma once

#include <vector>

#include "cp_api_internal.h"

struct ftk2b_stream {
  ftk2b_ctx* ctx = nullptr;
  int kind = 0;        // FTK2B_MESH_REGULAR / FTK2B_MESH_EXTRUDED
  int d = 0, m = 0;    // spacetime dims, codimension-1 simplex dim
  ftk2b_cp_params prm;
  int dtype = 0, layout = 0, ncomp = 0, location = 0;
  size_t es = 0;
  // regular: spatial part of RegularSimplicialMesh(local, offset, global) and
  // the array dims of one timestep
  uint64_t ld[3] = {0, 0, 0}, off[3] = {0, 0, 0}, gd[3] = {0, 0, 0}, adims[3] = {0, 0, 0};
  // extruded: the base mesh (cells copied at open)
  ftk2b_mesh_desc emesh;
  std::vector<uint64_t> ecells;
  uint64_t ebase_hash = 0;     // content hash of ecells (computed once)

  uint64_t T = 0;              // timesteps pushed
  size_t slice_elems = 0;      // elements of one timestep in one ring array
  ftk2b::DevBuf ring[3];       // two-slot rings: timestep t in slot t & 1

  // feature store; stream ids = order of discovery
  unsigned n = 0, cap = 0;
  ftk2b::DevBuf key, hi, lo, phase, lam, bary4, scalar, cls, parent;
  // star edges as stream-id pairs
  unsigned n_edges = 0, edge_cap = 0;
  ftk2b::DevBuf edges;
  // stream ids of the spatial features of the newest layer (the faces that the
  // next slab's top cells share with this one)
  unsigned n_prev = 0;
  ftk2b::DevBuf prev_ids, prev_ids2;
  unsigned n_first = 0;        // features of the first push (classified at the second)
  // per-push scratch
  ftk2b::DevBuf s_key, s_key2, s_id, s_id2, s_hi, s_lo, s_phase, wedges, tmp_simp, dummy;

  double last_ms = 0;
  unsigned last_new = 0;
};

namespace ftk2b {

// grow a device buffer keeping its first `used` bytes
cudaError_t grow_keep(DevBuf& b, size_t used, size_t want, cudaStream_t st);
// grows the feature store (and union-find / boundary lists) to hold `want`
ftk2b_status ensure_stream_store(ftk2b_stream* s, unsigned want);
// content hash of an extruded mesh's base cells (the prepared-mesh cache key)
uint64_t hash_base_cells(const uint64_t* p, uint64_t n);

}  // namespace ftk2b

// extruded streams (cp_extruded.cu)
ftk2b_status stream_push_extruded(ftk2b_stream* s);
ftk2b_status stream_result_extruded(ftk2b_stream* s, ftk2b_cp_result** out);
