// Extruded unstructured meshes (placeholder until the kernels land).
#include "cp_api_internal.h"

ftk2b_status run_extruded(ftk2b_ctx* ctx, const ftk2b_mesh_desc*, const ftk2b_field_desc*,
                          const ftk2b_cp_params*) {
  ctx->err = "extruded meshes are not implemented yet";
  return FTK2B_UNSUPPORTED;
}

uint64_t extruded_simplex_count(const ftk2b_mesh_desc*, int) { return 0; }
