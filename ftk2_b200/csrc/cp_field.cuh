// Value access of the regular-mesh kernels (engine.hpp:999-1009 for separate
// arrays indexed by global - offset, 1101-1124 for multicomponent arrays at
// global coordinates, per-vertex arrays by vertex id).
#pragma once

#include "cp_internal.h"

namespace ftk2b {

template <typename T>
__device__ __forceinline__ T field_at(const FieldAccess& fa, int j, const long long g[4], int d,
                                      unsigned long long vid) {
  // a select instead of an index into the parameter array: an index that
  // differs across lanes would copy the array to local memory
  const T* base = static_cast<const T*>(j == 0 ? fa.comp[0] : (j == 1 ? fa.comp[1] : fa.comp[2]));
  if (fa.per_vertex) return base[vid];
  long long o = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < d) {
      long long a = g[k] - fa.shift[k];
      if (k == d - 1) a ^= fa.tflip;
      o += a * fa.estride[k];
    }
  return base[o];
}

template <typename T>
__device__ __forceinline__ T scalar_at(const FieldAccess& fa, const long long g[4], int d,
                                       unsigned long long vid) {
  const T* base = static_cast<const T*>(fa.scalar);
  if (fa.scalar_per_vertex) return base[vid];
  long long o = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < d) o += g[k] * fa.sstride[k];
  return base[o];
}

}  // namespace ftk2b
