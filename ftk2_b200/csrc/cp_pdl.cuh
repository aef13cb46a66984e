// Programmatic dependent launch between consecutive kernels of a pipeline:
// a kernel launched with launch_pdl may be scheduled while its predecessor
// finishes; it waits (griddepcontrol.wait, its first statement) until the
// predecessor grid has completed and its memory is visible, then lets its
// own successor be scheduled.  Kernels launched the ordinary way execute the
// same two instructions as no-ops.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace ftk2b {

__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace ftk2b
