// Critical-point classification (placeholder until the classifier lands).
#include "cp_post.h"

namespace ftk2b {

__global__ void classify_none_kernel(unsigned* cls, const unsigned* n_ptr, unsigned cap) {
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) cls[i] = 0;
}

cudaError_t launch_classify_regular(int f64, const RegularMesh& mesh, const FieldAccess& fa, int nch,
                                    const PostBuffers& B, cudaStream_t st) {
  (void)f64; (void)mesh; (void)fa; (void)nch;
  classify_none_kernel<<<64, 256, 0, st>>>(B.cls, B.count, B.cap);
  return cudaGetLastError();
}

}  // namespace ftk2b
