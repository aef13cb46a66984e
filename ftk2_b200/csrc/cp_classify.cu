// Critical-point classification on regular meshes (no counterpart in the
// reference, which stores type = 0 for every feature: predicate.hpp:80, 119).
//
// For every feature, in canonical order: its first coface top cell (the
// prepended / lower-axis-first one of the two Kuhn cofaces of a codimension-1
// simplex), the field values at that cell's d+1 vertices, and the spatial
// Jacobian of the linear interpolant on it: along the chain of the cell each
// step adds one axis, so d v / d x_a = v(after the step along a) - v(before),
// in grid units and in the field precision.  The time column is dropped.  A
// feature without a coface top cell (a mesh one vertex thick along the axis
// its simplex lacks) is reported degenerate.
#include "cp_classify.cuh"
#include "cp_device.cuh"
#include "cp_field.cuh"
#include "cp_kuhn.cuh"
#include "cp_post.h"

namespace ftk2b {

template <typename T, int D>
__global__ void classify_regular_kernel(RegularMesh mesh, FieldAccess fa,
                                        const unsigned long long* __restrict__ simplices,
                                        const unsigned* n_ptr, unsigned cap, unsigned* __restrict__ cls) {
  constexpr int M = D - 1;
  const unsigned n = min(*n_ptr, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned long long v[M + 1];
#pragma unroll
    for (int k = 0; k <= M; ++k) v[k] = simplices[(size_t)i * (M + 1) + k];
    Decoded dc;
    decode_vertices(mesh, v, M, dc);
    long long cc[2][4];
    int cm[2][5];
    const int nc = top_cells(mesh, dc, cc, cm);
    if (nc == 0) {
      cls[i] = FTK2B_CLASS_DEGENERATE;
      continue;
    }
    T val[D + 1][M];
#pragma unroll
    for (int r = 0; r <= D; ++r) {
      long long g[4] = {0, 0, 0, 0};
      unsigned long long vid = 0;
#pragma unroll
      for (int k = 0; k < D; ++k) {
        g[k] = cc[0][k] + ((cm[0][r] >> k) & 1);
        vid += (unsigned long long)g[k] * mesh.gstride[k];
      }
#pragma unroll
      for (int j = 0; j < M; ++j) val[r][j] = field_at<T>(fa, j, g, D, vid);
    }
    T J[M][M];
#pragma unroll
    for (int r = 1; r <= D; ++r) {
      const int axis = __ffs(cm[0][r] ^ cm[0][r - 1]) - 1;
#pragma unroll
      for (int a = 0; a < M; ++a)
        if (axis == a)
#pragma unroll
          for (int j = 0; j < M; ++j) J[j][a] = fp<T>::sub(val[r][j], val[r - 1][j]);
    }
    cls[i] = classify_jacobian<M, T>(J);
  }
}

cudaError_t launch_classify_regular(int f64, const RegularMesh& mesh, const FieldAccess& fa, int nch,
                                    const PostBuffers& B, cudaStream_t st) {
  (void)nch;
  int g = (int)((B.cap + 255) / 256);
  if (g < 1) g = 1;
  if (g > 4096) g = 4096;
  if (mesh.d == 4) {
    if (f64) classify_regular_kernel<double, 4><<<g, 256, 0, st>>>(mesh, fa, B.simplices, B.count, B.cap, B.cls);
    else classify_regular_kernel<float, 4><<<g, 256, 0, st>>>(mesh, fa, B.simplices, B.count, B.cap, B.cls);
  } else {
    if (f64) classify_regular_kernel<double, 3><<<g, 256, 0, st>>>(mesh, fa, B.simplices, B.count, B.cap, B.cls);
    else classify_regular_kernel<float, 3><<<g, 256, 0, st>>>(mesh, fa, B.simplices, B.count, B.cap, B.cls);
  }
  return cudaGetLastError();
}

}  // namespace ftk2b
