// Geometry of the Freudenthal/Kuhn triangulation of a regular spacetime
// grid shared by the post-extraction kernels: a simplex as its corner plus the
// vertex masks of its chain (mesh.hpp:105-302), and the top cells (cofaces)
// of a codimension-1 simplex.
#pragma once

#include "cp_internal.h"

namespace ftk2b {

struct Decoded {
  long long g[4];  // global coords of the corner
  int mk[5];       // masks of the m+1 vertices (mk[0] = 0)
};

// Cofaces (top cells) of the feature's simplex inside the local box, each as
// corner + d+1 vertex masks.  A codimension-1 simplex of a Kuhn triangulation
// has exactly two: if one axis a never steps, prepend (corner - e_a) or append
// (full mask); otherwise split the one two-axis step in either order.
static __device__ int top_cells(const RegularMesh& mesh, const Decoded& dc, long long cc[2][4],
                         int cm[2][5]) {
  const int d = mesh.d, m = d - 1, full = (1 << d) - 1;
  int nc = 0;
  const int missing = full & ~dc.mk[m];
  if (missing) {
    const int a = __ffs(missing) - 1;
    if (dc.g[a] - mesh.off[a] >= 1) {
      for (int k = 0; k < 4; ++k) cc[nc][k] = dc.g[k];
      cc[nc][a] -= 1;
      cm[nc][0] = 0;
      for (int j = 0; j <= m; ++j) cm[nc][j + 1] = dc.mk[j] | (1 << a);
      ++nc;
    }
    if (dc.g[a] - mesh.off[a] + 1 < mesh.ld[a]) {
      for (int k = 0; k < 4; ++k) cc[nc][k] = dc.g[k];
      for (int j = 0; j <= m; ++j) cm[nc][j] = dc.mk[j];
      cm[nc][m + 1] = full;
      ++nc;
    }
  } else {
    for (int j = 1; j <= m; ++j) {
      const int step = dc.mk[j] & ~dc.mk[j - 1];
      if (__popc(step) == 2) {
        const int lo = step & -step, hi = step & ~lo;
        const int ins[2] = {lo, hi};
        for (int q = 0; q < 2; ++q) {
          for (int k = 0; k < 4; ++k) cc[nc][k] = dc.g[k];
          int w = 0;
          for (int jj = 0; jj <= m; ++jj) {
            if (jj == j) cm[nc][w++] = dc.mk[j - 1] | ins[q];
            cm[nc][w++] = dc.mk[jj];
          }
          ++nc;
        }
        break;
      }
    }
  }
  return nc;
}

// Corner and masks of a simplex from its ascending vertex ids: the corner is
// the first vertex; every other vertex differs from it by a sum of distinct
// axis strides, peeled off from the largest (an axis of extent 1 never steps,
// so equal strides resolve to the higher axis).
__device__ __forceinline__ void decode_vertices(const RegularMesh& mesh, const unsigned long long* v, int m,
                                                Decoded& dc) {
  unsigned long long v0 = v[0];
  for (int k = 0; k < 4; ++k) dc.g[k] = 0;
  for (int k = 0; k < mesh.d; ++k) {
    dc.g[k] = (long long)(v0 % (unsigned long long)mesh.gd[k]);
    v0 /= (unsigned long long)mesh.gd[k];
  }
  dc.mk[0] = 0;
  for (int j = 1; j <= m; ++j) {
    unsigned long long diff = v[j] - v[0];
    int msk = 0;
    for (int k = mesh.d - 1; k >= 0; --k)
      if (diff >= mesh.gstride[k]) {
        msk |= 1 << k;
        diff -= mesh.gstride[k];
      }
    dc.mk[j] = msk;
  }
}

}  // namespace ftk2b
