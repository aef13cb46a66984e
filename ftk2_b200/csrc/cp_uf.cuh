// Lock-free union-find on feature indices.  Links always go from a larger
// root to a smaller one, so every component's root is its smallest index:
// the reference's UnionFind with min-root linking (engine.hpp:46-74), whose
// find() after all unions is the canonical id of the component minimum.
#pragma once

#include <cuda_runtime.h>

namespace ftk2b {

__device__ __forceinline__ unsigned uf_root(unsigned* parent, unsigned x) {
  // follow parents to the root, halving the path on the way; parents only
  // ever decrease, so the halving writes (atomicMin) never undo a hook
  unsigned p = __ldcg(&parent[x]);
  while (p != x) {
    const unsigned gp = __ldcg(&parent[p]);
    if (gp < p) atomicMin(&parent[x], gp);
    x = p;
    p = gp;
  }
  return x;
}

// Joins the components of a and b.  Every retry follows a successful hook by
// another thread and links only go to smaller indices, so this terminates;
// the iteration bound is a safety net that raises bit 0 of *err.
__device__ __forceinline__ void uf_unite(unsigned* parent, unsigned a, unsigned b, unsigned* err) {
  int it = 0;
  for (; it < (1 << 20); ++it) {
    const unsigned ra = uf_root(parent, a), rb = uf_root(parent, b);
    if (ra == rb) return;
    const unsigned lo = min(ra, rb), hi = max(ra, rb);
    if (atomicCAS(&parent[hi], hi, lo) == hi) return;
    a = ra;
    b = rb;
  }
  atomicOr(err, 1u);
}

}  // namespace ftk2b
