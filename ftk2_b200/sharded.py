"""Critical-point extraction of one regular spacetime field split into time
slabs, one slab per GPU (or one after another on one GPU), merged into the
result of the whole mesh.

Slab k covers timesteps [t_k, t_{k+1}] of the global mesh (consecutive slabs
share one timestep) and is extracted as RegularSimplicialMesh(local, offset,
global) with offset t_k (mesh.hpp:256-265), so vertex ids stay global.  Every
Kuhn simplex spans at most one time step and every top cell exactly one, so:

- the features of the whole mesh are the union of the slabs' features (the
  purely spatial simplices of a shared timestep appear in both slabs with the
  same values, hence the same barycentrics);
- its star edges are the union of the slabs' edges (each top cell, with its
  star centre, lies in one slab);
- its trajectories join the slabs' trajectories through the shared features
  (each slab's tracks already hold its edges and, on 3D+t meshes, its coface
  unions; get_complex, engine.hpp:822-996).

The merge is the one exchange step: each rank's result goes to rank 0 (one
gather), which orders the features, remaps the edges and unites the tracks.
Track ids are the component's smallest feature index, as in a one-GPU call.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np

from . import api


def slab_bounds(nt: int, n: int) -> List[tuple]:
    """n time slabs [t0, t1] (inclusive) over nt timesteps, consecutive slabs
    sharing one timestep; fewer when nt - 1 < n."""
    n = max(1, min(n, nt - 1))
    cuts = [round(i * (nt - 1) / n) for i in range(n + 1)]
    return [(cuts[i], cuts[i + 1]) for i in range(n)]


def slab_mesh(global_dims: Sequence[int], t0: int, t1: int) -> api.MeshDesc:
    d = len(global_dims)
    local = list(global_dims[:-1]) + [t1 - t0 + 1]
    offset = [0] * (d - 1) + [t0]
    return api.regular_mesh_desc(local, offset, list(global_dims))


def merge(parts: Sequence) -> api.CPResult:
    """One result from the slab results (CPResult-like: simplices, lam, bary,
    track_id, type, cp_class, scalar, edges)."""
    parts = [p for p in parts if p is not None]
    k = parts[0].simplices.shape[1] if parts else 1
    rows = [p.simplices.reshape(-1, k) for p in parts]
    allrows = np.concatenate(rows, axis=0) if rows else np.zeros((0, k), np.uint64)
    uniq, first, inv = np.unique(allrows, axis=0, return_index=True, return_inverse=True)
    inv = inv.reshape(-1)
    n = len(uniq)
    # per-slab local index -> global index
    starts = np.cumsum([0] + [len(r) for r in rows])
    glob = [inv[starts[i]:starts[i + 1]] for i in range(len(rows))]

    def take(attr, width=None):
        arrs = [getattr(p, attr) for p in parts]
        if any(a is None for a in arrs):
            return None
        cat = np.concatenate(arrs, axis=0)
        return cat[first]

    # union-find over the global indices: every slab feature joins its slab root
    parent = np.arange(n, dtype=np.int64)

    def find(x):
        root = x
        while parent[root] != root:
            root = parent[root]
        while parent[x] != root:
            parent[x], x = root, parent[x]
        return root

    for p, g in zip(parts, glob):
        roots = g[p.track_id.astype(np.int64)]
        for a, b in zip(g.tolist(), roots.tolist()):
            ra, rb = find(a), find(b)
            if ra != rb:
                lo, hi = (ra, rb) if ra < rb else (rb, ra)
                parent[hi] = lo
    track = np.array([find(i) for i in range(n)], dtype=np.uint64)
    edges = []
    for p, g in zip(parts, glob):
        if len(p.edges):
            e = g[p.edges.astype(np.int64)]
            edges.append(np.sort(e, axis=1))
    E = np.unique(np.concatenate(edges, axis=0), axis=0).astype(np.uint32) if edges else np.zeros((0, 2), np.uint32)
    return api.CPResult(
        simplices=uniq.astype(np.uint64), lam=take("lam"), bary=take("bary"), track_id=track,
        type=take("type"), cp_class=take("cp_class"), scalar=take("scalar"), edges=E,
        n_tracks=int(len(np.unique(track))), n_simplices=int(sum(p.n_simplices for p in parts)),
        device_ms=float(max([p.device_ms for p in parts] or [0.0])))


def extract_local(ctx: api.Context, global_dims: Sequence[int], field, ncomp: int, n_shards: int,
                  prm: Optional[api.CPParams] = None, layout: int = api.LAYOUT_MULTICOMPONENT) -> api.CPResult:
    """All slabs one after another on this context's GPU, merged: equal to
    ctx.extract on the whole mesh."""
    keep: list = []
    fd = api.field_desc(field, layout, ncomp, keep=keep)
    parts = [ctx.extract(slab_mesh(global_dims, t0, t1), fd, prm)
             for t0, t1 in slab_bounds(int(global_dims[-1]), n_shards)]
    return merge(parts)


def extract_distributed(global_dims: Sequence[int], field, ncomp: int, prm: Optional[api.CPParams] = None,
                        layout: int = api.LAYOUT_MULTICOMPONENT, group=None,
                        extractor: Optional[Callable] = None):
    """One slab per rank of the default process group (torch.distributed);
    rank 0 gathers the slab results and returns the merged result, the other
    ranks return None.  extractor(mesh_desc, t0, t1) -> result replaces the
    rank's GPU extraction (tests run the merge on CPU ranks with it)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    bounds = slab_bounds(int(global_dims[-1]), world)
    mine = None
    if rank < len(bounds):
        t0, t1 = bounds[rank]
        mesh = slab_mesh(global_dims, t0, t1)
        if extractor is not None:
            mine = extractor(mesh, t0, t1)
        else:
            keep: list = []
            with api.Context(_local_device()) as ctx:
                mine = ctx.extract(mesh, api.field_desc(field, layout, ncomp, keep=keep), prm)
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0, group=group)
    if rank != 0:
        return None
    return merge([g for g in gathered if g is not None])


def _local_device() -> int:
    import os
    return int(os.environ.get("LOCAL_RANK", "0"))
