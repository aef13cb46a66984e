"""Critical-point extraction of one regular spacetime field split into time
slabs, one slab per GPU (or one after another on one GPU), combined into the
result of the whole mesh.

Slab k covers timesteps [t_k, t_{k+1}] of the global mesh (consecutive slabs
share one timestep) and is extracted as RegularSimplicialMesh(local, offset,
global) with offset t_k (mesh.hpp:256-265), so vertex ids stay global.  Every
Kuhn simplex spans at most one time step and every top cell exactly one, so:

- the features of the whole mesh are the union of the slabs' features; the
  purely spatial simplices of a shared timestep t_{k+1} appear in slabs k and
  k + 1 with the same values, hence the same barycentrics;
- vertex ids grow with time, so in the canonical (Simplex) order every
  feature of slab k whose lowest vertex lies before t_{k+1} precedes every
  feature of slab k + 1, and the features of slab k whose lowest vertex lies
  on t_{k+1} -- exactly the shared spatial ones -- are a suffix of slab k's
  list.  Slab k owns its features but that suffix, and the global index of
  an owned feature is the slab's offset (the owned counts of the slabs
  before it) plus its local index;
- star edges are the union of the slabs' edges (each top cell, with its star
  centre, lies in one slab);
- trajectories join the slabs' trajectories through the shared features.

The exchange step (collectives only, no field data): all-gather of the
per-slab counts, then of three short lists per slab -- the global indices of
its features on its first timestep, the global indices of the local track
roots of those features, and the roots of its shared suffix.  Every rank
then unites, for each shared feature, its root in slab k with its root in
slab k + 1 (a union-find over the interface only, min-root linking) and
relabels its own features: the track id is the component's smallest global
index, as in a one-GPU call (engine.hpp:46-74, 822-996).  Over NCCL the
lists travel as device tensors; over gloo (CPU tests) as host tensors.
"""
from __future__ import annotations

from dataclasses import dataclass
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


@dataclass
class ShardResult:
    """The features a slab owns, in canonical order, with global indices:
    feature i of this shard is global feature `offset + i`."""
    offset: int
    simplices: np.ndarray
    lam: np.ndarray
    bary: np.ndarray
    track_id: np.ndarray       # global: the component's smallest global index
    type: np.ndarray
    cp_class: Optional[np.ndarray]
    scalar: np.ndarray
    edges: np.ndarray          # (e, 2) global indices of this slab's star edges, rows sorted
    n_simplices: int = 0
    device_ms: float = 0.0


def _layout(part, t0: int, t1: int, first: bool, last: bool, tstride: int):
    """(shared suffix length, local indices of the features on timestep t0)."""
    s = part.simplices
    n = len(part.track_id)
    if n == 0:
        return 0, np.zeros(0, np.int64)
    s_up = 0 if last else int(np.count_nonzero(s[:, 0] // tstride == t1))
    if s_up and not np.all(s[n - s_up:, 0] // tstride == t1):
        raise RuntimeError("shared features are not a suffix of the slab's canonical order")
    lo_idx = np.zeros(0, np.int64) if first else np.nonzero(s[:, -1] // tstride == t0)[0].astype(np.int64)
    return s_up, lo_idx


def _interface_roots(pairs_up: Sequence[np.ndarray], pairs_lo: Sequence[np.ndarray]):
    """Union-find over interface roots: up[k][j] (root in slab k of shared
    feature j of the k / k+1 interface) meets lo[k+1][j].  Returns (keys,
    final) arrays: final[i] is the smallest global index joined to keys[i]."""
    a = np.concatenate([np.asarray(u, np.int64) for u in pairs_up] + [np.zeros(0, np.int64)])
    b = np.concatenate([np.asarray(v, np.int64) for v in pairs_lo] + [np.zeros(0, np.int64)])
    keys = np.unique(np.concatenate([a, b]))
    parent = np.arange(len(keys))
    ia, ib = np.searchsorted(keys, a), np.searchsorted(keys, b)

    def find(x):
        r = x
        while parent[r] != r:
            r = parent[r]
        while parent[x] != r:
            parent[x], x = r, parent[x]
        return r

    for x, y in zip(ia.tolist(), ib.tolist()):
        rx, ry = find(x), find(y)
        if rx != ry:  # keys are sorted, so the smaller position is the smaller global index
            parent[max(rx, ry)] = min(rx, ry)
    final = keys[[find(i) for i in range(len(keys))]] if len(keys) else keys
    return keys, final


def _relabel(root_g: np.ndarray, keys: np.ndarray, final: np.ndarray) -> np.ndarray:
    out = root_g.astype(np.int64).copy()
    if len(keys) and len(out):
        pos = np.searchsorted(keys, out)
        hit = (pos < len(keys)) & (keys[np.minimum(pos, len(keys) - 1)] == out)
        out[hit] = final[pos[hit]]
    return out.astype(np.uint64)


def _shard(part, offset: int, own: int, gidx: np.ndarray, track_g: np.ndarray) -> ShardResult:
    e = part.edges.astype(np.int64)
    E = np.sort(gidx[e], axis=1).astype(np.uint32) if len(e) else np.zeros((0, 2), np.uint32)
    cls = getattr(part, "cp_class", None)
    return ShardResult(offset=offset, simplices=part.simplices[:own], lam=part.lam[:own], bary=part.bary[:own],
                       track_id=track_g[:own], type=part.type[:own], cp_class=None if cls is None else cls[:own],
                       scalar=part.scalar[:own], edges=E, n_simplices=int(getattr(part, "n_simplices", 0)),
                       device_ms=float(getattr(part, "device_ms", 0.0)))


def assemble(shards: Sequence[ShardResult]) -> api.CPResult:
    """The whole mesh's result from every shard (in slab order)."""
    cat = lambda a: np.concatenate([getattr(s, a) for s in shards], axis=0)  # noqa: E731
    ed = [s.edges for s in shards if len(s.edges)]
    E = np.unique(np.concatenate(ed, axis=0), axis=0).astype(np.uint32) if ed else np.zeros((0, 2), np.uint32)
    track = cat("track_id")
    cls = None if any(s.cp_class is None for s in shards) else cat("cp_class")
    return api.CPResult(simplices=cat("simplices"), lam=cat("lam"), bary=cat("bary"), track_id=track,
                        type=cat("type"), cp_class=cls, scalar=cat("scalar"), edges=E,
                        n_tracks=int(len(np.unique(track))), n_simplices=int(sum(s.n_simplices for s in shards)),
                        device_ms=float(max([s.device_ms for s in shards] or [0.0])))


def combine(parts: Sequence, bounds: Sequence[tuple], global_dims: Sequence[int]) -> List[ShardResult]:
    """The exchange of extract_sharded, in one process: slab results (local
    canonical order) -> the shards with global indices and tracks."""
    tstride = int(np.prod(global_dims[:-1]))
    K = len(parts)
    lay = [_layout(p, t0, t1, k == 0, k == K - 1, tstride) for k, (p, (t0, t1)) in enumerate(zip(parts, bounds))]
    own = [len(p.track_id) - s for p, (s, _) in zip(parts, lay)]
    offs = np.concatenate([[0], np.cumsum(own)]).astype(np.int64)
    lo_g = [offs[k] + lay[k][1] for k in range(K)]
    gidx, root_g = [], []
    for k, p in enumerate(parts):
        g = np.empty(len(p.track_id), np.int64)
        g[:own[k]] = offs[k] + np.arange(own[k])
        if k + 1 < K:
            g[own[k]:] = lo_g[k + 1]
        gidx.append(g)
        root_g.append(g[p.track_id.astype(np.int64)])
    up_r = [root_g[k][own[k]:] for k in range(K)]
    lo_r = [root_g[k][lay[k][1]] for k in range(K)]
    keys, final = _interface_roots(up_r[:-1], lo_r[1:])
    return [_shard(p, int(offs[k]), own[k], gidx[k], _relabel(root_g[k], keys, final)) for k, p in enumerate(parts)]


def merge(parts: Sequence, bounds: Sequence[tuple], global_dims: Sequence[int]) -> api.CPResult:
    return assemble(combine(parts, bounds, global_dims))


def extract_local(ctx: api.Context, global_dims: Sequence[int], field, ncomp: int, n_shards: int,
                  prm: Optional[api.CPParams] = None, layout: int = api.LAYOUT_MULTICOMPONENT) -> api.CPResult:
    """All slabs one after another on this context's GPU, combined: equal to
    ctx.extract on the whole mesh."""
    keep: list = []
    fd = api.field_desc(field, layout, ncomp, keep=keep)
    bounds = slab_bounds(int(global_dims[-1]), n_shards)
    parts = [ctx.extract(slab_mesh(global_dims, t0, t1), fd, prm) for t0, t1 in bounds]
    return merge(parts, bounds, global_dims)


def _allgather_var(dist, group, arr: np.ndarray, lengths: Sequence[int], device) -> List[np.ndarray]:
    """All-gather of one int64 list per rank (lengths known to every rank)."""
    import torch
    world = len(lengths)
    m = max(1, max(lengths))
    buf = torch.full((m,), -1, dtype=torch.int64, device=device)
    if len(arr):
        buf[:len(arr)] = torch.as_tensor(np.asarray(arr, np.int64), device=device)
    out = [torch.empty((m,), dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    return [o[:n].cpu().numpy() for o, n in zip(out, lengths)]


def extract_sharded(global_dims: Sequence[int], field, ncomp: int, prm: Optional[api.CPParams] = None,
                    layout: int = api.LAYOUT_MULTICOMPONENT, group=None,
                    extractor: Optional[Callable] = None) -> ShardResult:
    """One slab per rank of the process group; returns this rank's shard with
    global indices and track ids.  The field stays in each rank's own memory;
    only counts and interface lists cross ranks.  extractor(mesh_desc, t0, t1)
    -> result replaces the rank's GPU extraction (CPU tests)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    dims = list(global_dims)
    bounds = slab_bounds(int(dims[-1]), world)
    K = len(bounds)
    tstride = int(np.prod(dims[:-1]))
    part = None
    if rank < K:
        t0, t1 = bounds[rank]
        mesh = slab_mesh(dims, t0, t1)
        if extractor is not None:
            part = extractor(mesh, t0, t1)
        else:
            keep: list = []
            with api.Context(_local_device()) as ctx:
                part = ctx.extract(mesh, api.field_desc(field, layout, ncomp, keep=keep), prm)
        s_up, lo_idx = _layout(part, t0, t1, rank == 0, rank == K - 1, tstride)
        n = len(part.track_id)
    else:
        s_up, lo_idx, n = 0, np.zeros(0, np.int64), 0
    # 1. counts: (features, shared suffix, features on the first timestep)
    cnt = torch.tensor([n, s_up, len(lo_idx)], dtype=torch.int64, device=device)
    allc = [torch.empty(3, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(allc, cnt, group=group)
    C = np.stack([c.cpu().numpy() for c in allc])
    own = C[:, 0] - C[:, 1]
    offs = np.concatenate([[0], np.cumsum(own)]).astype(np.int64)
    if rank + 1 < K and C[rank, 1] != C[rank + 1, 2]:
        raise RuntimeError("slabs disagree on their shared timestep's features")
    # 2. global indices of every slab's first-timestep features
    LOG = _allgather_var(dist, group, offs[rank] + lo_idx, C[:, 2].tolist(), device)
    gidx = np.empty(n, np.int64)
    gidx[:own[rank]] = offs[rank] + np.arange(own[rank])
    if rank + 1 < K:
        gidx[own[rank]:] = LOG[rank + 1]
    root_g = gidx[part.track_id.astype(np.int64)] if n else np.zeros(0, np.int64)
    # 3. interface roots
    UPR = _allgather_var(dist, group, root_g[own[rank]:], C[:, 1].tolist(), device)
    LOR = _allgather_var(dist, group, root_g[lo_idx] if n else np.zeros(0, np.int64), C[:, 2].tolist(), device)
    keys, final = _interface_roots(UPR[:K - 1], LOR[1:K])
    if part is None:
        z = np.zeros(0, np.uint64)
        return ShardResult(offset=int(offs[rank]), simplices=np.zeros((0, len(dims)), np.uint64), lam=np.zeros((0, len(dims))),
                           bary=np.zeros((0, len(dims)), np.float32), track_id=z, type=np.zeros(0, np.uint32),
                           cp_class=None, scalar=np.zeros(0, np.float32), edges=np.zeros((0, 2), np.uint32))
    return _shard(part, int(offs[rank]), int(own[rank]), gidx, _relabel(root_g, keys, final))


def extract_distributed(global_dims: Sequence[int], field, ncomp: int, prm: Optional[api.CPParams] = None,
                        layout: int = api.LAYOUT_MULTICOMPONENT, group=None,
                        extractor: Optional[Callable] = None):
    """extract_sharded, then the shards gathered to rank 0, which returns the
    whole mesh's result (the other ranks return None)."""
    import torch.distributed as dist
    mine = extract_sharded(global_dims, field, ncomp, prm, layout, group, extractor)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0, group=group)
    if rank != 0:
        return None
    return assemble([g for g in gathered if g is not None])


def _local_device() -> int:
    import os
    return int(os.environ.get("LOCAL_RANK", "0"))
