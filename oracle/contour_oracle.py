"""Restatement of the reference's level-set path in numpy (TEST INFRASTRUCTURE
ONLY: tests/ and the smoke check import it as a checker; the product never
does).  contour() covers regular meshes, contour_extruded() extruded ones.

SimplicialEngine<T, ContourPredicate<T>> on a RegularSimplicialMesh, execute()
then get_complex():

- nodes (engine.hpp:120-160): every mesh edge whose endpoints have different
  simulation-of-simplicity signs of value - threshold (sos.hpp:12-20,
  origin_inside<1> at sos.hpp:211-220).  The sign quantises in double,
  v*Q + (v > 0 ? 0.5 : -0.5), truncates to an integer and breaks a zero by the
  parity of the vertex id.  Every edge of the Freudenthal mesh joins a vertex
  c to c + e with e in {0,1}^d, so the edges sorted by (lower id, upper id)
  are the pairs (c, e) sorted by c's id and then by e read as a binary number
  with x the lowest bit.
- barycentrics (predicate.hpp:145-153, zero_crossing.hpp:93-104): d = v0 - v1;
  lambda0 = -v1 / d, lambda1 = 1 - lambda0 in the field precision; both 0.5
  when |d| < 1e-12 or lambda0 leaves [-1e-9, 1 + 1e-9].
- manifold cells (engine.hpp:165-181, marching_pentatope 1210-1279,
  marching_tetrahedron 1281-1339): for every Kuhn d-simplex of every
  hypercube (visited in the CPU mesh's permutation order, mesh.hpp:403-414),
  the vertices split into positive (A) and other (B) sets.  On 2D+t
  meshes a 1-3 split gives the triangle of the three crossing edges at the
  lone vertex; a 2-2 split gives the quad of the four crossing edges, cut into
  (n0, n1, n2) and (n0, n2, n3) of its sorted node indices.  On 3D+t meshes a
  1-4 split gives one tet; a 2-3 split, with T0 / T1 the crossing edges of the
  pair's first / second vertex to the triple in order, gives the tets
  {T0[0],T0[1],T0[2],T1[2]}, {T0[0],T0[1],T1[1],T1[2]}, {T0[0],T1[0],T1[1],T1[2]}.
- get_complex (engine.hpp:822-996, complex.hpp:27-57): cells sorted within and
  among themselves and made unique; every cell's first node is united with its
  others; the track id is the component's root, the smallest feature index
  (min-root union-find); vertices stay in simplex order.
"""
from __future__ import annotations

import itertools

import numpy as np


def sos_positive(adj: np.ndarray, gid: np.ndarray, q: float) -> np.ndarray:
    """sos::sign(v, id, Q) > 0 for the adjusted values (any float dtype)."""
    v = adj.astype(np.float64)
    x = v * q + np.where(adj > 0, 0.5, -0.5)
    pos = x >= 1.0
    neg = x <= -1.0
    tie = ~pos & ~neg
    return pos | (tie & (gid % 2 == 0))


def contour(field: np.ndarray, threshold: float, local_dims, offset=None, global_dims=None, q: float = 1e6):
    """field: C-order array of reversed Fortran shape (the local mesh's values,
    or a larger array indexed by local coordinates).  Returns a dict with
    simplices (n, 2) uint64, lam (n, 2) float64, bary (n, 2) float32,
    track_id (n,) uint64, scalar (n,) float32 and cells (c, d) uint32."""
    d = len(local_dims)
    T = field.dtype.type
    offset = list(offset) if offset is not None else [0] * d
    global_dims = list(global_dims) if global_dims is not None else list(local_dims)
    gs = [1] * d
    for i in range(1, d):
        gs[i] = gs[i - 1] * int(global_dims[i - 1])
    shape = tuple(int(n) for n in local_dims[::-1])
    vals = field[tuple(slice(0, n) for n in shape)]
    adj = (vals - T(threshold)).astype(T)
    grids = np.meshgrid(*[np.arange(int(n), dtype=np.uint64) for n in local_dims[::-1]], indexing="ij")
    coords = grids[::-1]  # coords[i] = axis i (x first), each of C shape
    gid = np.zeros(shape, dtype=np.uint64)
    for i in range(d):
        gid += (coords[i] + np.uint64(offset[i])) * np.uint64(gs[i])
    pos = sos_positive(adj, gid, q)

    # nodes: (vertex, direction) pairs with differing signs
    nv = int(np.prod(shape))
    lin = np.arange(nv, dtype=np.int64).reshape(shape)
    masks = np.zeros(shape, dtype=np.int64)
    for e in range(1, 1 << d):
        lo = [slice(None)] * d
        hi = [slice(None)] * d
        for i in range(d):
            ax = d - 1 - i
            if (e >> i) & 1:
                lo[ax] = slice(0, shape[ax] - 1)
                hi[ax] = slice(1, shape[ax])
        diff = pos[tuple(lo)] != pos[tuple(hi)]
        sub = masks[tuple(lo)]
        sub |= diff.astype(np.int64) << (e - 1)
        masks[tuple(lo)] = sub
    flat_mask = masks.reshape(-1)
    counts = _popcount(flat_mask)
    voff = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    n = int(counts.sum())
    verts = np.nonzero(flat_mask)[0]
    rows_v, rows_e = [], []
    for e in range(1, 1 << d):
        sel = verts[(flat_mask[verts] >> (e - 1)) & 1 == 1]
        rows_v.append(sel)
        rows_e.append(np.full(sel.size, e, dtype=np.int64))
    rv = np.concatenate(rows_v) if rows_v else np.zeros(0, np.int64)
    re_ = np.concatenate(rows_e) if rows_e else np.zeros(0, np.int64)
    order = np.lexsort((re_, rv))
    rv, re_ = rv[order], re_[order]
    lstride = [1] * d
    for i in range(1, d):
        lstride[i] = lstride[i - 1] * int(local_dims[i - 1])
    step = np.zeros(1 << d, dtype=np.int64)
    gstep = np.zeros(1 << d, dtype=np.uint64)
    for e in range(1 << d):
        step[e] = sum(lstride[i] for i in range(d) if (e >> i) & 1)
        gstep[e] = sum(gs[i] for i in range(d) if (e >> i) & 1)
    flat_gid = gid.reshape(-1)
    flat_adj = adj.reshape(-1)
    g0 = flat_gid[rv]
    simplices = np.stack([g0, g0 + gstep[re_]], axis=1).astype(np.uint64)
    a0 = flat_adj[rv]
    a1 = flat_adj[rv + step[re_]]
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        dd = (a0 - a1).astype(T)
        l0 = (-a1 / dd).astype(T)
        l1 = (T(1.0) - l0).astype(T)
    eps = T(1e-9)
    ok = (np.abs(dd) >= T(1e-12)) & (l0 >= -eps) & (l0 <= T(1.0) + eps)
    l0 = np.where(ok, l0, T(0.5)).astype(T)
    l1 = np.where(ok, l1, T(0.5)).astype(T)
    lam = np.stack([l0.astype(np.float64), l1.astype(np.float64)], axis=1)
    bary = np.stack([l0.astype(np.float32), l1.astype(np.float32)], axis=1)

    def node(a_lin, e):
        m = flat_mask[a_lin]
        below = m & ((np.int64(1) << (e - 1)) - 1)
        return voff[a_lin] + _popcount(below)

    # manifold cells over every Kuhn simplex of every hypercube
    cube_shape = tuple(s - 1 for s in shape)
    if min(cube_shape) <= 0:
        cells = np.zeros((0, d), dtype=np.uint32)
    else:
        base = lin[tuple(slice(0, s) for s in cube_shape)].reshape(-1)
        is_base = np.zeros(shape, dtype=bool)
        is_base[tuple(slice(0, s) for s in cube_shape)] = True
        is_base = is_base.reshape(-1)
        flat_pos = pos.reshape(-1)
        perms = [cpu_perm(i, d) for i in range(int(np.prod(range(1, d + 1))))]

        def tets(perm):
            path_e = [0]
            for ax in perm:
                path_e.append(path_e[-1] | (1 << ax))
            pv = [base + step[e] for e in path_e]
            ps = [flat_pos[v] for v in pv]
            npos = sum(p.astype(np.int64) for p in ps)

            def nd(i, j, sel):
                return node(pv[i][sel], path_e[j] ^ path_e[i])

            def late(i, sel):
                return ~is_base[pv[i][sel]]
            return pv, ps, npos, nd, late

        # 2D+t quads are cut along the diagonal from their node of smallest
        # engine id.  Nodes whose edge starts at a hypercube base got their ids
        # in simplex order in the first pass; the others (edges starting on an
        # upper boundary face) were first met while patching, visiting the
        # hypercubes in vertex order, their Kuhn simplices in permutation
        # order and each simplex's crossing edges in enumeration order.
        order_key = np.arange(n, dtype=np.int64)
        if d == 3 and n:
            first = np.full(n, np.iinfo(np.int64).max, dtype=np.int64)
            for p_idx, perm in enumerate(perms):
                pv, ps, npos, nd, late = tets(perm)
                for lone in range(4):
                    for single_pos in (True, False):
                        s2 = (npos == (1 if single_pos else 3)) & (ps[lone] == single_pos)
                        if not s2.any():
                            continue
                        for k_, o in enumerate(o for o in range(4) if o != lone):
                            i, j = min(lone, o), max(lone, o)
                            lt = late(i, s2)
                            key = (base[s2] * len(perms) + p_idx) * 4 + k_
                            np.minimum.at(first, nd(i, j, s2)[lt], key[lt])
                for A in itertools.combinations(range(4), 2):
                    B = [i for i in range(4) if i not in A]
                    s2 = (npos == 2) & ps[A[0]] & ps[A[1]]
                    if not s2.any():
                        continue
                    for k_, (a, b) in enumerate((a, b) for a in A for b in B):
                        i, j = min(a, b), max(a, b)
                        lt = late(i, s2)
                        key = (base[s2] * len(perms) + p_idx) * 4 + k_
                        np.minimum.at(first, nd(i, j, s2)[lt], key[lt])
            met = first != np.iinfo(np.int64).max
            order_key = np.where(met, n + first, order_key)

        out = []
        for p_idx, perm in enumerate(perms):
            pv, ps, npos, nd, late = tets(perm)
            if d == 3:
                for single_pos in (True, False):
                    sel = npos == (1 if single_pos else 3)
                    if not sel.any():
                        continue
                    for lone in range(4):
                        s2 = sel & (ps[lone] == single_pos)
                        if not s2.any():
                            continue
                        others = [o for o in range(4) if o != lone]
                        tri = [nd(min(lone, o), max(lone, o), s2) for o in others]
                        out.append(np.sort(np.stack(tri, axis=1), axis=1))
                sel = npos == 2
                if sel.any():
                    for A in itertools.combinations(range(4), 2):
                        B = [i for i in range(4) if i not in A]
                        s2 = sel & ps[A[0]] & ps[A[1]]
                        if not s2.any():
                            continue
                        q4 = np.stack([nd(min(a, b), max(a, b), s2) for a in A for b in B], axis=1)
                        q4 = np.take_along_axis(q4, np.argsort(order_key[q4], axis=1), axis=1)
                        out.append(np.sort(q4[:, [0, 1, 2]], axis=1))
                        out.append(np.sort(q4[:, [0, 2, 3]], axis=1))
            else:
                for single_pos in (True, False):
                    sel = npos == (1 if single_pos else 4)
                    if not sel.any():
                        continue
                    for lone in range(5):
                        s2 = sel & (ps[lone] == single_pos)
                        if not s2.any():
                            continue
                        others = [o for o in range(5) if o != lone]
                        tet = [nd(min(lone, o), max(lone, o), s2) for o in others]
                        out.append(np.sort(np.stack(tet, axis=1), axis=1))
                for two_pos in (True, False):
                    sel = npos == (2 if two_pos else 3)
                    if not sel.any():
                        continue
                    for two in itertools.combinations(range(5), 2):
                        three = [i for i in range(5) if i not in two]
                        s2 = sel & (ps[two[0]] == two_pos) & (ps[two[1]] == two_pos)
                        if not s2.any():
                            continue
                        T0 = [nd(min(two[0], t), max(two[0], t), s2) for t in three]
                        T1 = [nd(min(two[1], t), max(two[1], t), s2) for t in three]
                        for c in ((T0[0], T0[1], T0[2], T1[2]), (T0[0], T0[1], T1[1], T1[2]),
                                  (T0[0], T1[0], T1[1], T1[2])):
                            out.append(np.sort(np.stack(c, axis=1), axis=1))
        cells = np.concatenate(out, axis=0) if out else np.zeros((0, d), dtype=np.int64)
        cells = np.unique(cells, axis=0).astype(np.uint32)

    # union-find over each cell's first node and its others: the components of
    # those links, each rooted at its smallest feature index
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    k = cells.shape[1] if cells.size else 0
    a = np.repeat(cells[:, 0].astype(np.int64), max(k - 1, 0)) if k else np.zeros(0, np.int64)
    b = cells[:, 1:].reshape(-1).astype(np.int64) if k else np.zeros(0, np.int64)
    g = coo_matrix((np.ones(a.size, dtype=np.int8), (a, b)), shape=(n, n))
    _, label = connected_components(g, directed=False)
    root = np.full(label.max() + 1 if n else 0, n, dtype=np.int64)
    np.minimum.at(root, label, np.arange(n, dtype=np.int64))
    track = root[label].astype(np.uint64)
    return {"simplices": simplices, "lam": lam, "bary": bary, "track_id": track,
            "scalar": np.full(n, np.float32(T(threshold)), dtype=np.float32), "cells": cells}


def cpu_perm(p_idx: int, d: int):
    """Axis order of the p_idx-th Kuhn simplex of a hypercube as the CPU mesh
    decodes it (mesh.hpp:407-409): successive swaps p[i] <-> p[i + j] with
    j = p_idx % (d - i), p_idx /= (d - i)."""
    p = list(range(d))
    t = p_idx
    for i in range(d):
        j = t % (d - i)
        p[i], p[i + j] = p[i + j], p[i]
        t //= d - i
    return tuple(p)


_POP16 = np.array([bin(i).count("1") for i in range(1 << 16)], dtype=np.int64)


def _popcount(a: np.ndarray) -> np.ndarray:
    """Set bits of direction masks (below 2^15)."""
    return _POP16[np.asarray(a, dtype=np.int64)]


def contour_extruded(field: np.ndarray, cells, n_base_verts: int, n_layers: int, threshold: float,
                     q: float = 1e6):
    """Level sets on ExtrudedSimplicialMesh(UnstructuredSimplicialMesh, L)
    (mesh.hpp:542-599): field holds one value per vertex id s + t * S.

    The mesh's edges are the spatial edges of every layer, the vertical edges
    and the prism diagonals (v_a at t, v_b at t + 1, a < b: the Kuhn split of a
    prism over a sorted base cell); the reference's first pass visits the
    spatial and vertical ones, its patching meets the diagonals while visiting
    the cells by layer, base cell (stored order, each sorted) and Kuhn index j
    (vertices v_0..v_j at t, v_j..v_k at t + 1).  Same output layout as
    contour()."""
    T = field.dtype.type
    S, L = int(n_base_verts), int(n_layers)
    nv = S * (L + 1)
    cells = np.sort(np.asarray(cells, dtype=np.int64), axis=1)
    d = cells.shape[1]  # spacetime dims (base cell has d vertices)
    adj = (field[:nv] - T(threshold)).astype(T)
    pos = sos_positive(adj, np.arange(nv, dtype=np.uint64), q)
    pairs = np.unique(np.concatenate([cells[:, [i, j]] for i in range(d) for j in range(i + 1, d)]), axis=0)
    cand = []
    for t in range(L + 1):
        cand.append(np.stack([pairs[:, 0] + t * S, pairs[:, 1] + t * S], 1))
    for t in range(L):
        s = np.arange(S, dtype=np.int64)
        cand.append(np.stack([s + t * S, s + (t + 1) * S], 1))
        cand.append(np.stack([pairs[:, 0] + t * S, pairs[:, 1] + (t + 1) * S], 1))
    cand = np.concatenate(cand)
    cand = cand[pos[cand[:, 0]] != pos[cand[:, 1]]]
    order = np.lexsort((cand[:, 1], cand[:, 0]))
    edges = cand[order]
    n = len(edges)
    key = edges[:, 0] * nv + edges[:, 1]

    def node(x, y):
        lo, hi = np.minimum(x, y), np.maximum(x, y)
        return np.searchsorted(key, lo * nv + hi)

    a0, a1 = adj[edges[:, 0]], adj[edges[:, 1]]
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        dd = (a0 - a1).astype(T)
        l0 = (-a1 / dd).astype(T)
        l1 = (T(1.0) - l0).astype(T)
    eps = T(1e-9)
    ok = (np.abs(dd) >= T(1e-12)) & (l0 >= -eps) & (l0 <= T(1.0) + eps)
    l0 = np.where(ok, l0, T(0.5)).astype(T)
    l1 = np.where(ok, l1, T(0.5)).astype(T)

    # spacetime cells in the reference's visiting order
    nc = len(cells)
    verts = []
    for t in range(L):
        for j in range(d):
            v = np.concatenate([cells[:, :j + 1] + t * S, cells[:, j:] + (t + 1) * S], axis=1)
            verts.append((t, j, v))
    vlist = np.zeros((L * nc * d, d + 1), dtype=np.int64)
    for t, j, v in verts:
        idx = (t * nc + np.arange(nc)) * d + j
        vlist[idx] = v
    ps = pos[vlist]
    npos = ps.sum(axis=1)
    qidx = np.arange(len(vlist), dtype=np.int64)

    def late(x, y):
        return (y >= (x // S + 1) * S) & (y != x + S)

    order_key = np.arange(n, dtype=np.int64)
    if d == 3 and n:
        first = np.full(n, np.iinfo(np.int64).max, dtype=np.int64)
        for lone in range(4):
            for single_pos in (True, False):
                s2 = (npos == (1 if single_pos else 3)) & (ps[:, lone] == single_pos)
                for k_, o in enumerate(o for o in range(4) if o != lone):
                    i, j = min(lone, o), max(lone, o)
                    x, y = vlist[s2, i], vlist[s2, j]
                    lt = late(x, y)
                    np.minimum.at(first, node(x, y)[lt], (qidx[s2] * 4 + k_)[lt])
        for A in itertools.combinations(range(4), 2):
            B = [i for i in range(4) if i not in A]
            s2 = (npos == 2) & ps[:, A[0]] & ps[:, A[1]]
            for k_, (a, b) in enumerate((a, b) for a in A for b in B):
                i, j = min(a, b), max(a, b)
                x, y = vlist[s2, i], vlist[s2, j]
                lt = late(x, y)
                np.minimum.at(first, node(x, y)[lt], (qidx[s2] * 4 + k_)[lt])
        met = first != np.iinfo(np.int64).max
        order_key = np.where(met, n + first, order_key)

    def nd(i, j, sel):
        return node(vlist[sel, min(i, j)], vlist[sel, max(i, j)])

    out = []
    nvtx = d + 1
    for single_pos in (True, False):
        sel = npos == (1 if single_pos else d)
        for lone in range(nvtx):
            s2 = sel & (ps[:, lone] == single_pos)
            if not s2.any():
                continue
            c = [nd(lone, o, s2) for o in range(nvtx) if o != lone]
            out.append(np.sort(np.stack(c, axis=1), axis=1))
    if d == 3:
        for A in itertools.combinations(range(4), 2):
            B = [i for i in range(4) if i not in A]
            s2 = (npos == 2) & ps[:, A[0]] & ps[:, A[1]]
            if not s2.any():
                continue
            q4 = np.stack([nd(a, b, s2) for a in A for b in B], axis=1)
            q4 = np.take_along_axis(q4, np.argsort(order_key[q4], axis=1), axis=1)
            out.append(np.sort(q4[:, [0, 1, 2]], axis=1))
            out.append(np.sort(q4[:, [0, 2, 3]], axis=1))
    else:
        for two_pos in (True, False):
            sel = npos == (2 if two_pos else 3)
            for two in itertools.combinations(range(5), 2):
                three = [i for i in range(5) if i not in two]
                s2 = sel & (ps[:, two[0]] == two_pos) & (ps[:, two[1]] == two_pos)
                if not s2.any():
                    continue
                T0 = [nd(two[0], t, s2) for t in three]
                T1 = [nd(two[1], t, s2) for t in three]
                for c in ((T0[0], T0[1], T0[2], T1[2]), (T0[0], T0[1], T1[1], T1[2]),
                          (T0[0], T1[0], T1[1], T1[2])):
                    out.append(np.sort(np.stack(c, axis=1), axis=1))
    cells_out = np.unique(np.concatenate(out), axis=0).astype(np.uint32) if out else np.zeros((0, d), np.uint32)

    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    k = cells_out.shape[1]
    ua = np.repeat(cells_out[:, 0].astype(np.int64), k - 1)
    ub = cells_out[:, 1:].reshape(-1).astype(np.int64)
    g = coo_matrix((np.ones(ua.size, dtype=np.int8), (ua, ub)), shape=(n, n))
    _, label = connected_components(g, directed=False)
    root = np.full(label.max() + 1 if n else 0, n, dtype=np.int64)
    np.minimum.at(root, label, np.arange(n, dtype=np.int64))
    track = root[label].astype(np.uint64)
    return {"simplices": edges.astype(np.uint64),
            "lam": np.stack([l0.astype(np.float64), l1.astype(np.float64)], axis=1),
            "bary": np.stack([l0.astype(np.float32), l1.astype(np.float32)], axis=1),
            "track_id": track, "scalar": np.full(n, np.float32(T(threshold)), dtype=np.float32),
            "cells": cells_out}
