"""Seeded inputs of the level-set (contour) and fiber parity cases.

Each maker returns a dict: field (C-order, reversed Fortran shape of the local
mesh), local_dims, offset, global_dims, threshold, q.  The moving sphere is
the reference's own level-set example (tests/test_examples.cpp:225-256,
66418 feature vertices); the others are seeded Gaussian sums, an integer field
full of exact zeros (simulation-of-simplicity ties), a sub-box mesh with an
offset, a single time layer and a field with no crossing at all.
"""
from __future__ import annotations

import numpy as np


def gaussian_potential(dims, nt, seed, n_blobs, dtype, sigma=(2.0, 6.0), drift=0.5):
    """Sum of drifting Gaussians, shape (nt, [nz,] ny, nx)."""
    rng = np.random.default_rng(seed)
    d = len(dims)
    centers = rng.uniform(0, 1, (n_blobs, d)) * np.array(dims, dtype=np.float64)
    amps = rng.standard_normal(n_blobs)
    sig = rng.uniform(sigma[0], sigma[1], n_blobs)
    vel = rng.uniform(-drift, drift, (n_blobs, d))
    axes = [np.arange(n, dtype=np.float64) for n in dims]
    out = np.zeros((nt,) + tuple(dims[::-1]), dtype=np.float64)
    for t in range(nt):
        for b in range(n_blobs):
            c = centers[b] + vel[b] * t
            r2 = 0.0
            for i in range(d):
                shape = [1] * d
                shape[d - 1 - i] = dims[i]
                r2 = r2 + ((axes[i] - c[i]) ** 2).reshape(shape)
            out[t] += amps[b] * np.exp(-r2 / (2.0 * sig[b] ** 2))
    return out.astype(dtype)


def moving_sphere():
    """The reference's levelset_3d test field: |p - c(t)| - 8 on 32^3 x 10,
    c(t) = (16 + 0.2 t, 16, 16), float, threshold 0."""
    DW = DH = DD = 32
    DT = 10
    x = np.arange(DW, dtype=np.float32)
    S = np.empty((DT, DD, DH, DW), dtype=np.float32)
    for t in range(DT):
        cx = np.float32(16.0) + np.float32(t) * np.float32(0.2)
        c16 = np.float32(16.0)
        dx = (x - cx).astype(np.float64)
        dy = (x - c16).astype(np.float64)
        dz = (x - c16).astype(np.float64)
        s = dx[None, None, :] ** 2 + dy[None, :, None] ** 2
        s = s + dz[:, None, None] ** 2
        S[t] = np.sqrt(s).astype(np.float32) - np.float32(8.0)
    return dict(field=S, local_dims=[DW, DH, DD, DT], offset=None, global_dims=None, threshold=0.0, q=1e6)


def gauss_2d_f64():
    f = gaussian_potential((40, 36), 6, seed=11, n_blobs=12, dtype=np.float64)
    return dict(field=f, local_dims=[40, 36, 6], offset=None, global_dims=None, threshold=0.05, q=1e6)


def gauss_3d_f32_offset():
    """A 12x10x9x4 sub-box at offset (3,4,2,1) of a 20x18x16x5 mesh; the
    array holds the sub-box's values."""
    g = gaussian_potential((20, 18, 16), 5, seed=5, n_blobs=10, dtype=np.float32, sigma=(2.0, 5.0))
    sub = np.ascontiguousarray(g[1:5, 2:11, 4:14, 3:15])
    return dict(field=sub, local_dims=[12, 10, 9, 4], offset=[3, 4, 2, 1], global_dims=[20, 18, 16, 5],
                threshold=-0.2, q=2.0 ** 20)


def ties_2d():
    """Integer values in {-1, 0, 1}: every zero is decided by vertex parity."""
    rng = np.random.default_rng(3)
    f = rng.integers(-1, 2, (4, 16, 16)).astype(np.float64)
    return dict(field=f, local_dims=[16, 16, 4], offset=None, global_dims=None, threshold=0.0, q=1e6)


def ties_2d_offset():
    """Integer values on a 14x12x4 sub-box at offset (3, 4, 1) of a 20x18x5
    mesh: parity ties and quads cut at the sub-box's upper faces."""
    rng = np.random.default_rng(4)
    full = rng.integers(-1, 2, (5, 18, 20)).astype(np.float64)
    sub = np.ascontiguousarray(full[1:5, 4:16, 3:17])
    return dict(field=sub, local_dims=[14, 12, 4], offset=[3, 4, 1], global_dims=[20, 18, 5], threshold=0.0,
                q=1e6)


def single_layer_3d():
    f = gaussian_potential((10, 10, 10), 2, seed=8, n_blobs=6, dtype=np.float64)
    return dict(field=f, local_dims=[10, 10, 10, 2], offset=None, global_dims=None, threshold=-0.01, q=1e6)


def no_crossing():
    f = np.full((3, 8, 8), 2.5, dtype=np.float64)
    return dict(field=f, local_dims=[8, 8, 3], offset=None, global_dims=None, threshold=0.0, q=1e6)


CASES = {
    "moving_sphere": moving_sphere,
    "gauss_2d_f64": gauss_2d_f64,
    "gauss_3d_f32_offset": gauss_3d_f32_offset,
    "ties_2d": ties_2d,
    "ties_2d_offset": ties_2d_offset,
    "single_layer_3d": single_layer_3d,
    "no_crossing": no_crossing,
}

# the reference's own known answer (tests/test_examples.cpp:256)
SPHERE_VERTICES = 66418


# ---- fibers (FiberPredicate<T>): two scalar fields F, G on 2D+t meshes.
# Makers return a dict: fields (F, G; C-order, reversed Fortran shape),
# local_dims, offset, global_dims, thresholds, q.

def fiber_gauss_f64():
    f = gaussian_potential((40, 36), 6, seed=31, n_blobs=10, dtype=np.float64)
    g = gaussian_potential((40, 36), 6, seed=32, n_blobs=10, dtype=np.float64)
    return dict(fields=(f, g), local_dims=[40, 36, 6], offset=None, global_dims=None, thresholds=(0.05, -0.02),
                q=1e6)


def fiber_seeded(dims=(160, 144), nt=12, dtype=np.float32):
    """Two seeded 24-blob potentials at their medians: hundreds of fiber
    points, most of them where the f32 solve fails (centroid fallback)."""
    f = gaussian_potential(dims, nt, seed=41, n_blobs=24, dtype=dtype)
    g = gaussian_potential(dims, nt, seed=42, n_blobs=24, dtype=dtype)
    return dict(fields=(f, g), local_dims=[dims[0], dims[1], nt], offset=None, global_dims=None,
                thresholds=(float(np.median(f)), float(np.median(g))), q=2.0 ** 20)


def fiber_surface_seeded(dims=(32, 28, 24), nt=5, dtype=np.float32):
    """Two seeded potentials on a 3D+t mesh at their medians: thousands of
    fiber-surface triangles across many blocks of the device pipeline."""
    f = gaussian_potential(dims, nt, seed=61, n_blobs=16, dtype=dtype, sigma=(2.0, 5.0))
    g = gaussian_potential(dims, nt, seed=62, n_blobs=16, dtype=dtype, sigma=(2.0, 5.0))
    return dict(fields=(f, g), local_dims=list(dims) + [nt], offset=None, global_dims=None,
                thresholds=(float(np.median(f)), float(np.median(g))), q=2.0 ** 20)


def fiber_f32_offset():
    """A 24x20x5 sub-box at offset (3, 4, 1) of a 30x28x7 mesh; the arrays
    hold the sub-box's values."""
    f = gaussian_potential((30, 28), 7, seed=33, n_blobs=8, dtype=np.float32)
    g = gaussian_potential((30, 28), 7, seed=34, n_blobs=8, dtype=np.float32)
    sub = tuple(np.ascontiguousarray(a[1:6, 4:24, 3:27]) for a in (f, g))
    thr = tuple(float(np.median(a)) for a in sub)  # levels that cross inside the box
    return dict(fields=sub, local_dims=[24, 20, 5], offset=[3, 4, 1], global_dims=[30, 28, 7],
                thresholds=thr, q=2.0 ** 20)


def fiber_ties():
    """Integer values in {-1, 0, 1}: zeros decided by vertex parity, and
    degenerate triangles where the solve fails and the centroid is kept."""
    rng = np.random.default_rng(35)
    f = rng.integers(-1, 2, (4, 14, 15)).astype(np.float64)
    g = rng.integers(-1, 2, (4, 14, 15)).astype(np.float64)
    return dict(fields=(f, g), local_dims=[15, 14, 4], offset=None, global_dims=None, thresholds=(0.0, 0.0),
                q=1e6)


def fiber_near_quantum():
    """Values of a few 1/Q: many triangles whose quantised values are zero or
    one unit, where the simulation of simplicity finds the origin inside but
    the solve's pivot falls below 1e-12 and the centroid is kept."""
    rng = np.random.default_rng(36)
    f = rng.uniform(-3e-6, 3e-6, (4, 18, 20))
    g = rng.uniform(-3e-6, 3e-6, (4, 18, 20))
    return dict(fields=(f, g), local_dims=[20, 18, 4], offset=None, global_dims=None, thresholds=(0.0, 0.0),
                q=1e6)


FIBER_CASES = {
    "fiber_gauss_f64": fiber_gauss_f64,
    "fiber_f32_offset": fiber_f32_offset,
    "fiber_ties": fiber_ties,
    "fiber_near_quantum": fiber_near_quantum,
}


# ---- fiber surfaces (FiberPredicate<T> on 3D+t meshes): two scalar fields.

def fs_gauss_f64():
    f = gaussian_potential((10, 9, 8), 4, seed=51, n_blobs=6, dtype=np.float64, sigma=(1.5, 4.0))
    g = gaussian_potential((10, 9, 8), 4, seed=52, n_blobs=6, dtype=np.float64, sigma=(1.5, 4.0))
    return dict(fields=(f, g), local_dims=[10, 9, 8, 4], offset=None, global_dims=None, thresholds=(0.0, 0.0),
                q=1e6)


def fs_f32_offset():
    """A 11x10x9x3 sub-box at offset (2, 1, 3, 1) of a 14x12x13x5 mesh."""
    f = gaussian_potential((14, 12, 13), 5, seed=53, n_blobs=7, dtype=np.float32, sigma=(1.5, 4.0))
    g = gaussian_potential((14, 12, 13), 5, seed=54, n_blobs=7, dtype=np.float32, sigma=(1.5, 4.0))
    sub = tuple(np.ascontiguousarray(a[1:4, 3:12, 1:11, 2:13]) for a in (f, g))
    thr = tuple(float(np.median(a)) for a in sub)
    return dict(fields=sub, local_dims=[11, 10, 9, 3], offset=[2, 1, 3, 1], global_dims=[14, 12, 13, 5],
                thresholds=thr, q=2.0 ** 20)


def fs_near_quantum():
    """Values of a few 1/Q: the centroid fallback and many ties."""
    rng = np.random.default_rng(55)
    f = rng.uniform(-3e-6, 3e-6, (3, 6, 7, 8))
    g = rng.uniform(-3e-6, 3e-6, (3, 6, 7, 8))
    return dict(fields=(f, g), local_dims=[8, 7, 6, 3], offset=None, global_dims=None, thresholds=(0.0, 0.0),
                q=1e6)


FIBER_SURFACE_CASES = {
    "fs_gauss_f64": fs_gauss_f64,
    "fs_f32_offset": fs_f32_offset,
    "fs_near_quantum": fs_near_quantum,
}


# ---- level sets on ExtrudedSimplicialMesh(UnstructuredSimplicialMesh, L):
# makers return a dict: coords, cells (base), n_layers, field (one value per
# vertex id s + t * S), threshold, q.

def ext_tri_2d():
    """A triangulated 8x8 grid (jittered), 5 layers: 2D+t."""
    from ftk2_b200 import synthetic as S
    coords, _ = S.extruded_tet_mesh(8, 8, 2, seed=1)
    coords = coords[:64]
    nx = 8
    i, j = np.meshgrid(np.arange(7), np.arange(7), indexing="xy")
    p = (i + nx * j).ravel()
    tris = np.sort(np.concatenate([np.stack([p, p + 1, p + nx + 1], 1),
                                   np.stack([p, p + nx + 1, p + nx], 1)]), 1).astype(np.uint64)
    L = 5
    t = np.arange(L + 1)[:, None]
    f = (np.sin(coords[None, :, 0] / 1.7) + np.cos(coords[None, :, 1] / 2.3) + 0.15 * t - 0.4).reshape(-1)
    return dict(coords=coords, cells=tris, n_layers=L, field=np.ascontiguousarray(f), threshold=0.0, q=1e6)


def ext_tet_3d():
    """A jittered 7x6x4 tet mesh, 3 layers: 3D+t."""
    from ftk2_b200 import synthetic as S
    coords, tets = S.extruded_tet_mesh(7, 6, 4, seed=2)
    L = 3
    t = np.arange(L + 1)[:, None]
    f = (np.sin(coords[None, :, 0] / 1.3) * np.cos(coords[None, :, 1] / 1.9) + 0.2 * coords[None, :, 2] - 0.3
         + 0.1 * t).reshape(-1)
    return dict(coords=coords, cells=tets, n_layers=L, field=np.ascontiguousarray(f), threshold=0.0, q=1e6)


def ext_tri_ties_f32():
    """Integer values on the 2D+t grid, float32: parity ties everywhere."""
    c = ext_tri_2d()
    rng = np.random.default_rng(9)
    c["field"] = rng.integers(-1, 2, c["field"].shape).astype(np.float32)
    return c


EXTRUDED_CASES = {
    "ext_tri_2d": ext_tri_2d,
    "ext_tet_3d": ext_tet_3d,
    "ext_tri_ties_f32": ext_tri_ties_f32,
}


# ---- fibers on extruded 2D+t meshes (two per-vertex fields)

def fiber_ext_tri():
    c = ext_tri_2d()
    coords, L = c["coords"], c["n_layers"]
    t = np.arange(L + 1)[:, None]
    f = (np.sin(coords[None, :, 0] / 1.7) + 0.1 * t - 0.2).reshape(-1)
    g = (np.cos(coords[None, :, 1] / 2.1) - 0.15 * t + 0.1).reshape(-1)
    return dict(coords=coords, cells=c["cells"], n_layers=L, fields=(np.ascontiguousarray(f), np.ascontiguousarray(g)),
                thresholds=(0.0, 0.0), q=1e6)


def fiber_ext_near_quantum():
    c = ext_tri_2d()
    rng = np.random.default_rng(12)
    n = c["field"].size
    return dict(coords=c["coords"], cells=c["cells"], n_layers=c["n_layers"],
                fields=(rng.uniform(-3e-6, 3e-6, n), rng.uniform(-3e-6, 3e-6, n)), thresholds=(0.0, 0.0), q=1e6)


FIBER_EXTRUDED_CASES = {
    "fiber_ext_tri": fiber_ext_tri,
    "fiber_ext_near_quantum": fiber_ext_near_quantum,
}


# ---- fiber surfaces on extruded 3D+t meshes (ExtrudedSimplicialMesh over
# tets, two per-vertex fields); the reference numbers the triangles it finds
# while patching in the order its workers meet them, so fixtures come from
# its one-worker build

def _ext_tet_fields(nx, ny, nz, L, seed, dtype=np.float64, n_blobs=6):
    from ftk2_b200 import synthetic as S
    coords, tets = S.extruded_tet_mesh(nx, ny, nz, seed=seed)
    f = S.gaussian_sum_gradient_at(coords, L + 1, seed=seed, n_blobs=n_blobs, sigma=(1.0, 2.5), drift=0.4)
    return coords, tets, (np.ascontiguousarray(f[0].astype(dtype)), np.ascontiguousarray(f[1].astype(dtype)))


def fs_ext_gauss_f64():
    coords, tets, fields = _ext_tet_fields(7, 6, 5, 4, 2)
    return dict(coords=coords, cells=tets, n_layers=4, fields=fields, thresholds=(0.0, 0.0), q=2.0 ** 20)


def fs_ext_f32_thresholds():
    coords, tets, fields = _ext_tet_fields(6, 6, 6, 3, 3, np.float32)
    return dict(coords=coords, cells=tets, n_layers=3, fields=fields, thresholds=(0.01, -0.02), q=2.0 ** 20)


def fs_ext_near_quantum():
    """Values of a few 1/Q: ties in the origin test and failed solves (the
    centroid fallback)."""
    from ftk2_b200 import synthetic as S
    coords, tets = S.extruded_tet_mesh(5, 5, 4, seed=4)
    rng = np.random.default_rng(14)
    n = coords.shape[0] * 4
    return dict(coords=coords, cells=tets, n_layers=3,
                fields=(rng.uniform(-3e-6, 3e-6, n), rng.uniform(-3e-6, 3e-6, n)), thresholds=(0.0, 0.0), q=1e6)


def fs_ext_seeded(nx=14, ny=12, nz=8, L=5, dtype=np.float32):
    coords, tets, fields = _ext_tet_fields(nx, ny, nz, L, 7, dtype, n_blobs=12)
    return dict(coords=coords, cells=tets, n_layers=L, fields=fields, thresholds=(0.0, 0.0), q=2.0 ** 20)


FIBER_SURFACE_EXTRUDED_CASES = {
    "fs_ext_gauss_f64": fs_ext_gauss_f64,
    "fs_ext_f32_thresholds": fs_ext_f32_thresholds,
    "fs_ext_near_quantum": fs_ext_near_quantum,
}
