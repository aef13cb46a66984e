"""Seeded synthetic inputs for the critical-point path.

The reference ships no generator for these workloads (its tests build fields
in-test, tests/test_examples.cpp:153-173, or call ndarray's
synthetic_woven_2Dt, which is not vendored), so the fields are defined here
from the workload descriptions and are deterministic given the seed:

* ``analytic_2d``: gradient of f(x,y,t) = cos(x cos t - y sin t) *
  sin(x sin t + y cos t) on [0,10]^2, dt = 0.1, stored as a multicomponent
  [2, nx, ny, nt] float64 array (component fastest, Fortran order).
* ``gaussian_sum_gradient``: analytic gradient of a sum of drifting Gaussians
  A_b * exp(-|p - c_b - v_b t|^2 / (2 sigma_b^2)), p in voxel units, stored as
  [ncomp, nx, ny, (nz,) nt].

Arrays are returned as numpy arrays in C order with the component axis LAST
in memory, i.e. shape (nt, [nz,] ny, nx, ncomp): the same bytes as the
reference's Fortran-order [ncomp, nx, ny, (nz,) nt] ndarray.
"""
from __future__ import annotations

import numpy as np


def analytic_2d(nx: int = 64, ny: int = 64, nt: int = 10, extent: float = 10.0,
                dt: float = 0.1) -> np.ndarray:
    """Gradient of cos(x cos t - y sin t) * sin(x sin t + y cos t).

    Returns float64 array of shape (nt, ny, nx, 2).
    """
    x = extent * np.arange(nx, dtype=np.float64) / (nx - 1)
    y = extent * np.arange(ny, dtype=np.float64) / (ny - 1)
    out = np.empty((nt, ny, nx, 2), dtype=np.float64)
    X, Y = np.meshgrid(x, y, indexing="xy")  # (ny, nx)
    for k in range(nt):
        t = dt * k
        c, s = np.cos(t), np.sin(t)
        u = X * c - Y * s
        w = X * s + Y * c
        cu, su, cw, sw = np.cos(u), np.sin(u), np.cos(w), np.sin(w)
        out[k, :, :, 0] = -su * c * sw + cu * cw * s
        out[k, :, :, 1] = su * s * sw + cu * cw * c
    return out


def gaussian_blobs(seed: int, n_blobs: int, box, sigma=(4.0, 12.0), drift=0.5):
    """Blob parameters: centers U[0, box), amplitudes N(0,1), sigma U[lo,hi],
    drift U[-drift, drift] voxels per step.  Returns dict of float64 arrays."""
    rng = np.random.default_rng(seed)
    ndim = len(box)
    centers = rng.uniform(0.0, 1.0, size=(n_blobs, ndim)) * np.asarray(box, dtype=np.float64)
    amps = rng.standard_normal(n_blobs)
    sig = rng.uniform(sigma[0], sigma[1], size=n_blobs)
    vel = rng.uniform(-drift, drift, size=(n_blobs, ndim))
    return {"centers": centers, "amps": amps, "sigma": sig, "vel": vel}


def gaussian_sum_gradient(dims, nt: int, seed: int = 1234, n_blobs: int = 32,
                          dtype=np.float64, noise: float = 0.0, noise_seed: int | None = None,
                          sigma=(4.0, 12.0), drift=0.5, box=None, origin=None,
                          t0: int = 0) -> np.ndarray:
    """Analytic gradient of a drifting Gaussian sum on a regular grid.

    dims: spatial dims (nx, ny) or (nx, ny, nz) of the evaluated region.
    Blob centres are drawn over ``box`` (default ``dims``); ``origin`` and
    ``t0`` place the evaluated region inside a larger field, so a corner of a
    big field can be generated alone.  Returns array of shape
    (nt, [nz,] ny, nx, ncomp) in ``dtype``; computed in float64 and rounded.
    """
    ndim = len(dims)
    blobs = gaussian_blobs(seed, n_blobs, box if box is not None else dims, sigma, drift)
    origin = origin if origin is not None else [0] * ndim
    axes = [origin[i] + np.arange(n, dtype=np.float64) for i, n in enumerate(dims)]
    # grids in (.., y, x) order
    grids = np.meshgrid(*axes[::-1], indexing="ij")[::-1]  # grids[k] is coord k, shape rev(dims)
    shape = tuple(dims[::-1])
    out = np.zeros((nt,) + shape + (ndim,), dtype=np.float64)
    for k in range(nt):
        acc = [np.zeros(shape) for _ in range(ndim)]
        for b in range(n_blobs):
            c = blobs["centers"][b] + blobs["vel"][b] * (k + t0)
            s2 = blobs["sigma"][b] ** 2
            d = [grids[i] - c[i] for i in range(ndim)]
            r2 = sum(di * di for di in d)
            e = blobs["amps"][b] * np.exp(-r2 / (2.0 * s2))
            for i in range(ndim):
                acc[i] -= e * d[i] / s2
        for i in range(ndim):
            out[k, ..., i] = acc[i]
    if noise:
        rng = np.random.default_rng(seed + 1 if noise_seed is None else noise_seed)
        out += noise * rng.standard_normal(out.shape)
    return out.astype(dtype)


def extruded_tet_mesh(nx: int = 100, ny: int = 100, n_layers: int = 40, jitter: float = 0.3,
                      seed: int = 7, h: float = 1.0):
    """Jittered triangulated plane extruded into a conforming tet mesh.

    The nx*ny grid of points is jittered by U[-jitter, jitter]*h in x and y,
    each quad is split into two triangles along a fixed diagonal, and the
    plane is stacked n_layers times in z (layer spacing h).  Each prism
    between layers is split into 3 tets by the sorted-vertex (staircase) rule:
    with bottom vertices a < b < c (by id) and tops a' < b' < c', the tets are
    (a,b,c,c'), (a,b,b',c'), (a,a',b',c').  Shared quad faces then split the
    same way from both sides, so the mesh is conforming.

    Returns (coords (nv, 3) float64, tets (n_tet, 4) uint64).
    """
    rng = np.random.default_rng(seed)
    jx = rng.uniform(-jitter, jitter, size=(ny, nx)) * h
    jy = rng.uniform(-jitter, jitter, size=(ny, nx)) * h
    X, Y = np.meshgrid(np.arange(nx) * h, np.arange(ny) * h, indexing="xy")
    X = X + jx
    Y = Y + jy
    npl = nx * ny
    coords = np.empty((n_layers * npl, 3), dtype=np.float64)
    for k in range(n_layers):
        coords[k * npl:(k + 1) * npl, 0] = X.ravel()
        coords[k * npl:(k + 1) * npl, 1] = Y.ravel()
        coords[k * npl:(k + 1) * npl, 2] = k * h
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="xy")
    p00 = (i + nx * j).ravel()
    p10 = p00 + 1
    p01 = p00 + nx
    p11 = p01 + 1
    tris = np.concatenate([np.stack([p00, p10, p11], 1), np.stack([p00, p11, p01], 1)], 0)
    tris = np.sort(tris, axis=1).astype(np.int64)
    tets = []
    for k in range(n_layers - 1):
        a, b, c = (tris[:, 0] + k * npl, tris[:, 1] + k * npl, tris[:, 2] + k * npl)
        a2, b2, c2 = a + npl, b + npl, c + npl
        tets.append(np.stack([a, b, c, c2], 1))
        tets.append(np.stack([a, b, b2, c2], 1))
        tets.append(np.stack([a, a2, b2, c2], 1))
    tets = np.concatenate(tets, 0).astype(np.uint64)
    return coords, tets


def gaussian_sum_gradient_at(points: np.ndarray, nt: int, seed: int = 1234, n_blobs: int = 32,
                             box=None, dtype=np.float64, sigma=(4.0, 12.0), drift=0.5) -> np.ndarray:
    """The drifting Gaussian-sum gradient sampled at arbitrary points.

    points: (nv, ndim).  Returns (ndim, nt * nv) in ``dtype``: one per-vertex
    array per component, vertex id = spatial id + t * nv, as the extruded
    mesh numbers its vertices (mesh.hpp:714-720).
    """
    points = np.asarray(points, dtype=np.float64)
    nv, ndim = points.shape
    if box is None:
        box = points.max(axis=0) + 1.0
    blobs = gaussian_blobs(seed, n_blobs, box, sigma, drift)
    out = np.zeros((ndim, nt, nv), dtype=np.float64)
    for k in range(nt):
        for b in range(n_blobs):
            c = blobs["centers"][b] + blobs["vel"][b] * k
            s2 = blobs["sigma"][b] ** 2
            d = points - c
            e = blobs["amps"][b] * np.exp(-(d * d).sum(1) / (2.0 * s2))
            out[:, k, :] -= (e[:, None] * d / s2).T
    return out.reshape(ndim, nt * nv).astype(dtype)
