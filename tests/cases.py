"""Seeded input cases shared by the golden-fixture script, the oracle tests and
the GPU parity tests.  Each case builds a mesh spec and a field exactly the way
the reference's own tests and examples do (tests/test_examples.cpp:39-186,
examples/critical_point_2d.cpp, tests/test_unstructured.cpp)."""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from ftk2_b200 import synthetic as S

MULTI, SEPARATE, PER_VERTEX = 0, 1, 2


@dataclass
class Case:
    name: str
    kind: str                     # "regular" | "extruded"
    ncomp: int
    layout: int
    arrays: object                # MULTI: one array; else list of arrays
    sos_q: float
    local_dims: list = field(default_factory=list)
    offset: Optional[list] = None
    global_dims: Optional[list] = None
    scalar: Optional[np.ndarray] = None
    coords: Optional[np.ndarray] = None
    cells: Optional[np.ndarray] = None
    n_layers: int = 0

    def input_digest(self) -> str:
        h = hashlib.sha256()
        arrs = [self.arrays] if self.layout == MULTI else list(self.arrays)
        for a in arrs:
            h.update(np.ascontiguousarray(a).tobytes())
        if self.scalar is not None:
            h.update(np.ascontiguousarray(self.scalar).tobytes())
        if self.cells is not None:
            h.update(np.ascontiguousarray(self.cells).tobytes())
        return h.hexdigest()


def c1_analytic_2d() -> Case:
    """Config 1: 64x64x10 gradient of cos(x cos t - y sin t) sin(x sin t + y cos t)."""
    return Case("c1_analytic_2d", "regular", 2, MULTI, S.analytic_2d(64, 64, 10), 1e6, [64, 64, 10])


def linear_24() -> Case:
    """tests/test_examples.cpp:153-186: float linear field moving 0.1 voxel/step,
    separate U/V/W arrays and a zero scalar; exercises every SoS fallback level."""
    DW, DT = 24, 8
    x = np.arange(DW, dtype=np.float32)
    U = np.empty((DT, DW, DW, DW), np.float32)
    V = np.empty_like(U)
    W = np.empty_like(U)
    for t in range(DT):
        cx = np.float32(16.0) + np.float32(t) * np.float32(0.1)
        U[t] = x[None, None, :] - cx
        V[t] = x[None, :, None] - np.float32(16)
        W[t] = x[:, None, None] - np.float32(16)
    return Case("linear_24", "regular", 3, SEPARATE, [U, V, W], 1e6, [DW, DW, DW, DT],
                scalar=np.zeros_like(U))


def gauss3d_16() -> Case:
    g = S.gaussian_sum_gradient((16, 16, 16), 4, seed=42, n_blobs=32)
    return Case("gauss3d_16", "regular", 3, MULTI, g, 2.0 ** 20, [16, 16, 16, 4])


def offset2d_legacy() -> Case:
    """Core-region mesh with offset over separate arrays plus a scalar
    (examples/critical_point_2d.cpp:65-84 pattern)."""
    g = S.gaussian_sum_gradient((20, 18), 6, seed=3, n_blobs=8, sigma=(2, 4))
    U, V = np.ascontiguousarray(g[..., 0]), np.ascontiguousarray(g[..., 1])
    sc = np.random.default_rng(0).standard_normal(U.shape)
    return Case("offset2d_legacy", "regular", 2, SEPARATE, [U, V], 1e6, [16, 14, 6], [2, 1, 0],
                [20, 18, 6], scalar=sc)


def offset2d_multi() -> Case:
    g = S.gaussian_sum_gradient((20, 18), 6, seed=3, n_blobs=8, sigma=(2, 4))
    return Case("offset2d_multi", "regular", 2, MULTI, g, 1e6, [16, 14, 6], [2, 1, 0], [20, 18, 6])


def f32_2d() -> Case:
    g = S.gaussian_sum_gradient((40, 40), 6, seed=5, n_blobs=12, dtype=np.float32, sigma=(2, 5))
    return Case("f32_2d", "regular", 2, MULTI, g, 1e6, [40, 40, 6])


def f32_3d_noise_offset() -> Case:
    g = S.gaussian_sum_gradient((14, 12, 10), 4, seed=9, n_blobs=16, dtype=np.float32, noise=1e-3,
                                sigma=(2, 4))
    return Case("f32_3d_noise_offset", "regular", 3, MULTI, g, 2.0 ** 20, [12, 10, 8, 3],
                [1, 2, 1, 1], [14, 12, 10, 4])


def extruded_3d(seed: int = 0) -> Case:
    coords, tets = S.extruded_tet_mesh(10, 9, 7, seed=seed)
    L = 4
    vals = S.gaussian_sum_gradient_at(coords, L + 1, seed=100 + seed, n_blobs=20, sigma=(1.0, 2.5),
                                      drift=0.8)
    return Case(f"extruded_3d_s{seed}", "extruded", 3, PER_VERTEX, [vals[0], vals[1], vals[2]],
                2.0 ** 20, coords=coords, cells=tets, n_layers=L)


def extruded_2d() -> Case:
    coords, _ = S.extruded_tet_mesh(8, 8, 2, seed=1)
    coords = coords[:64]
    nx = 8
    i, j = np.meshgrid(np.arange(7), np.arange(7), indexing="xy")
    p = (i + nx * j).ravel()
    tris = np.sort(np.concatenate([np.stack([p, p + 1, p + nx + 1], 1),
                                   np.stack([p, p + nx + 1, p + nx], 1)]), 1).astype(np.uint64)
    vals = S.gaussian_sum_gradient_at(coords[:, :2], 6, seed=4, n_blobs=6, sigma=(1, 3))
    return Case("extruded_2d", "extruded", 2, PER_VERTEX, [vals[0], vals[1]], 1e6,
                coords=coords, cells=tris, n_layers=5)


GOLDEN_CASES: dict[str, Callable[[], Case]] = {
    "c1_analytic_2d": c1_analytic_2d,
    "linear_24": linear_24,
    "gauss3d_16": gauss3d_16,
    "offset2d_legacy": offset2d_legacy,
    "offset2d_multi": offset2d_multi,
    "f32_2d": f32_2d,
    "f32_3d_noise_offset": f32_3d_noise_offset,
    "extruded_3d_s0": lambda: extruded_3d(0),
    "extruded_3d_s4": lambda: extruded_3d(4),
    "extruded_2d": extruded_2d,
}


def oracle_inputs(case: Case, keep: list, n_threads: int = 0):
    """(mesh, field) descriptors for oracle/bridge.py."""
    from oracle import bridge as B
    if case.kind == "regular":
        mesh = B.make_regular_mesh(case.local_dims, case.offset, case.global_dims)
    else:
        mesh = B.make_extruded_mesh(case.coords, case.cells, case.n_layers, keep)
    fld = B.make_field(case.arrays, case.layout, case.ncomp, scalar=case.scalar, sos_q=case.sos_q,
                       n_threads=n_threads, keep=keep)
    return mesh, fld


def gpu_inputs(case: Case, keep: list):
    """(mesh, field) descriptors for ftk2_b200.api."""
    from ftk2_b200 import api
    if case.kind == "regular":
        mesh = api.regular_mesh_desc(case.local_dims, case.offset, case.global_dims)
    else:
        mesh = api.extruded_mesh_desc(case.coords.shape[0], case.cells, case.n_layers, keep)
    fld = api.field_desc(case.arrays, case.layout, case.ncomp, scalar=case.scalar, keep=keep)
    return mesh, fld
