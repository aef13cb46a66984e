"""GPU parity of the extruded-mesh path (ExtrudedSimplicialMesh over an
UnstructuredSimplicialMesh, mesh.hpp:542-730) through the C ABI.

* the reference engine's own outputs (golden fixtures): identical simplex ids,
  float barycentrics, lambdas, scalars, track ids and edges;
* seeded medium meshes, float64 and float32, with and without a scalar:
  identical to the exact C restatement;
* the refined-FP32 reporting mode keeps the accepted set and trajectories;
* the prepared base mesh is reused only while the cells are unchanged.
"""
import os

import numpy as np
import pytest

from ftk2_b200 import api
from ftk2_b200 import synthetic as S
from oracle import bridge
import cases

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
EXTRUDED_GOLDEN = [n for n in sorted(cases.GOLDEN_CASES) if n.startswith("extruded")]


def gpu_run(ctx, case, **kw):
    keep: list = []
    mesh, fld = cases.gpu_inputs(case, keep)
    return ctx.extract(mesh, fld, api.params(case.sos_q, **kw))


def oracle_run(case):
    keep: list = []
    mesh, fld = cases.oracle_inputs(case, keep)
    return bridge.run_restatement(mesh, fld)


def assert_identical(g, o, lam=True):
    assert g.simplices.shape == o.simplices.shape, (g.simplices.shape, o.simplices.shape)
    assert np.array_equal(g.simplices, o.simplices)
    assert np.array_equal(g.track_id, o.track_id)
    assert np.array_equal(g.edges, o.edges)
    assert np.array_equal(g.bary, o.bary)
    assert np.array_equal(g.scalar, o.scalar)
    assert np.array_equal(g.type, o.type)
    if lam:
        assert np.array_equal(g.lam, o.lam)


@pytest.mark.parametrize("name", EXTRUDED_GOLDEN)
def test_golden_extruded(ctx, name):
    case = cases.GOLDEN_CASES[name]()
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    assert str(z["input_sha256"]) == case.input_digest()
    g = gpu_run(ctx, case)
    ref = bridge.CPResult(simplices=z["simplices"], bary=z["bary"], lam=z["lam"],
                          track_id=z["track_id"], type=z["type"], scalar=z["scalar"],
                          edges=z["edges"])
    assert_identical(g, ref)
    assert g.n_tracks == len(np.unique(ref.track_id))


def _tri_plane(nx, ny, seed):
    coords, _ = S.extruded_tet_mesh(nx, ny, 2, seed=seed)
    coords = coords[: nx * ny]
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="xy")
    p = (i + nx * j).ravel()
    tris = np.sort(np.concatenate([np.stack([p, p + 1, p + nx + 1], 1),
                                   np.stack([p, p + nx + 1, p + nx], 1)]), 1).astype(np.uint64)
    return coords, tris


def _medium_cases():
    out = []
    for seed, dtype in ((1, np.float64), (2, np.float32)):
        coords, tets = S.extruded_tet_mesh(24, 22, 9, seed=seed)
        L = 5
        vals = S.gaussian_sum_gradient_at(coords, L + 1, seed=200 + seed, n_blobs=24,
                                          sigma=(1.0, 3.0), drift=0.6, dtype=dtype)
        out.append(cases.Case(f"ext3d_{np.dtype(dtype).name}_s{seed}", "extruded", 3, cases.PER_VERTEX,
                              [vals[0], vals[1], vals[2]], 2.0 ** 20, coords=coords, cells=tets,
                              n_layers=L))
    coords, tets = S.extruded_tet_mesh(20, 18, 7, seed=3)
    L = 4
    vals = S.gaussian_sum_gradient_at(coords, L + 1, seed=303, n_blobs=20, sigma=(1.0, 3.0), drift=0.6)
    sc = np.random.default_rng(9).standard_normal(vals.shape[1])
    out.append(cases.Case("ext3d_scalar", "extruded", 3, cases.PER_VERTEX, [vals[0], vals[1], vals[2]],
                          2.0 ** 20, coords=coords, cells=tets, n_layers=L, scalar=sc))
    for seed, dtype in ((4, np.float64), (5, np.float32)):
        coords, tris = _tri_plane(60, 50, seed)
        L = 9
        vals = S.gaussian_sum_gradient_at(coords[:, :2], L + 1, seed=400 + seed, n_blobs=30,
                                          sigma=(2.0, 5.0), dtype=dtype)
        out.append(cases.Case(f"ext2d_{np.dtype(dtype).name}_s{seed}", "extruded", 2, cases.PER_VERTEX,
                              [vals[0], vals[1]], 1e6, coords=coords, cells=tris, n_layers=L))
    # shuffled cell order and unsorted vertices within cells: the mesh is the same
    coords, tets = S.extruded_tet_mesh(16, 15, 6, seed=6)
    rng = np.random.default_rng(6)
    tets = tets[rng.permutation(len(tets))]
    tets = np.take_along_axis(tets, rng.permuted(np.tile(np.arange(4), (len(tets), 1)), axis=1), 1)
    L = 3
    vals = S.gaussian_sum_gradient_at(coords, L + 1, seed=606, n_blobs=16, sigma=(1.0, 2.5), drift=0.8)
    out.append(cases.Case("ext3d_shuffled", "extruded", 3, cases.PER_VERTEX, [vals[0], vals[1], vals[2]],
                          2.0 ** 20, coords=coords, cells=np.ascontiguousarray(tets), n_layers=L))
    return out


@pytest.mark.parametrize("case", _medium_cases(), ids=lambda c: c.name)
def test_medium_extruded_vs_restatement(ctx, case):
    g = gpu_run(ctx, case)
    o = oracle_run(case)
    assert len(o.track_id) > 0
    assert_identical(g, o)
    assert g.n_simplices == o.n_tested


def test_extruded_refined_same_set(ctx):
    case = _medium_cases()[1]  # float32
    e = gpu_run(ctx, case)
    r = gpu_run(ctx, case, precision=api.PRECISION_REFINED)
    assert np.array_equal(e.simplices, r.simplices)
    assert np.array_equal(e.track_id, r.track_id)
    assert np.array_equal(e.edges, r.edges)
    assert np.array_equal(e.bary, r.bary)
    assert np.abs(r.lam - e.lam).max() < 1e-3


def test_extruded_base_mesh_cache_follows_content(ctx):
    a = cases.GOLDEN_CASES["extruded_3d_s0"]()
    b = cases.GOLDEN_CASES["extruded_3d_s4"]()
    ga1 = gpu_run(ctx, a)
    gb = gpu_run(ctx, b)
    ga2 = gpu_run(ctx, a)
    assert_identical(ga1, ga2)
    assert_identical(gb, oracle_run(b))


def test_extruded_rejects_bad_vertex_ids(ctx):
    case = cases.GOLDEN_CASES["extruded_2d"]()
    cells = case.cells.copy()
    cells[3, 1] = case.coords.shape[0] + 5
    keep: list = []
    mesh = api.extruded_mesh_desc(case.coords.shape[0], cells, case.n_layers, keep)
    fld = api.field_desc(case.arrays, case.layout, case.ncomp, keep=keep)
    with pytest.raises(api.Ftk2bError) as e:
        ctx.extract(mesh, fld, api.params(case.sos_q))
    assert e.value.status == api.INVALID_ARG
    # the context stays usable
    assert_identical(gpu_run(ctx, case), oracle_run(case))
