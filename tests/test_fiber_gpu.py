"""Fibers on the GPU (ftk2b_fiber_extract) against the reference engine with
FiberPredicate<T> (predicate.hpp:341-362): on 2D+t meshes the features, float
and field-precision barycentrics (centroid where the solve fails), track ids
and star edges are identical to the reference's fixtures
(tests/golden/make_contour_golden.py) and, where the prebuilt reference
library is present, to a live reference run."""
import os

import numpy as np
import pytest

import contour_cases
from ftk2_b200 import api
from oracle import bridge

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "fiber")


def run_gpu(ctx, case, fields=None):
    keep: list = []
    mesh = api.regular_mesh_desc(case["local_dims"], case["offset"], case["global_dims"])
    fd = api.field_desc(list(case["fields"] if fields is None else fields), api.LAYOUT_SEPARATE, 2, keep=keep)
    return ctx.fiber(mesh, fd, case["thresholds"], case["q"])


def assert_same(r, want, name=""):
    assert len(r.track_id) == len(want["track_id"]), name
    assert np.array_equal(r.simplices, want["simplices"]), name
    assert np.array_equal(r.bary.view(np.uint32), want["bary"].view(np.uint32)), name
    assert np.array_equal(r.lam.view(np.uint64), want["lam"].view(np.uint64)), name
    assert np.array_equal(r.track_id, want["track_id"]), name
    assert np.array_equal(r.edges, want["edges"]), name
    assert not r.type.any() and not r.scalar.any()


@pytest.mark.parametrize("name", list(contour_cases.FIBER_CASES))
def test_fiber_matches_reference_fixture(ctx, name):
    case = contour_cases.FIBER_CASES[name]()
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    r = run_gpu(ctx, case)
    assert len(r.track_id) > 0
    assert_same(r, {k: g[k] for k in ("simplices", "bary", "lam", "track_id", "edges")}, name)
    assert r.n_tracks == len(set(r.track_id.tolist()))


@pytest.mark.parametrize("seed,dims,thr", [(41, [19, 17, 5], (0.0, 0.0)), (42, [8, 9, 3], (0.02, -0.01))])
def test_fiber_random_vs_live_reference(ctx, seed, dims, thr):
    if not bridge.ref_available():
        pytest.skip("reference build absent")
    f = contour_cases.gaussian_potential(tuple(dims[:2]), dims[2], seed=seed, n_blobs=6, dtype=np.float64,
                                         sigma=(1.5, 4.0))
    g = contour_cases.gaussian_potential(tuple(dims[:2]), dims[2], seed=seed + 100, n_blobs=6, dtype=np.float64,
                                         sigma=(1.5, 4.0))
    case = dict(fields=(f, g), local_dims=dims, offset=None, global_dims=None, thresholds=thr, q=1e6)
    keep: list = []
    ref = bridge.run_reference_fiber(bridge.make_regular_mesh(dims),
                                     bridge.make_field([f, g], bridge.LAYOUT_SEPARATE, 2, sos_q=1e6, keep=keep), thr)
    assert_same(run_gpu(ctx, case), {"simplices": ref.simplices, "bary": ref.bary, "lam": ref.lam,
                                     "track_id": ref.track_id, "edges": ref.edges}, str(seed))


def test_fiber_device_input_and_3d_mesh_rejected(ctx):
    torch = pytest.importorskip("torch")
    case = contour_cases.fiber_gauss_f64()
    host = run_gpu(ctx, case)
    dev = run_gpu(ctx, case, [torch.from_numpy(a).cuda() for a in case["fields"]])
    assert np.array_equal(host.simplices, dev.simplices) and np.array_equal(host.edges, dev.edges)
    a = np.zeros((3, 4, 5, 6))
    keep: list = []
    with pytest.raises(api.Ftk2bError):
        ctx.fiber(api.regular_mesh_desc([6, 5, 4, 3]), api.field_desc([a, a], api.LAYOUT_SEPARATE, 2, keep=keep))


FS_GOLD = os.path.join(os.path.dirname(__file__), "golden", "fiber_surface")


@pytest.mark.parametrize("name", list(contour_cases.FIBER_SURFACE_CASES))
def test_fiber_surface_matches_reference_fixture(ctx, name):
    """Fiber surfaces on 3D+t meshes (ftk2b_fiber_surface_extract): triangle
    features, barycentrics (centroid where the solve fails), track ids and the
    star-fan triangles of get_complex, bit for bit."""
    case = contour_cases.FIBER_SURFACE_CASES[name]()
    g = np.load(os.path.join(FS_GOLD, f"{name}.npz"))
    keep: list = []
    mesh = api.regular_mesh_desc(case["local_dims"], case["offset"], case["global_dims"])
    fd = api.field_desc(list(case["fields"]), api.LAYOUT_SEPARATE, 2, keep=keep)
    r = ctx.fiber_surface(mesh, fd, case["thresholds"], case["q"])
    assert len(r.track_id) == len(g["track_id"]) > 0
    assert np.array_equal(r.simplices, g["simplices"])
    assert np.array_equal(r.bary.view(np.uint32), g["bary"].view(np.uint32))
    assert np.array_equal(r.lam.view(np.uint64), g["lam"].view(np.uint64))
    assert np.array_equal(r.track_id, g["track_id"])
    assert np.array_equal(r.cells, g["cells"])
    assert r.n_tracks == len(set(r.track_id.tolist()))
    assert not r.scalar.any()


def test_fiber_surface_vs_live_reference(ctx):
    if not bridge.ref_available():
        pytest.skip("reference build absent")
    dims = [9, 8, 7, 3]
    f = contour_cases.gaussian_potential(tuple(dims[:3]), dims[3], seed=61, n_blobs=5, dtype=np.float64,
                                         sigma=(1.5, 3.5))
    g = contour_cases.gaussian_potential(tuple(dims[:3]), dims[3], seed=62, n_blobs=5, dtype=np.float64,
                                         sigma=(1.5, 3.5))
    thr = (float(np.median(f)), float(np.median(g)))  # levels that cross inside the box
    keep: list = []
    ref, cells = bridge.run_reference_fiber_surface(
        bridge.make_regular_mesh(dims), bridge.make_field([f, g], bridge.LAYOUT_SEPARATE, 2, sos_q=1e6, keep=keep),
        thr)
    r = ctx.fiber_surface(api.regular_mesh_desc(dims), api.field_desc([f, g], api.LAYOUT_SEPARATE, 2, keep=keep),
                          thr, 1e6)
    assert len(r.track_id) == len(ref.track_id) > 0
    assert np.array_equal(r.simplices, ref.simplices)
    assert np.array_equal(r.lam.view(np.uint64), ref.lam.view(np.uint64))
    assert np.array_equal(r.track_id, ref.track_id)
    assert np.array_equal(r.cells, cells)


@pytest.mark.parametrize("name,gold,conn", [("fiber_gauss_f64", "fiber", "edges"),
                                            ("fs_gauss_f64", "fiber_surface", "cells")])
def test_fiber_cpp_dropin_matches_reference_fixture(tmp_path, name, gold, conn):
    """SimplicialEngine<T, FiberPredicate<T>> of include/ftk2b/engine.hpp on a
    2D+t (star edges) and a 3D+t (star-fan triangles) mesh."""
    import subprocess
    from ftk2_b200 import build as fb
    cases = dict(contour_cases.FIBER_CASES, **contour_cases.FIBER_SURFACE_CASES)
    case = cases[name]()
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", gold, f"{name}.npz"))
    exe = fb.build_contour_test()
    paths = []
    for j, a in enumerate(case["fields"]):
        p = tmp_path / f"f{j}.bin"
        a.tofile(p)
        paths.append(str(p))
    dt = "f64" if case["fields"][0].dtype == np.float64 else "f32"
    out = tmp_path / "out.txt"
    r = subprocess.run([exe, "fiber", *paths, dt, ",".join(str(x) for x in case["local_dims"]),
                        repr(case["thresholds"][0]), repr(case["thresholds"][1]), repr(case["q"]), str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    feats, rows = [], []
    for line in open(out):
        if line.startswith("F"):
            vs, bs, tr = line[1:].split("|")
            feats.append(([int(x) for x in vs.split()], [int(x, 16) for x in bs.split()], int(tr)))
        elif line.startswith("C"):
            rows.append([int(x) for x in line.split()[2:]])
    assert len(feats) == len(g["track_id"]) > 0
    assert np.array_equal(np.array([v for v, _, _ in feats], dtype=np.uint64), g["simplices"])
    assert np.array_equal(np.array([b for _, b, _ in feats], dtype=np.uint32), g["bary"].view(np.uint32))
    assert np.array_equal(np.array([t for _, _, t in feats], dtype=np.uint64), g["track_id"])
    want = g[conn]
    assert np.array_equal(np.array(rows, dtype=np.uint32).reshape(-1, want.shape[1]), want)


FIBER_EXT_GOLD = os.path.join(os.path.dirname(__file__), "golden", "fiber_extruded")


@pytest.mark.parametrize("name", list(contour_cases.FIBER_EXTRUDED_CASES))
def test_fiber_extruded_matches_reference_fixture(ctx, name):
    """Fibers on ExtrudedSimplicialMesh over triangles (the extruded pipeline's
    fiber mode): features, barycentrics (centroid where the solve fails),
    tracks and star edges identical to the reference engine's."""
    case = contour_cases.FIBER_EXTRUDED_CASES[name]()
    g = np.load(os.path.join(FIBER_EXT_GOLD, f"{name}.npz"))
    keep: list = []
    mesh = api.extruded_mesh_desc(case["coords"].shape[0], case["cells"], case["n_layers"], keep)
    fd = api.field_desc(list(case["fields"]), api.LAYOUT_PER_VERTEX, 2, keep=keep)
    r = ctx.fiber(mesh, fd, case["thresholds"], case["q"])
    assert len(r.track_id) == len(g["track_id"]) > 0
    assert_same(r, {k: g[k] for k in ("simplices", "bary", "lam", "track_id", "edges")}, name)


# ---------------------------------------------------------------------------
# fiber surfaces on ExtrudedSimplicialMesh over tets (the reference numbers the
# triangles inside its prisms as its one-worker patching meets them)

FS_EXT_GOLD = os.path.join(os.path.dirname(__file__), "golden", "fiber_surface_extruded")


def run_fs_ext(ctx, case, device=False, layout=api.LAYOUT_SEPARATE):
    keep: list = []
    nv = case["coords"].shape[0]
    mesh = api.extruded_mesh_desc(nv, case["cells"], case["n_layers"], keep)
    arrays = list(case["fields"])
    if device:
        import torch
        arrays = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]
        keep.append(arrays)
    fd = api.field_desc(arrays, layout, 2, keep=keep)
    return ctx.fiber_surface(mesh, fd, case["thresholds"], case["q"])


def assert_same_surface(r, want, cells, name=""):
    assert len(r.track_id) == len(want["track_id"]) > 0, name
    assert np.array_equal(r.simplices, want["simplices"]), name
    assert np.array_equal(r.bary.view(np.uint32), want["bary"].view(np.uint32)), name
    assert np.array_equal(r.lam.view(np.uint64), want["lam"].view(np.uint64)), name
    assert np.array_equal(r.track_id, want["track_id"]), name
    assert np.array_equal(r.cells, cells), name
    assert r.n_tracks == len(set(r.track_id.tolist()))
    assert not r.scalar.any()


@pytest.mark.parametrize("name", list(contour_cases.FIBER_SURFACE_EXTRUDED_CASES))
def test_extruded_fiber_surface_matches_reference_fixture(ctx, name):
    """Features (spatial, over base edges, inside prisms), barycentrics with
    the centroid fallback, star-fan triangles and tracks equal the reference's
    one-worker run bit for bit."""
    case = contour_cases.FIBER_SURFACE_EXTRUDED_CASES[name]()
    g = np.load(os.path.join(FS_EXT_GOLD, f"{name}.npz"))
    assert_same_surface(run_fs_ext(ctx, case), g, g["cells"], name)


def test_extruded_fiber_surface_device_input_and_per_vertex_layout(ctx):
    case = contour_cases.FIBER_SURFACE_EXTRUDED_CASES["fs_ext_gauss_f64"]()
    a = run_fs_ext(ctx, case)
    for r in (run_fs_ext(ctx, case, device=True), run_fs_ext(ctx, case, layout=api.LAYOUT_PER_VERTEX)):
        assert_same_surface(r, {"simplices": a.simplices, "bary": a.bary, "lam": a.lam, "track_id": a.track_id},
                            a.cells)


def test_extruded_fiber_surface_vs_live_reference_and_restatement(ctx):
    case = contour_cases.fs_ext_seeded()
    r = run_fs_ext(ctx, case)
    keep: list = []
    mesh = bridge.make_extruded_mesh(case["coords"], case["cells"], case["n_layers"], keep)
    o = bridge.run_restatement(mesh, bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2,
                                                       sos_q=case["q"], keep=keep, fiber_thr=case["thresholds"]))
    assert len(r.track_id) > 500
    assert_same_surface(r, {"simplices": o.simplices, "bary": o.bary, "lam": o.lam, "track_id": o.track_id},
                        o.cells, "restatement")
    if bridge.ref_available():
        raw = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep)
        ref, cells = bridge.run_reference_fiber_surface(mesh, raw, case["thresholds"], one_thread=True)
        assert_same_surface(r, {"simplices": ref.simplices, "bary": ref.bary, "lam": ref.lam,
                                "track_id": ref.track_id}, cells, "reference")


def test_extruded_fiber_surface_python_mirror(ctx):
    case = contour_cases.FIBER_SURFACE_EXTRUDED_CASES["fs_ext_f32_thresholds"]()
    g = np.load(os.path.join(FS_EXT_GOLD, "fs_ext_f32_thresholds.npz"))
    base = api.UnstructuredSimplicialMesh(3, 3, case["coords"], case["cells"])
    mesh = api.ExtrudedSimplicialMesh(base, case["n_layers"])
    pred = api.FiberPredicate(var_names=["F", "G"], thresholds=case["thresholds"], sos_q=case["q"])
    eng = api.SimplicialEngine(mesh, pred, ctx)
    eng.execute({"F": case["fields"][0], "G": case["fields"][1]})
    assert_same_surface(eng.get_complex(), g, g["cells"])
