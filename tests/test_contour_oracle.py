"""The level-set restatement (oracle/contour_oracle.py) is pinned before the
GPU path is checked against it.

1. It reproduces the reference's own known answer: 66418 feature vertices on
   the moving sphere (tests/test_examples.cpp:225-256).
2. On every contour case it reproduces, bit for bit, the fixtures that the
   reference's own engine produced (tests/golden/make_contour_golden.py):
   simplices, float and widened barycentrics, track ids, scalars and the
   manifold cells of get_complex.
3. Where the reference build is present, it matches a live reference run.
"""
import hashlib
import os

import numpy as np
import pytest

import contour_cases
from oracle import bridge
from oracle import contour_oracle as co

GOLD = os.path.join(os.path.dirname(__file__), "golden", "contour")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def restate(case):
    return co.contour(case["field"], case["threshold"], case["local_dims"], case["offset"],
                      case["global_dims"], case["q"])


def check_against_fixture(name, res):
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    for k in ("simplices", "bary", "lam", "track_id", "scalar", "cells"):
        a = res[k]
        if k == "cells":
            a = a.astype(np.uint32).reshape(-1, g["cells_shape"][1] if g["cells_shape"].size > 1 else 1) \
                if a.size else a
        assert tuple(a.shape) == tuple(g[k + "_shape"]) or a.size == 0 == int(np.prod(g[k + "_shape"])), k
        if a.size:
            assert digest(a) == str(g[k + "_sha256"]), (name, k)


def test_sphere_known_answer():
    res = restate(contour_cases.moving_sphere())
    assert len(res["track_id"]) == contour_cases.SPHERE_VERTICES
    assert res["cells"].shape[1] == 4  # 3D+t: tets


@pytest.mark.parametrize("name", list(contour_cases.CASES))
def test_restatement_matches_reference_fixtures(name):
    case = contour_cases.CASES[name]()
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    assert digest(case["field"]) == str(g["input_sha256"]), "generator drift"
    check_against_fixture(name, restate(case))


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name", ["gauss_2d_f64", "ties_2d", "gauss_3d_f32_offset"])
def test_restatement_matches_live_reference(name):
    case = contour_cases.CASES[name]()
    keep: list = []
    mesh = bridge.make_regular_mesh(case["local_dims"], case["offset"], case["global_dims"])
    fld = bridge.make_field([case["field"]], bridge.LAYOUT_SEPARATE, 1, sos_q=case["q"], keep=keep)
    ref, cells = bridge.run_reference_contour(mesh, fld, case["threshold"])
    res = restate(case)
    assert len(ref.track_id) > 0
    assert np.array_equal(res["simplices"], ref.simplices)
    assert np.array_equal(res["bary"].view(np.uint32), ref.bary.view(np.uint32))
    assert np.array_equal(res["lam"].view(np.uint64), ref.lam.view(np.uint64))
    assert np.array_equal(res["track_id"], ref.track_id)
    assert np.array_equal(res["cells"], cells)


def test_sos_sign_ties_follow_vertex_parity():
    adj = np.array([0.0, 0.0, 4e-7, -4e-7, 6e-7, -6e-7])
    gid = np.array([2, 3, 5, 6, 7, 8], dtype=np.uint64)
    # 0 -> parity; |v|*1e6 + 0.5 below 1 -> parity; above -> its own sign
    assert co.sos_positive(adj, gid, 1e6).tolist() == [True, False, False, True, True, False]


FIBER_GOLD = os.path.join(os.path.dirname(__file__), "golden", "fiber")


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name", list(contour_cases.FIBER_CASES))
def test_fiber_reference_reproduces_fixtures_on_one_and_many_workers(name):
    """The fiber fixtures are the reference engine's output; its result does
    not depend on its worker count (star centres go by simplex code)."""
    case = contour_cases.FIBER_CASES[name]()
    g = np.load(os.path.join(FIBER_GOLD, f"{name}.npz"))
    assert digest(np.concatenate([a.reshape(-1) for a in case["fields"]])) == str(g["input_sha256"])
    for one in (False, True):
        keep: list = []
        mesh = bridge.make_regular_mesh(case["local_dims"], case["offset"], case["global_dims"])
        fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep)
        r = bridge.run_reference_fiber(mesh, fld, case["thresholds"], one_thread=one)
        assert len(r.track_id) > 0
        assert np.array_equal(r.simplices, g["simplices"])
        assert np.array_equal(r.bary.view(np.uint32), g["bary"].view(np.uint32))
        assert np.array_equal(r.lam.view(np.uint64), g["lam"].view(np.uint64))
        assert np.array_equal(r.track_id, g["track_id"])
        assert np.array_equal(r.edges, g["edges"])


def test_fiber_fixture_exercises_the_centroid_fallback():
    """Near the quantum 1/Q the reference keeps simplices whose solve fails,
    at 1/3 each (predicate.hpp:354); the fixture holds such features."""
    g = np.load(os.path.join(FIBER_GOLD, "fiber_near_quantum.npz"))
    third = np.float64(1.0) / 3.0
    assert (g["lam"] == third).all(axis=1).sum() > 10


FS_GOLD = os.path.join(os.path.dirname(__file__), "golden", "fiber_surface")


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name", list(contour_cases.FIBER_SURFACE_CASES))
def test_fiber_surface_reference_reproduces_fixtures(name):
    """Fiber surfaces (3D+t): the fixtures are the reference engine's output
    (features, barycentrics, tracks, star-fan triangles)."""
    case = contour_cases.FIBER_SURFACE_CASES[name]()
    g = np.load(os.path.join(FS_GOLD, f"{name}.npz"))
    assert digest(np.concatenate([a.reshape(-1) for a in case["fields"]])) == str(g["input_sha256"])
    keep: list = []
    mesh = bridge.make_regular_mesh(case["local_dims"], case["offset"], case["global_dims"])
    fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep)
    r, cells = bridge.run_reference_fiber_surface(mesh, fld, case["thresholds"])
    assert len(r.track_id) > 0 and len(cells) > 0
    assert np.array_equal(r.simplices, g["simplices"])
    assert np.array_equal(r.lam.view(np.uint64), g["lam"].view(np.uint64))
    assert np.array_equal(r.track_id, g["track_id"])
    assert np.array_equal(cells, g["cells"])


def test_fiber_surface_fixture_exercises_the_centroid_fallback():
    g = np.load(os.path.join(FS_GOLD, "fs_near_quantum.npz"))
    assert (g["lam"] == np.float64(1.0) / 3.0).all(axis=1).sum() > 10


EXT_GOLD = os.path.join(os.path.dirname(__file__), "golden", "contour_extruded")


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name", list(contour_cases.EXTRUDED_CASES))
def test_extruded_level_set_reference_reproduces_fixtures(name):
    """Level sets on ExtrudedSimplicialMesh: the fixtures are the one-worker
    reference engine's output (its patching numbers the prism diagonals in the
    order it meets them)."""
    case = contour_cases.EXTRUDED_CASES[name]()
    g = np.load(os.path.join(EXT_GOLD, f"{name}.npz"))
    assert digest(case["field"]) == str(g["input_sha256"])
    keep: list = []
    mesh = bridge.make_extruded_mesh(case["coords"], case["cells"], case["n_layers"], keep)
    fld = bridge.make_field([case["field"]], bridge.LAYOUT_SEPARATE, 1, sos_q=case["q"], keep=keep)
    r, cells = bridge.run_reference_contour(mesh, fld, case["threshold"])
    assert len(r.track_id) > 0
    assert np.array_equal(r.simplices, g["simplices"])
    assert np.array_equal(r.lam.view(np.uint64), g["lam"].view(np.uint64))
    assert np.array_equal(r.track_id, g["track_id"])
    assert np.array_equal(cells, g["cells"])


@pytest.mark.parametrize("name", list(contour_cases.EXTRUDED_CASES))
def test_extruded_restatement_matches_reference_fixtures(name):
    case = contour_cases.EXTRUDED_CASES[name]()
    g = np.load(os.path.join(EXT_GOLD, f"{name}.npz"))
    res = co.contour_extruded(case["field"], case["cells"], case["coords"].shape[0], case["n_layers"],
                              case["threshold"], case["q"])
    for k in ("simplices", "track_id", "cells"):
        assert np.array_equal(res[k], g[k]), (name, k)
    assert np.array_equal(res["bary"].view(np.uint32), g["bary"].view(np.uint32))
    assert np.array_equal(res["lam"].view(np.uint64), g["lam"].view(np.uint64))


FIBER_EXT_GOLD = os.path.join(os.path.dirname(__file__), "golden", "fiber_extruded")


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name", list(contour_cases.FIBER_EXTRUDED_CASES))
def test_extruded_fiber_reference_reproduces_fixtures(name):
    case = contour_cases.FIBER_EXTRUDED_CASES[name]()
    g = np.load(os.path.join(FIBER_EXT_GOLD, f"{name}.npz"))
    keep: list = []
    r = bridge.run_reference_fiber(bridge.make_extruded_mesh(case["coords"], case["cells"], case["n_layers"], keep),
                                   bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"],
                                                     keep=keep), case["thresholds"])
    assert len(r.track_id) > 0
    assert np.array_equal(r.simplices, g["simplices"])
    assert np.array_equal(r.lam.view(np.uint64), g["lam"].view(np.uint64))
    assert np.array_equal(r.track_id, g["track_id"])
    assert np.array_equal(r.edges, g["edges"])


def _same_fiber(r, g, name):
    assert len(r.track_id) == len(g["track_id"]) > 0, name
    assert np.array_equal(r.simplices, g["simplices"]), name
    assert np.array_equal(r.bary.view(np.uint32), g["bary"].view(np.uint32)), name
    assert np.array_equal(r.lam.view(np.uint64), g["lam"].view(np.uint64)), name
    assert np.array_equal(r.track_id, g["track_id"]), name
    assert np.array_equal(r.edges, g["edges"]), name


@pytest.mark.parametrize("name", list(contour_cases.FIBER_CASES))
def test_fiber_restatement_matches_reference_fixtures(name):
    """The C restatement's fiber mode (oracle/cp_oracle.c: values less the
    thresholds in the field precision, centroid where the solve fails,
    predicate.hpp:341-362) reproduces the reference engine's fiber fixtures on
    regular 2D+t meshes, offsets and near-quantum ties included."""
    case = contour_cases.FIBER_CASES[name]()
    g = np.load(os.path.join(FIBER_GOLD, f"{name}.npz"))
    keep: list = []
    mesh = bridge.make_regular_mesh(case["local_dims"], case["offset"], case["global_dims"])
    fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep,
                            fiber_thr=case["thresholds"])
    _same_fiber(bridge.run_restatement(mesh, fld), g, name)


@pytest.mark.parametrize("name", list(contour_cases.FIBER_EXTRUDED_CASES))
def test_extruded_fiber_restatement_matches_reference_fixtures(name):
    case = contour_cases.FIBER_EXTRUDED_CASES[name]()
    g = np.load(os.path.join(FIBER_EXT_GOLD, f"{name}.npz"))
    keep: list = []
    mesh = bridge.make_extruded_mesh(case["coords"], case["cells"], case["n_layers"], keep)
    fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_PER_VERTEX, 2, sos_q=case["q"], keep=keep,
                            fiber_thr=case["thresholds"])
    _same_fiber(bridge.run_restatement(mesh, fld), g, name)


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
def test_fiber_restatement_matches_live_reference_seeded():
    """A larger seeded fiber case (96x80x10 f32, ~500 features, centroid
    fallbacks among them): restatement == live reference engine."""
    case = contour_cases.fiber_seeded((96, 80), 10)
    keep: list = []
    mesh = bridge.make_regular_mesh(case["local_dims"])
    ref = bridge.run_reference_fiber(mesh, bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2,
                                                             sos_q=case["q"], keep=keep), case["thresholds"])
    fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep,
                            fiber_thr=case["thresholds"])
    _same_fiber(bridge.run_restatement(mesh, fld),
                {k: getattr(ref, k) for k in ("simplices", "bary", "lam", "track_id", "edges")}, "fiber_seeded")


@pytest.mark.parametrize("name", list(contour_cases.FIBER_SURFACE_CASES))
def test_fiber_surface_restatement_matches_reference_fixtures(name):
    """Fiber surfaces on 3D+t meshes: the restatement's triangle features (the
    50 triangle types of the 4-D Kuhn cube, the 2-D origin test, the solve
    with its centroid fallback), its star-fan triangles
    (form_general_manifold_patches with k = 2) and its tracks equal the
    reference's bit for bit."""
    case = contour_cases.FIBER_SURFACE_CASES[name]()
    g = np.load(os.path.join(FS_GOLD, f"{name}.npz"))
    keep: list = []
    mesh = bridge.make_regular_mesh(case["local_dims"], case["offset"], case["global_dims"])
    r = bridge.run_restatement(mesh, bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2,
                                                       sos_q=case["q"], keep=keep, fiber_thr=case["thresholds"]))
    assert len(r.track_id) == len(g["track_id"]) > 0
    assert np.array_equal(r.simplices, g["simplices"])
    assert np.array_equal(r.lam.view(np.uint64), g["lam"].view(np.uint64))
    assert np.array_equal(r.bary.view(np.uint32), g["bary"].view(np.uint32))
    assert np.array_equal(r.cells, g["cells"])
    assert np.array_equal(r.track_id, g["track_id"])


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
def test_fiber_surface_restatement_matches_live_reference_seeded():
    case = contour_cases.fiber_surface_seeded((16, 14, 12), 4)
    keep: list = []
    mesh = bridge.make_regular_mesh(case["local_dims"])
    ref, cells = bridge.run_reference_fiber_surface(
        mesh, bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep),
        case["thresholds"])
    r = bridge.run_restatement(mesh, bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2,
                                                       sos_q=case["q"], keep=keep, fiber_thr=case["thresholds"]))
    assert len(r.track_id) > 100 and len(cells) > 0
    assert np.array_equal(r.simplices, ref.simplices)
    assert np.array_equal(r.lam.view(np.uint64), ref.lam.view(np.uint64))
    assert np.array_equal(r.track_id, ref.track_id)
    assert np.array_equal(r.cells, cells)


FS_EXT_GOLD = os.path.join(os.path.dirname(__file__), "golden", "fiber_surface_extruded")


def _fs_ext_inputs(case, keep, fiber=True):
    mesh = bridge.make_extruded_mesh(case["coords"], case["cells"], case["n_layers"], keep)
    fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep,
                            fiber_thr=case["thresholds"] if fiber else None)
    return mesh, fld


def _same_surface(r, cells, g, name):
    assert len(r.track_id) == len(g["track_id"]) > 0, name
    assert np.array_equal(r.simplices, g["simplices"]), name
    assert np.array_equal(r.lam.view(np.uint64), g["lam"].view(np.uint64)), name
    assert np.array_equal(r.bary.view(np.uint32), g["bary"].view(np.uint32)), name
    assert np.array_equal(r.track_id, g["track_id"]), name
    assert np.array_equal(cells, g["cells"]), name


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name", list(contour_cases.FIBER_SURFACE_EXTRUDED_CASES))
def test_extruded_fiber_surface_reference_reproduces_fixtures(name):
    case = contour_cases.FIBER_SURFACE_EXTRUDED_CASES[name]()
    g = np.load(os.path.join(FS_EXT_GOLD, f"{name}.npz"))
    keep: list = []
    mesh, fld = _fs_ext_inputs(case, keep, fiber=False)
    r, cells = bridge.run_reference_fiber_surface(mesh, fld, case["thresholds"], one_thread=True)
    _same_surface(r, cells, g, name)


@pytest.mark.parametrize("name", list(contour_cases.FIBER_SURFACE_EXTRUDED_CASES))
def test_extruded_fiber_surface_restatement_matches_reference_fixtures(name):
    """Fiber surfaces on ExtrudedSimplicialMesh over tets: the restatement's
    phase-1 triangles, the prism-interior triangles numbered in the order
    sequential patching meets them, its star-fan triangles and tracks equal
    the reference's one-worker run bit for bit (centroid fallbacks and ties
    included)."""
    case = contour_cases.FIBER_SURFACE_EXTRUDED_CASES[name]()
    g = np.load(os.path.join(FS_EXT_GOLD, f"{name}.npz"))
    keep: list = []
    r = bridge.run_restatement(*_fs_ext_inputs(case, keep))
    _same_surface(r, r.cells, g, name)


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
def test_extruded_fiber_surface_restatement_matches_live_reference_seeded():
    case = contour_cases.fs_ext_seeded()
    keep: list = []
    mesh, raw = _fs_ext_inputs(case, keep, fiber=False)
    ref, cells = bridge.run_reference_fiber_surface(mesh, raw, case["thresholds"], one_thread=True)
    r = bridge.run_restatement(*_fs_ext_inputs(case, keep))
    assert len(r.track_id) > 500
    _same_surface(r, r.cells, {"simplices": ref.simplices, "lam": ref.lam, "bary": ref.bary,
                               "track_id": ref.track_id, "cells": cells}, "fs_ext_seeded")
