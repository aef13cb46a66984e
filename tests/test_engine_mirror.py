"""The Python mirror of the reference's engine (ftk2_b200.api.SimplicialEngine)
routes each predicate to its C-ABI entry point with the reference's variable
and threshold semantics (predicate.hpp:50-128, 136-181, 341-387).  On the CPU a
recording stand-in for the context takes the calls; the gpu-marked tests run
the mirror on the device against the reference's fixtures."""
import os

import numpy as np
import pytest

import contour_cases
from ftk2_b200 import api

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


class Recorder:
    def __init__(self):
        self.calls = []

    def _rec(self, name, mesh, fld, *rest):
        self.calls.append((name, mesh.kind, mesh.ndims, fld.ncomp, fld.layout, fld.nd, rest))
        return name

    def extract(self, mesh, fld, prm):
        return self._rec("extract", mesh, fld, prm.sos_q)

    def contour(self, mesh, fld, threshold, sos_q):
        return self._rec("contour", mesh, fld, threshold, sos_q)

    def fiber(self, mesh, fld, thresholds, sos_q):
        return self._rec("fiber", mesh, fld, tuple(thresholds), sos_q)

    def fiber_surface(self, mesh, fld, thresholds, sos_q):
        return self._rec("fiber_surface", mesh, fld, tuple(thresholds), sos_q)


def test_contour_predicate_routes_to_level_sets():
    rec = Recorder()
    s = np.zeros((4, 6, 7))
    e = api.SimplicialEngine(api.RegularSimplicialMesh([7, 6, 4]),
                             api.ContourPredicate(var_name="S", threshold=0.25, sos_q=2.0 ** 20), ctx=rec)
    e.execute({"S": s})
    assert e.get_complex() == "contour"
    name, kind, ndims, ncomp, layout, nd, rest = rec.calls[0]
    assert (kind, ndims, ncomp, layout, nd) == (api.MESH_REGULAR, 3, 1, api.LAYOUT_SEPARATE, 3)
    assert rest == (0.25, 2.0 ** 20)
    # variables passed to execute win over the predicate's name
    e.execute({"T": s}, ["T"])
    assert rec.calls[1][0] == "contour"


def test_fiber_predicate_routes_by_mesh_dimension():
    rec = Recorder()
    f2, f3 = np.zeros((3, 5, 6)), np.zeros((3, 4, 5, 6))
    p = api.FiberPredicate(var_names=["F", "G"], thresholds=(0.1, -0.2))
    api.SimplicialEngine(api.RegularSimplicialMesh([6, 5, 3]), p, ctx=rec).execute({"F": f2, "G": f2})
    api.SimplicialEngine(api.RegularSimplicialMesh([6, 5, 4, 3]), p, ctx=rec).execute({"F": f3, "G": f3})
    assert [c[0] for c in rec.calls] == ["fiber", "fiber_surface"]
    assert rec.calls[0][3] == 2 and rec.calls[0][6][0] == (0.1, -0.2)
    # extruded triangle meshes read per-vertex arrays
    base = api.UnstructuredSimplicialMesh(2, 2, np.zeros((4, 3)), np.array([[0, 1, 2], [1, 2, 3]]))
    v = np.zeros(4 * 3)
    api.SimplicialEngine(api.ExtrudedSimplicialMesh(base, 2), p, ctx=rec).execute({"F": v, "G": v})
    name, kind, ndims, ncomp, layout, nd, _ = rec.calls[2]
    assert (name, kind, ndims, layout, nd) == ("fiber", api.MESH_EXTRUDED, 3, api.LAYOUT_PER_VERTEX, 1)


def test_critical_point_predicate_still_extracts():
    rec = Recorder()
    v = np.zeros((4, 5, 6, 2))
    api.SimplicialEngine(api.RegularSimplicialMesh([6, 5, 4]),
                         api.CriticalPointPredicate(2, vector_var_name="v"), ctx=rec).execute({"v": v})
    assert rec.calls[0][0] == "extract" and rec.calls[0][4] == api.LAYOUT_MULTICOMPONENT


# On the GPU: the mirror's results are the reference engine's fixtures (and,
# for the regular level sets, whose fixtures hold digests, the restatement).


def _same(r, g, keys):
    for k in keys:
        a, b = getattr(r, k), g[k]
        if k in ("bary", "scalar"):
            a, b = a.view(np.uint32), b.view(np.uint32)
        elif k == "lam":
            a, b = a.view(np.uint64), b.view(np.uint64)
        elif k == "cells":
            a, b = a.astype(np.uint32), b.astype(np.uint32)
        assert np.array_equal(a, b), k


def _regular(case):
    return api.RegularSimplicialMesh(case["local_dims"], case["offset"], case["global_dims"])


def _extruded(case):
    cells = case["cells"]
    base = api.UnstructuredSimplicialMesh(3, cells.shape[1] - 1, case["coords"], cells)
    return api.ExtrudedSimplicialMesh(base, case["n_layers"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["gauss_2d_f64", "moving_sphere"])
def test_gpu_contour_predicate_regular(ctx, name):
    from oracle import contour_oracle as co
    case = contour_cases.CASES[name]()
    e = api.SimplicialEngine(_regular(case), api.ContourPredicate("s", case["threshold"], case["q"]), ctx=ctx)
    e.execute({"s": case["field"]})
    r = e.get_complex()
    want = co.contour(case["field"], case["threshold"], case["local_dims"], case["offset"],
                      case["global_dims"], case["q"])
    assert len(r.track_id) > 0
    for k in ("simplices", "track_id", "cells"):
        assert np.array_equal(getattr(r, k).astype(want[k].dtype), want[k]), k
    assert np.array_equal(r.lam.view(np.uint64), want["lam"].view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(contour_cases.EXTRUDED_CASES))
def test_gpu_contour_predicate_extruded(ctx, name):
    case = contour_cases.EXTRUDED_CASES[name]()
    g = np.load(os.path.join(GOLDEN, "contour_extruded", f"{name}.npz"))
    e = api.SimplicialEngine(_extruded(case), api.ContourPredicate("s", case["threshold"], case["q"]), ctx=ctx)
    e.execute({"s": case["field"]})
    r = e.get_complex()
    assert len(r.track_id) == len(g["track_id"]) > 0
    _same(r, g, ("simplices", "bary", "lam", "track_id", "cells"))


@pytest.mark.gpu
def test_gpu_fiber_predicate_regular_and_extruded(ctx):
    case = contour_cases.FIBER_CASES["fiber_gauss_f64"]()
    g = np.load(os.path.join(GOLDEN, "fiber", "fiber_gauss_f64.npz"))
    e = api.SimplicialEngine(_regular(case), api.FiberPredicate(["f", "g"], case["thresholds"], case["q"]), ctx=ctx)
    e.execute({"f": case["fields"][0], "g": case["fields"][1]})
    r = e.get_complex()
    assert len(r.track_id) == len(g["track_id"]) > 0
    _same(r, g, ("simplices", "bary", "lam", "track_id", "edges"))

    case = contour_cases.FIBER_EXTRUDED_CASES["fiber_ext_tri"]()
    g = np.load(os.path.join(GOLDEN, "fiber_extruded", "fiber_ext_tri.npz"))
    e = api.SimplicialEngine(_extruded(case), api.FiberPredicate(["f", "g"], case["thresholds"], case["q"]), ctx=ctx)
    e.execute({"f": case["fields"][0], "g": case["fields"][1]})
    r = e.get_complex()
    assert len(r.track_id) == len(g["track_id"]) > 0
    _same(r, g, ("simplices", "bary", "lam", "track_id", "edges"))


@pytest.mark.gpu
def test_gpu_fiber_predicate_surfaces(ctx):
    case = contour_cases.FIBER_SURFACE_CASES["fs_gauss_f64"]()
    g = np.load(os.path.join(GOLDEN, "fiber_surface", "fs_gauss_f64.npz"))
    e = api.SimplicialEngine(_regular(case), api.FiberPredicate(["f", "g"], case["thresholds"], case["q"]), ctx=ctx)
    e.execute({"f": case["fields"][0], "g": case["fields"][1]})
    r = e.get_complex()
    assert len(r.track_id) == len(g["track_id"]) > 0
    _same(r, g, ("simplices", "bary", "lam", "track_id", "cells"))


def test_level_set_results_are_views_freed_after_the_last_one():
    """Level-set and fiber-surface results are numpy views of the library's
    result memory; the result is freed once, after the last view goes."""
    import ctypes as C
    import gc
    n, c = 5, 3
    simp = (C.c_uint64 * (2 * n))(*range(10, 20))
    lam = (C.c_double * (2 * n))(*[i / 8 for i in range(2 * n)])
    bary = (C.c_float * (2 * n))(*[i / 4 for i in range(2 * n)])
    track = (C.c_uint64 * n)(0, 0, 2, 2, 4)
    scal = (C.c_float * n)(*([0.5] * n))
    cells = (C.c_uint32 * (3 * c))(*range(9))
    r = api.ContourResultC(n_features=n, cell_dim=2, n_cells=c, n_tracks=3, n_simplices=77, device_ms=1.5)
    r.simplices, r.lambda_, r.barycentric = simp, lam, bary
    r.track_id, r.scalar, r.cells = track, scal, cells
    freed = []
    out = C.pointer(r)
    res = api._contour_from_c(out.contents, api._CResultOwner(lambda p: freed.append(p.contents.n_features), out))
    assert res.simplices.shape == (n, 2) and res.simplices[4].tolist() == [18, 19]
    assert res.lam[1].tolist() == [0.25, 0.375] and res.bary.dtype == np.float32
    assert res.track_id.tolist() == [0, 0, 2, 2, 4] and res.cells.shape == (c, 3) and res.cells[2, 2] == 8
    assert (res.n_tracks, res.n_simplices, res.device_ms) == (3, 77, 1.5)
    keep = res.cells[1:]
    del res
    gc.collect()
    assert freed == []
    assert keep.tolist() == [[3, 4, 5], [6, 7, 8]]
    del keep
    gc.collect()
    assert freed == [n]

    # nothing to view: freed at once, empty arrays of the right shapes
    e = api.ContourResultC(n_features=0, cell_dim=1, n_cells=0)
    out = C.pointer(e)
    res = api._contour_from_c(out.contents, api._CResultOwner(lambda p: freed.append("empty"), out))
    gc.collect()
    assert freed[-1] == "empty" and res.simplices.shape == (0, 2) and res.cells.shape == (0, 2)
