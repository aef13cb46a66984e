"""The Python mirror of the reference's engine (ftk2_b200.api.SimplicialEngine)
routes each predicate to its C-ABI entry point with the reference's variable
and threshold semantics (predicate.hpp:22-64, 135-183, 341-362).  Host logic
only: a recording stand-in for the context takes the calls."""
import numpy as np

from ftk2_b200 import api


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
