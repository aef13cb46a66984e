"""Seeded fiber and fiber-surface cases larger than the reference fixtures,
on the device against the C restatement's fiber mode (oracle/cp_oracle.c),
which reproduces the reference's fixtures and live runs
(tests/test_contour_oracle.py).  Fibers: features, both barycentric
precisions, tracks and star edges.  Fiber surfaces: features, barycentrics,
star-fan triangles and tracks, plus properties that hold at any size (track
ids are component minima, every triangle joins features of one track, no
triangle repeats)."""
import numpy as np
import pytest

import contour_cases
from ftk2_b200 import api
from oracle import bridge

pytestmark = pytest.mark.gpu


def restate(case):
    keep: list = []
    return bridge.run_restatement(
        bridge.make_regular_mesh(case["local_dims"]),
        bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep,
                          fiber_thr=case["thresholds"]))


def device(ctx, case, surface):
    keep: list = []
    mesh = api.regular_mesh_desc(case["local_dims"])
    fd = api.field_desc(list(case["fields"]), api.LAYOUT_SEPARATE, 2, keep=keep)
    if surface:
        return ctx.fiber_surface(mesh, fd, case["thresholds"], case["q"])
    return ctx.fiber(mesh, fd, case["thresholds"], case["q"])


def same_features(r, want):
    assert np.array_equal(r.simplices, want.simplices)
    assert np.array_equal(r.bary.view(np.uint32), want.bary.view(np.uint32))
    assert np.array_equal(r.lam.view(np.uint64), want.lam.view(np.uint64))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_fiber_seeded_160x144x12(ctx, dtype):
    case = contour_cases.fiber_seeded(dtype=dtype)
    want = restate(case)
    r = device(ctx, case, False)
    assert len(want.track_id) > 100
    same_features(r, want)
    assert np.array_equal(r.track_id, want.track_id)
    assert np.array_equal(r.edges, want.edges)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_fiber_surface_seeded_32x28x24x5(ctx, dtype):
    case = contour_cases.fiber_surface_seeded(dtype=dtype)
    want = restate(case)
    r = device(ctx, case, True)
    assert len(want.track_id) > 1000
    same_features(r, want)
    n = len(r.track_id)
    t = r.track_id.astype(np.int64)
    assert (t <= np.arange(n)).all() and (t[t] == t).all()
    assert r.n_tracks == len(np.unique(t))
    c = r.cells.astype(np.int64)
    assert len(c) > 0 and c.max() < n
    assert (t[c[:, 0]] == t[c[:, 1]]).all() and (t[c[:, 1]] == t[c[:, 2]]).all()
    assert len(np.unique(np.sort(c, axis=1), axis=0)) == len(c)
    assert np.array_equal(r.cells.astype(np.uint32), want.cells)
    assert np.array_equal(r.track_id, want.track_id)
