"""Level sets on the GPU (ftk2b_contour_extract) against the reference.

Every contour case is compared bit for bit with the fixtures the reference's
own engine produced (one worker thread; tests/golden/make_contour_golden.py)
and with the numpy restatement (oracle/contour_oracle.py): edge vertex ids,
float barycentrics and the field-precision values they came from, track ids,
scalars and the manifold cells of get_complex.  The moving sphere is the
reference's own level-set test (66418 vertices).  At full size (128^3 x 16)
the result is checked through properties that do not need the oracle."""
import hashlib
import os

import numpy as np
import pytest

import contour_cases
from ftk2_b200 import api
from oracle import contour_oracle as co

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "contour")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_gpu(ctx, case, field=None):
    mesh = api.regular_mesh_desc(case["local_dims"], case["offset"], case["global_dims"])
    return ctx.contour(mesh, case["field"] if field is None else field, case["threshold"], case["q"])


def as_dict(r):
    return {"simplices": r.simplices, "bary": r.bary, "lam": r.lam, "track_id": r.track_id,
            "scalar": r.scalar, "cells": r.cells}


def assert_same(got: dict, want: dict, name=""):
    assert np.array_equal(got["simplices"], want["simplices"]), name
    assert np.array_equal(got["bary"].view(np.uint32), want["bary"].view(np.uint32)), name
    assert np.array_equal(got["lam"].view(np.uint64), want["lam"].view(np.uint64)), name
    assert np.array_equal(got["track_id"], want["track_id"]), name
    assert np.array_equal(got["scalar"].view(np.uint32), want["scalar"].view(np.uint32)), name
    assert np.array_equal(got["cells"].astype(np.uint32), want["cells"].astype(np.uint32)), name


@pytest.mark.parametrize("name", list(contour_cases.CASES))
def test_contour_matches_reference_fixture(ctx, name):
    case = contour_cases.CASES[name]()
    r = run_gpu(ctx, case)
    got = as_dict(r)
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    for k, v in got.items():
        shape = tuple(int(x) for x in g[k + "_shape"])
        if v.size == 0 and int(np.prod(shape)) == 0:
            continue
        assert v.shape == shape, (name, k, v.shape, shape)
        assert digest(v) == str(g[k + "_sha256"]), (name, k)
    if name == "moving_sphere":
        assert len(r.track_id) == contour_cases.SPHERE_VERTICES
    assert r.n_tracks == len(set(r.track_id.tolist()))


@pytest.mark.parametrize("name", ["gauss_2d_f64", "ties_2d", "gauss_3d_f32_offset", "single_layer_3d"])
def test_contour_matches_restatement(ctx, name):
    case = contour_cases.CASES[name]()
    want = co.contour(case["field"], case["threshold"], case["local_dims"], case["offset"],
                      case["global_dims"], case["q"])
    assert_same(as_dict(run_gpu(ctx, case)), want, name)


def test_contour_device_and_per_vertex_inputs(ctx):
    torch = pytest.importorskip("torch")
    case = contour_cases.gauss_2d_f64()
    host = as_dict(run_gpu(ctx, case))
    dev = as_dict(run_gpu(ctx, case, torch.from_numpy(case["field"]).cuda()))
    assert_same(dev, host, "device input")
    flat = np.ascontiguousarray(case["field"].reshape(-1))  # global vertex order (offset 0)
    pv = as_dict(run_gpu(ctx, case, flat))
    assert_same(pv, host, "per-vertex input")


@pytest.mark.parametrize("seed,dims,dtype,thr", [
    (21, [17, 13, 5], np.float64, 0.0),
    (22, [9, 11, 7, 3], np.float32, 0.1),
    (23, [2, 2, 2], np.float64, 0.0),
    (24, [5, 4, 3, 2], np.float64, -0.05),
])
def test_contour_random_small_vs_restatement(ctx, seed, dims, dtype, thr):
    sp = dims[:-1]
    f = contour_cases.gaussian_potential(tuple(sp), dims[-1], seed=seed, n_blobs=5, dtype=dtype,
                                         sigma=(1.0, 3.0))
    case = dict(field=f, local_dims=dims, offset=None, global_dims=None, threshold=thr, q=1e6)
    want = co.contour(f, thr, dims, q=1e6)
    assert_same(as_dict(run_gpu(ctx, case)), want, str(seed))


def test_contour_full_size_properties(ctx):
    """128^3 x 16 float64 Gaussian-sum potential (32 blobs, the 3D plain
    drop-in generator's scalar), threshold 0: features in strict simplex
    order, every feature a mesh edge whose endpoint signs differ, cells sorted,
    unique and within one track, track ids the components' minima; a window
    of the same field identical to the restatement."""
    pytest.importorskip("torch")
    dims, nt = (128, 128, 128), 16
    q = 2.0 ** 20
    from ftk2_b200 import generate
    dev = generate.gaussian_potential_device(dims, nt, seed=1234, n_blobs=32)
    mesh = api.regular_mesh_desc([*dims, nt])
    r = ctx.contour(mesh, dev, 0.0, q)
    f = dev.cpu().numpy()
    n = len(r.track_id)
    assert n > 1000
    s = r.simplices.astype(np.int64)
    assert (s[:, 0] < s[:, 1]).all()
    d0 = np.diff(s[:, 0])
    assert (d0 >= 0).all() and (np.diff(s[:, 1])[d0 == 0] > 0).all()
    flat = f.reshape(-1)
    gid = np.arange(flat.size, dtype=np.uint64)
    pos = co.sos_positive(flat, gid, q)
    assert (pos[s[:, 0]] != pos[s[:, 1]]).all()
    lam = r.lam
    assert np.allclose(lam.sum(axis=1), 1.0, atol=1e-12)
    assert (lam >= -1e-9).all() and (lam <= 1 + 1e-9).all()
    t = r.track_id.astype(np.int64)
    assert (t <= np.arange(n)).all() and (t[t] == t).all()
    assert r.n_tracks == len(np.unique(t))
    c = r.cells.astype(np.int64)
    assert c.shape[1] == 4 and len(c) > n
    assert (np.diff(c, axis=1) > 0).all() and (c < n).all()
    # rows strictly increasing in lexicographic order (sorted and unique)
    dc = np.diff(c, axis=0)
    nz = dc != 0
    assert nz.any(axis=1).all()
    assert (dc[np.arange(len(dc)), nz.argmax(axis=1)] > 0).all()
    assert (t[c] == t[c[:, :1]]).all()
    win = np.ascontiguousarray(f[:6, :24, :20, :18])
    case = dict(field=win, local_dims=[18, 20, 24, 6], offset=None, global_dims=None, threshold=0.0, q=q)
    want = co.contour(win, 0.0, [18, 20, 24, 6], q=q)
    assert_same(as_dict(run_gpu(ctx, case)), want, "window")


@pytest.mark.parametrize("name", ["gauss_2d_f64", "single_layer_3d", "ties_2d"])
def test_contour_cpp_dropin_matches_restatement(tmp_path, name):
    """SimplicialEngine<T, ContourPredicate<T>> of include/ftk2b/engine.hpp,
    driven as the reference's own level-set test drives its engine."""
    import subprocess
    from ftk2_b200 import build as fb
    case = contour_cases.CASES[name]()
    exe = fb.build_contour_test()
    f = case["field"]
    path = tmp_path / "f.bin"
    f.tofile(path)
    dt = "f64" if f.dtype == np.float64 else "f32"
    out = tmp_path / "out.txt"
    r = subprocess.run([exe, str(path), dt, ",".join(str(x) for x in case["local_dims"]), repr(case["threshold"]),
                        repr(case["q"]), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    feats, cells = [], []
    for line in open(out):
        if line.startswith("F"):
            vs, bs, tr, sc = line[1:].split("|")
            feats.append(([int(x) for x in vs.split()], [int(x, 16) for x in bs.split()], int(tr), int(sc, 16)))
        elif line.startswith("C"):
            cells.append([int(x) for x in line.split()[2:]])
    want = co.contour(f, case["threshold"], case["local_dims"], q=case["q"])
    assert len(feats) == len(want["track_id"]) > 0
    assert np.array_equal(np.array([v for v, _, _, _ in feats], dtype=np.uint64), want["simplices"])
    assert np.array_equal(np.array([b for _, b, _, _ in feats], dtype=np.uint32), want["bary"].view(np.uint32))
    assert np.array_equal(np.array([t for _, _, t, _ in feats], dtype=np.uint64), want["track_id"])
    assert np.array_equal(np.array([s for _, _, _, s in feats], dtype=np.uint32), want["scalar"].view(np.uint32))
    assert np.array_equal(np.array(cells, dtype=np.uint32).reshape(-1, want["cells"].shape[1]), want["cells"])


EXT_GOLD = os.path.join(os.path.dirname(__file__), "golden", "contour_extruded")


@pytest.mark.parametrize("name", list(contour_cases.EXTRUDED_CASES))
def test_contour_extruded_matches_reference_fixture(ctx, name):
    """Level sets on ExtrudedSimplicialMesh(UnstructuredSimplicialMesh, L):
    edge features (spatial, vertical, prism diagonals), barycentrics, tracks
    and manifold cells identical to the reference engine's."""
    case = contour_cases.EXTRUDED_CASES[name]()
    g = np.load(os.path.join(EXT_GOLD, f"{name}.npz"))
    keep: list = []
    mesh = api.extruded_mesh_desc(case["coords"].shape[0], case["cells"], case["n_layers"], keep)
    r = ctx.contour(mesh, api.field_desc([case["field"]], api.LAYOUT_SEPARATE, 1, keep=keep), case["threshold"],
                    case["q"])
    assert_same(as_dict(r), {k: g[k] for k in ("simplices", "bary", "lam", "track_id", "scalar", "cells")}, name)
    assert r.n_tracks == len(set(r.track_id.tolist()))
