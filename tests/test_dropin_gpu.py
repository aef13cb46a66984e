"""The C++ drop-in header (include/ftk2b/engine.hpp) used like the reference's
engine: a C++ program builds a RegularSimplicialMesh and a
CriticalPointPredicate, calls execute() and get_complex(), and its
FeatureComplex matches the reference engine's own output on config 1."""
import os
import struct
import subprocess

import numpy as np
import pytest

import cases
from ftk2_b200 import build as fb

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_cpp_dropin_matches_reference(tmp_path):
    exe = fb.build_dropin_test()
    case = cases.c1_analytic_2d()
    field = tmp_path / "c1.f64"
    np.ascontiguousarray(case.arrays).tofile(field)
    out = tmp_path / "c1.out"
    subprocess.run([exe, str(field), str(out)], check=True, timeout=120)
    buf = out.read_bytes()
    n = struct.unpack_from("<Q", buf, 0)[0]
    rec = np.dtype([("v", "<u8", 3), ("b", "<f4", 3), ("t", "<u8")])
    feats = np.frombuffer(buf, dtype=rec, count=n, offset=8)
    off = 8 + n * rec.itemsize
    ne = struct.unpack_from("<Q", buf, off)[0]
    edges = np.frombuffer(buf, dtype="<u4", count=2 * ne, offset=off + 8).reshape(ne, 2)
    z = np.load(os.path.join(GOLDEN, "c1_analytic_2d.npz"))
    assert np.array_equal(feats["v"], z["simplices"])
    assert np.array_equal(feats["b"], z["bary"])
    assert np.array_equal(feats["t"], z["track_id"])
    assert np.array_equal(edges, z["edges"])
