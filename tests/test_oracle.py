"""The oracle is pinned before it is trusted.

1. Its primitives reproduce the reference's own unit-test vectors
   (tests/test_sos.cpp:29-71, tests/test_zero_crossing.cpp:25-66,
   tests/test_3d_cp.cpp:33-60, mesh.hpp:231-237 simplex-type counts behind
   tests/test_mesh.cpp:41-63).
2. On every golden case it reproduces, bit for bit, the fixtures that the
   reference's own engine produced (tests/golden/make_golden.py).
3. Where the reference build is present, it matches a live reference run on a
   few more seeded inputs.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import bridge
import cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def olib():
    lib = C.CDLL(bridge.ORC_LIB)
    lib.cporacle_sos_sign.argtypes = [C.c_double, C.c_uint64, C.c_double]
    lib.cporacle_det2.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_uint64,
                                  C.c_uint64, C.c_double]
    lib.cporacle_inside.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.c_double]
    lib.cporacle_solve.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return lib


def dp(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def test_sos_sign_vectors(olib):
    # tests/test_sos.cpp:36-39
    assert olib.cporacle_sos_sign(1.0, 0, 1e6) == 1
    assert olib.cporacle_sos_sign(-1.0, 0, 1e6) == -1
    assert olib.cporacle_sos_sign(0.0, 0, 1e6) == 1


def test_det2_tie_break_antisymmetric(olib):
    # tests/test_sos.cpp:42-50: collinear with the origin, tie broken by index order
    a, pa = dp([1.0, 0.0])
    b, pb = dp([2.0, 0.0])
    s1 = olib.cporacle_det2(pa, pb, 0, 1, 1e6)
    s2 = olib.cporacle_det2(pa, pb, 1, 0, 1e6)
    assert s1 != 0 and s1 == -s2


def test_zero_crossing_vectors(olib):
    # tests/test_zero_crossing.cpp:38-63
    v2, p2 = dp([[-0.25, -0.25], [0.75, -0.25], [-0.25, 0.75]])
    lam = np.zeros(4)
    assert olib.cporacle_solve(2, 1, p2, lam.ctypes.data_as(C.POINTER(C.c_double)))
    np.testing.assert_allclose(lam[:3], [0.5, 0.25, 0.25], atol=1e-9)
    v3, p3 = dp([[-0.2, -0.2, -0.2], [0.8, -0.2, -0.2], [-0.2, 0.8, -0.2], [-0.2, -0.2, 0.8]])
    assert olib.cporacle_solve(3, 1, p3, lam.ctypes.data_as(C.POINTER(C.c_double)))
    np.testing.assert_allclose(lam, [0.4, 0.2, 0.2, 0.2], atol=1e-9)


def test_single_tet_known_answer(olib):
    # tests/test_3d_cp.cpp:33-58: inside, and lambda == 0.25 exactly
    v, p = dp([[-0.25, -0.25, -0.25], [0.75, -0.25, -0.25], [-0.25, 0.75, -0.25],
               [-0.25, -0.25, 0.75]])
    idx = np.array([0, 1, 2, 3], dtype=np.uint64)
    assert olib.cporacle_inside(3, p, idx.ctypes.data_as(C.POINTER(C.c_uint64)), 1e6)
    lam = np.zeros(4)
    assert olib.cporacle_solve(3, 1, p, lam.ctypes.data_as(C.POINTER(C.c_double)))
    assert list(lam) == [0.25, 0.25, 0.25, 0.25]


def test_simplex_type_counts(olib):
    # cpu_get_num_simplex_types (mesh.hpp:231-237); test_mesh.cpp:52,63 count
    # 2 triangles per square and 6 tets per cube
    want = {(2, 1): 3, (2, 2): 2, (3, 1): 7, (3, 2): 12, (3, 3): 6, (4, 1): 15, (4, 2): 50,
            (4, 3): 60, (4, 4): 24}
    for (d, m), n in want.items():
        assert olib.cporacle_chain_count(d, m) == n


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return {k: z[k] for k in z.files}


def assert_same(res, g, exact_lambda=True):
    assert res.simplices.shape == g["simplices"].shape
    assert np.array_equal(res.simplices, g["simplices"])
    assert np.array_equal(res.track_id, g["track_id"])
    assert np.array_equal(res.edges, g["edges"])
    assert np.array_equal(res.bary, g["bary"])
    assert np.array_equal(res.scalar, g["scalar"])
    assert np.array_equal(res.type, g["type"])
    if exact_lambda:
        assert np.array_equal(res.lam, g["lam"])


@pytest.mark.parametrize("name", sorted(cases.GOLDEN_CASES))
def test_restatement_matches_reference_fixtures(name):
    case = cases.GOLDEN_CASES[name]()
    g = load_golden(name)
    assert str(g["input_sha256"]) == case.input_digest(), "input generator drifted"
    keep: list = []
    mesh, fld = cases.oracle_inputs(case, keep)
    res = bridge.run_restatement(mesh, fld)
    assert_same(res, g)


LIVE = [
    ("gauss2d_seed", lambda: cases.Case(
        "g2", "regular", 2, cases.MULTI,
        cases.S.gaussian_sum_gradient((36, 30), 7, seed=21, n_blobs=10, sigma=(2, 4)), 1e6, [36, 30, 7])),
    ("gauss3d_f32_offset", lambda: cases.Case(
        "g3", "regular", 3, cases.MULTI,
        cases.S.gaussian_sum_gradient((12, 11, 10), 4, seed=33, n_blobs=12, dtype=np.float32,
                                      sigma=(2, 3)), 2.0 ** 20, [10, 9, 8, 3], [1, 1, 2, 1],
        [12, 11, 10, 4])),
    ("extruded_3d_s2", lambda: cases.extruded_3d(2)),
]


@pytest.mark.skipif(not bridge.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name,make", LIVE, ids=[n for n, _ in LIVE])
def test_restatement_matches_live_reference(name, make):
    case = make()
    keep: list = []
    mesh, fld = cases.oracle_inputs(case, keep)
    ref = bridge.run_reference(mesh, fld)
    res = bridge.run_restatement(mesh, fld)
    assert len(ref.track_id) > 0
    assert_same(res, {"simplices": ref.simplices, "track_id": ref.track_id, "edges": ref.edges,
                      "bary": ref.bary, "scalar": ref.scalar, "type": ref.type, "lam": ref.lam})


@pytest.mark.skipif(not os.path.exists(bridge.REF_CUDA_LIB), reason="reference GPU build absent")
def test_reference_gpu_build_loads():
    """The reference's GPU engine, built only to time the incumbent GPU path,
    loads without a device and exports its three entry points."""
    lib = C.CDLL(bridge.REF_CUDA_LIB)
    for name in ("ftk2refcuda_run", "ftk2refcuda_time_kernel", "ftk2refcuda_free"):
        assert hasattr(lib, name)
