"""The C-ABI library loads, exports every symbol include/ftk2b.h declares, and
refuses to run without a GPU instead of falling back to the CPU.  No compute
call is made here."""
import ctypes as C
import os
import re

import pytest

from ftk2_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(ftk2b_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = api.load_library()
    names = declared_symbols()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_symbols()) <= set(api.SIGNATURES)


def test_no_cpu_fallback_without_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(api.Ftk2bError) as e:
        api.Context(0)
    assert e.value.status == api.NO_DEVICE


def test_simplex_count_matches_restatement():
    # the unit of work: every m-simplex of the local box, upper-boundary
    # faces included (n_tested of the oracle restatement)
    from oracle import bridge
    import cases
    case = cases.c1_analytic_2d()
    keep: list = []
    mesh, fld = cases.oracle_inputs(case, keep)
    res = bridge.run_restatement(mesh, fld)
    assert api.simplex_count(api.regular_mesh_desc([64, 64, 10]), 2) == res.n_tested
    # LUT part alone is 12 * 63 * 63 * 9 (mesh.hpp:270-302)
    assert res.n_tested > 12 * 63 * 63 * 9


def test_extruded_simplex_count_matches_restatement():
    # spatial cells at every layer, lateral prism pieces over every unique base
    # face and the interior pieces (engine.hpp:573 counts the first two)
    from oracle import bridge
    import cases
    for name in ("extruded_2d", "extruded_3d_s0"):
        case = cases.GOLDEN_CASES[name]()
        keep: list = []
        mesh, fld = cases.oracle_inputs(case, keep)
        res = bridge.run_restatement(mesh, fld)
        desc = api.extruded_mesh_desc(case.coords.shape[0], case.cells, case.n_layers, keep)
        assert api.simplex_count(desc, case.ncomp) == res.n_tested


def test_no_server_without_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(api.Ftk2bError) as e:
        api.Server(0, n_slots=2)
    assert e.value.status == api.NO_DEVICE
