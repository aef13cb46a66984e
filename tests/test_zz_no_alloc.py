"""The allocation-free entry point, ftk2b_cp_features_noalloc, through the C ABI.

It exists for callers that may not allocate device memory while they run (an
in-situ step inside a simulation that owns the device's memory, a serving
loop held to a fixed budget, a host recording calls where cudaMalloc is
forbidden).  Its results must be the features the regular entry point finds:
the same simplices and bit-identical barycentrics, on two calls in a row (the
second call reuses the static scratch the first one left behind).

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from ftk2_b200 import api
from ftk2_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def chain_masks(d, m):
    """Chain types in canonical order (the same construction as the library)."""
    full = (1 << d) - 1
    out = []

    def rec(prev, depth, acc):
        for nx in range(prev + 1, full + 1):
            if (nx & prev) == prev and nx != prev:
                if depth == m:
                    out.append(acc + [nx])
                else:
                    rec(nx, depth + 1, acc + [nx])

    rec(0, 1, [])
    return out


def decode(keys, dims):
    """Canonical keys -> sorted vertex ids of each simplex."""
    d = len(dims)
    chains = chain_masks(d, d - 1)
    nch = len(chains)
    strides = [1] * d
    for k in range(1, d):
        strides[k] = strides[k - 1] * dims[k - 1]
    rows = []
    for key in keys.tolist():
        vid0, ch = divmod(key, nch)
        row = [vid0]
        for mk in chains[ch]:
            row.append(vid0 + sum(strides[k] for k in range(d) if (mk >> k) & 1))
        rows.append(row)
    return np.array(rows, dtype=np.uint64).reshape(-1, d)


def run_noalloc(lib, mesh, fld, q, capacity, stream):
    import torch
    keys = torch.zeros(capacity, dtype=torch.int64, device="cuda")
    lam = torch.zeros(4 * capacity, dtype=torch.float64, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    n = C.c_uint64()
    st = lib.ftk2b_cp_features_noalloc(C.byref(mesh), C.byref(fld), q, stream, keys.data_ptr(),
                                       lam.data_ptr(), capacity, count.data_ptr(), C.byref(n))
    return st, keys, lam, int(n.value)


CASES = [
    ("3d_f64", lambda: S.gaussian_sum_gradient((48, 40, 36), 6, seed=1, n_blobs=24), [48, 40, 36, 6],
     2.0 ** 20),
    ("3d_f32", lambda: S.gaussian_sum_gradient((40, 36, 32), 5, seed=7, n_blobs=24, dtype=np.float32,
                                               noise=1e-3, sigma=(3, 8)), [40, 36, 32, 5], 2.0 ** 20),
    ("2d_f64", lambda: S.analytic_2d(64, 64, 10), [64, 64, 10], 1e6),
]


@pytest.mark.parametrize("name,make,dims,q", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_regular_entry_point_twice(name, make, dims, q):
    torch = pytest.importorskip("torch")
    field = torch.from_numpy(make()).cuda()
    m = len(dims) - 1
    keep: list = []
    mesh = api.regular_mesh_desc(dims)
    fld = api.field_desc(field, api.LAYOUT_MULTICOMPONENT, m, keep=keep)
    with api.Context(0) as ctx:
        ref = ctx.extract(mesh, fld, api.params(q))
    assert len(ref.track_id) > 0
    lib = api.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):
        st, keys, lam, n = run_noalloc(lib, mesh, fld, q, 1 << 16, stream)
        assert st == api.OK, api.STATUS_NAMES[st]
        k = keys[:n].cpu().numpy().astype(np.uint64)
        lm = lam[:4 * n].cpu().numpy().reshape(n, 4)
        order = np.argsort(k, kind="stable")
        k, lm = k[order], lm[order]
        outs.append((k, lm))
        assert np.array_equal(decode(k, dims), ref.simplices)
        assert np.array_equal(lm[:, :m + 1], ref.lam)  # bit-identical (tolerance 0)
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_noalloc_rejects_what_it_cannot_hold():
    torch = pytest.importorskip("torch")
    lib = api.load_library()
    field = torch.from_numpy(S.analytic_2d(32, 32, 4)).cuda()
    keep: list = []
    mesh = api.regular_mesh_desc([32, 32, 4])
    fld = api.field_desc(field, api.LAYOUT_MULTICOMPONENT, 2, keep=keep)
    stream = torch.cuda.current_stream().cuda_stream
    # output capacity beyond the static scratch limit (2^18 features)
    st, _, _, _ = run_noalloc(lib, mesh, fld, 1e6, (1 << 18) + 1, stream)
    assert st == api.INVALID_ARG
    # host memory would need a staging allocation
    host = api.field_desc(S.analytic_2d(32, 32, 4), api.LAYOUT_MULTICOMPONENT, 2, keep=keep)
    st, _, _, _ = run_noalloc(lib, mesh, host, 1e6, 1024, stream)
    assert st == api.INVALID_ARG
    # an output too small for the features found is reported, not truncated silently
    st, _, _, n = run_noalloc(lib, mesh, fld, 1e6, 4, stream)
    assert st == api.OVERFLOW_RETRY and n > 4
