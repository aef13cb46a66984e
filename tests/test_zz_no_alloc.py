"""The allocation-free entry point, ftk2b_cp_features_noalloc, through the C ABI.

It exists for callers that may not allocate device memory while they run: an
in-situ analysis step inside a simulation whose memory manager owns the whole
device, or a serving loop held to a fixed memory budget that cannot absorb
cudaMalloc's implicit synchronisation.  Its results must be the features the
regular entry point finds: the same simplices and bit-identical barycentrics
(tolerance 0), on two calls in a row (the second call reuses the static
scratch the first one left behind).

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
    # a non-positive or NaN quantisation scale
    for q in (0.0, -1.0, float("nan")):
        st, _, _, _ = run_noalloc(lib, mesh, fld, q, 1024, stream)
        assert st == api.INVALID_ARG, q
    # only 2D+t and 3D+t regular meshes
    for nd in (2, 5):
        bad = api.regular_mesh_desc([32, 32, 4])
        bad.ndims = nd
        st, _, _, _ = run_noalloc(lib, bad, fld, 1e6, 1024, stream)
        assert st == api.UNSUPPORTED, nd


def test_noalloc_separate_arrays_on_offset_sub_box_twice():
    """SEPARATE layout: M arrays of the local box, read at global - offset
    (engine.hpp:999-1009), on a sub-box of a larger mesh."""
    torch = pytest.importorskip("torch")
    local, off, glob = [40, 36, 30, 5], [5, 3, 2, 1], [56, 48, 40, 8]
    v = S.gaussian_sum_gradient(tuple(local[:3]), local[3], seed=11, n_blobs=24,
                                origin=off[:3], t0=off[3], box=tuple(glob[:3]))
    comps = [torch.from_numpy(np.ascontiguousarray(v[..., j])).cuda() for j in range(3)]
    keep: list = []
    mesh = api.regular_mesh_desc(local, off, glob)
    fld = api.field_desc(comps, api.LAYOUT_SEPARATE, 3, keep=keep)
    with api.Context(0) as ctx:
        ref = ctx.extract(mesh, fld, api.params(2.0 ** 20))
    assert len(ref.track_id) > 0
    lib = api.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):
        st, keys, lam, n = run_noalloc(lib, mesh, fld, 2.0 ** 20, 1 << 16, stream)
        assert st == api.OK, api.STATUS_NAMES[st]
        k = keys[:n].cpu().numpy().astype(np.uint64)
        lm = lam[:4 * n].cpu().numpy().reshape(n, 4)
        order = np.argsort(k, kind="stable")
        k, lm = k[order], lm[order]
        assert np.array_equal(decode(k, glob), ref.simplices)
        assert np.array_equal(lm, ref.lam)
        outs.append((k, lm))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_noalloc_too_many_survivors_is_unsupported_then_recovers():
    """Pure noise leaves nearly every hypercube of a 64^3 x 3 box (500k)
    after the cull, more than the static scratch's 2^18 candidates: the call
    says the box must be split (no retry can succeed).  The next call on a
    normal field still matches the regular entry point."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    noise = torch.from_numpy(rng.standard_normal((3, 64, 64, 64, 3)).astype(np.float32)).cuda()
    keep: list = []
    lib = api.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    st, _, _, _ = run_noalloc(lib, api.regular_mesh_desc([64, 64, 64, 3]),
                              api.field_desc(noise, api.LAYOUT_MULTICOMPONENT, 3, keep=keep),
                              2.0 ** 20, 1 << 18, stream)
    assert st == api.UNSUPPORTED, api.STATUS_NAMES[st]
    v = torch.from_numpy(S.analytic_2d(48, 40, 6)).cuda()
    mesh = api.regular_mesh_desc([48, 40, 6])
    fld = api.field_desc(v, api.LAYOUT_MULTICOMPONENT, 2, keep=keep)
    with api.Context(0) as ctx:
        ref = ctx.extract(mesh, fld, api.params(1e6))
    st, keys, lam, n = run_noalloc(lib, mesh, fld, 1e6, 1 << 16, stream)
    assert st == api.OK, api.STATUS_NAMES[st]
    k = keys[:n].cpu().numpy().astype(np.uint64)
    order = np.argsort(k, kind="stable")
    assert np.array_equal(decode(k[order], [48, 40, 6]), ref.simplices)
    assert np.array_equal(lam[:4 * n].cpu().numpy().reshape(n, 4)[order][:, :3], ref.lam)
