"""Batched extraction (ftk2b_cp_*_batch): every field's result in a batch is
identical to the single-field extraction of that field (and so to the
oracle), whatever the mix of 2D / 3D fields, sizes, layouts, offsets and
per-field parameters; graph replay, time chunking and device inputs change
nothing."""
import numpy as np
import pytest

from ftk2_b200 import api
from ftk2_b200 import synthetic as S
from oracle import bridge
import cases

pytestmark = pytest.mark.gpu


def assert_identical(g, o):
    assert g.simplices.shape == o.simplices.shape, (g.simplices.shape, o.simplices.shape)
    assert np.array_equal(g.simplices, o.simplices)
    assert np.array_equal(g.track_id, o.track_id)
    assert np.array_equal(g.edges, o.edges)
    assert np.array_equal(g.bary, o.bary)
    assert np.array_equal(g.lam, o.lam)
    assert np.array_equal(g.scalar, o.scalar)
    assert g.n_tracks == o.n_tracks
    assert g.n_simplices == o.n_simplices


def mixed_cases(seed, n, dtype=np.float32, small=False):
    """Seeded 2D / 3D multicomponent fields of uneven sizes."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        three = i % 2 == 1
        hi = (24 if small else 40) if three else (48 if small else 150)
        dims = tuple(int(v) for v in rng.integers(6, hi, size=3 if three else 2))
        nt = int(rng.integers(2, 6))
        g = S.gaussian_sum_gradient(dims, nt, seed=100 + i, n_blobs=int(rng.integers(8, 24)), dtype=dtype,
                                    noise=1e-3 if dtype == np.float32 else 0.0, sigma=(2, 6))
        q = 2.0 ** 20 if three else 1e6
        out.append(cases.Case(f"b{i}", "regular", 3 if three else 2, cases.MULTI, g, q, list(dims) + [nt]))
    return out


def descriptors(case_list, keep):
    meshes, fields = [], []
    for c in case_list:
        m, f = cases.gpu_inputs(c, keep)
        meshes.append(m)
        fields.append(f)
    return meshes, fields


def singles(ctx, case_list, prms):
    out = []
    for c, p in zip(case_list, prms):
        keep: list = []
        m, f = cases.gpu_inputs(c, keep)
        out.append(ctx.extract(m, f, p))
    return out


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_batch_equals_single_field_runs(ctx, dtype):
    cl = mixed_cases(3, 14, dtype)
    prms = [api.params(c.sos_q) for c in cl]
    keep: list = []
    meshes, fields = descriptors(cl, keep)
    res = ctx.extract_batch(meshes, fields, prms)
    assert len(res) == len(cl)
    ref = singles(ctx, cl, prms)
    assert sum(len(r.track_id) for r in ref) > 0
    for r, s in zip(res, ref):
        assert_identical(r, s)
    # and the restatement, on two of them
    for i in (0, 1):
        okeep: list = []
        om, of = cases.oracle_inputs(cl[i], okeep)
        o = bridge.run_restatement(om, of)
        assert np.array_equal(res[i].simplices, o.simplices)
        assert np.array_equal(res[i].track_id, o.track_id)
        assert np.array_equal(res[i].edges, o.edges)
        assert np.array_equal(res[i].lam, o.lam)


def test_batch_replay_chunks_and_eager_agree(ctx):
    cl = mixed_cases(5, 9)
    prms = [api.params(c.sos_q) for c in cl]
    keep: list = []
    meshes, fields = descriptors(cl, keep)
    first = ctx.extract_batch(meshes, fields, prms)  # time chunk tuned for this shape
    assert ctx.get_option(api.INFO_LAST_BATCH_TIME_CHUNK) in (2, 4, 0xFFFF)
    again = ctx.extract_batch(meshes, fields, prms)  # replayed graph pair
    for a, b in zip(first, again):
        assert_identical(a, b)
    for tc in (1, 2):
        ctx.set_option(api.OPT_BATCH_TIME_CHUNK, tc)
        try:
            r = ctx.extract_batch(meshes, fields, prms)
        finally:
            ctx.set_option(api.OPT_BATCH_TIME_CHUNK, 0)
        for a, b in zip(first, r):
            assert_identical(a, b)
    ctx.set_option(api.OPT_USE_GRAPHS, 0)
    try:
        r = ctx.extract_batch(meshes, fields, prms)
    finally:
        ctx.set_option(api.OPT_USE_GRAPHS, 1)
    for a, b in zip(first, r):
        assert_identical(a, b)


def test_batch_separate_arrays_offsets_and_scalars(ctx):
    cl = []
    for i in range(6):
        if i % 2:
            g = S.gaussian_sum_gradient((34, 33, 35), 5, seed=40 + i, n_blobs=20, dtype=np.float32)
            comps = [np.ascontiguousarray(g[..., j]) for j in range(3)]
            cl.append(cases.Case(f"s3_{i}", "regular", 3, cases.SEPARATE, comps, 2.0 ** 20,
                                 [30 - i, 29, 31, 4], [2, 3, 1, 1], [34, 33, 35, 5]))
        else:
            g = S.gaussian_sum_gradient((130, 97), 9, seed=50 + i, n_blobs=30, dtype=np.float32, sigma=(2, 6))
            U, V = np.ascontiguousarray(g[..., 0]), np.ascontiguousarray(g[..., 1])
            sc = np.random.default_rng(i).standard_normal(U.shape).astype(np.float32)
            cl.append(cases.Case(f"s2_{i}", "regular", 2, cases.SEPARATE, [U, V], 1e6,
                                 [120 - i, 90, 8], [5, 4, 1], [130, 97, 9], scalar=sc))
    prms = [api.params(c.sos_q) for c in cl]
    keep: list = []
    meshes, fields = descriptors(cl, keep)
    res = ctx.extract_batch(meshes, fields, prms)
    for r, s in zip(res, singles(ctx, cl, prms)):
        assert_identical(r, s)


def test_batch_per_field_parameters(ctx):
    cl = mixed_cases(8, 8, small=True)
    prec = [api.PRECISION_REFINED if i % 3 == 0 else api.PRECISION_EXACT for i in range(len(cl))]
    prms = [api.params(c.sos_q * (1 + i % 2), precision=prec[i], want_edges=(i % 4 != 2)) for i, c in enumerate(cl)]
    keep: list = []
    meshes, fields = descriptors(cl, keep)
    res = ctx.extract_batch(meshes, fields, prms)
    for i, (r, s) in enumerate(zip(res, singles(ctx, cl, prms))):
        assert_identical(r, s)
        if i % 4 == 2:
            assert len(r.edges) == 0 and np.array_equal(r.track_id, np.arange(len(r.track_id)))


def test_batch_of_one_and_device_inputs(ctx):
    torch = pytest.importorskip("torch")
    cl = mixed_cases(11, 4, small=True)
    prms = [api.params(c.sos_q) for c in cl]
    keep: list = []
    m0, f0 = cases.gpu_inputs(cl[1], keep)
    one = ctx.extract_batch([m0], [f0], [prms[1]])
    assert_identical(one[0], singles(ctx, cl[1:2], prms[1:2])[0])
    meshes, fields = descriptors(cl, keep)
    host = ctx.extract_batch(meshes, fields, prms)
    devf = []
    for c in cl:
        t = torch.from_numpy(c.arrays).cuda()
        keep.append(t)
        devf.append(api.field_desc(t, api.LAYOUT_MULTICOMPONENT, c.ncomp, keep=keep))
    dev = ctx.extract_batch(meshes, devf, prms)
    for a, b in zip(host, dev):
        assert_identical(a, b)


def test_batch_rejects_mixed_dtypes(ctx):
    a = mixed_cases(1, 2, np.float32, small=True)
    b = mixed_cases(2, 2, np.float64, small=True)
    keep: list = []
    meshes, fields = descriptors([a[0], b[1]], keep)
    with pytest.raises(api.Ftk2bError):
        ctx.extract_batch(meshes, fields, None)
