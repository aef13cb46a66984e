"""GPU parity: the CUDA path, called through the C ABI, against the oracle.

* every golden case: identical to the reference engine's own output
  (simplex ids, float barycentrics, lambdas, track ids, edges, scalars);
* seeded medium cases: identical to the exact C restatement;
* full-size configuration: size-independent invariants of the result plus
  windows of it against the restatement;
* host and device inputs give the same bytes; repeated runs are identical;
* buffer overflow is recovered by the retry path.
"""
import os

import numpy as np
import pytest

from ftk2_b200 import api
from ftk2_b200 import synthetic as S
from oracle import bridge
import cases

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def gpu_run(ctx, case, **kw):
    keep: list = []
    mesh, fld = cases.gpu_inputs(case, keep)
    return ctx.extract(mesh, fld, api.params(case.sos_q, **kw))


def oracle_run(case):
    keep: list = []
    mesh, fld = cases.oracle_inputs(case, keep)
    return bridge.run_restatement(mesh, fld)


def assert_identical(g, o, lam=True):
    assert g.simplices.shape == o.simplices.shape, (g.simplices.shape, o.simplices.shape)
    assert np.array_equal(g.simplices, o.simplices)
    assert np.array_equal(g.track_id, o.track_id)
    assert np.array_equal(g.edges, o.edges)
    assert np.array_equal(g.bary, o.bary)
    assert np.array_equal(g.scalar, o.scalar)
    assert np.array_equal(g.type, o.type)
    if lam:
        assert np.array_equal(g.lam, o.lam)


REGULAR_GOLDEN = [n for n in sorted(cases.GOLDEN_CASES) if not n.startswith("extruded")]
EXTRUDED_GOLDEN = [n for n in sorted(cases.GOLDEN_CASES) if n.startswith("extruded")]


@pytest.mark.parametrize("staging", ["tma", "plain"])
@pytest.mark.parametrize("name", REGULAR_GOLDEN)
def test_golden_regular(ctx, name, staging):
    case = cases.GOLDEN_CASES[name]()
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    assert str(z["input_sha256"]) == case.input_digest()
    ctx.set_option(api.OPT_DISABLE_TMA, 1 if staging == "plain" else 0)
    try:
        g = gpu_run(ctx, case)
        if staging == "plain":
            assert ctx.get_option(api.INFO_LAST_TMA) == 0
    finally:
        ctx.set_option(api.OPT_DISABLE_TMA, 0)
    ref = bridge.CPResult(simplices=z["simplices"], bary=z["bary"], lam=z["lam"],
                          track_id=z["track_id"], type=z["type"], scalar=z["scalar"],
                          edges=z["edges"])
    assert_identical(g, ref)
    assert g.n_tracks == len(np.unique(ref.track_id))


def _medium_cases():
    out = []
    for seed in (1, 2):
        g = S.gaussian_sum_gradient((48, 40, 36), 6, seed=seed, n_blobs=24)
        out.append(cases.Case(f"g3d_f64_s{seed}", "regular", 3, cases.MULTI, g, 2.0 ** 20,
                              [48, 40, 36, 6]))
    g = S.gaussian_sum_gradient((40, 36, 32), 5, seed=7, n_blobs=24, dtype=np.float32, noise=1e-3,
                                sigma=(3, 8))
    out.append(cases.Case("g3d_f32_noise", "regular", 3, cases.MULTI, g, 2.0 ** 20, [40, 36, 32, 5]))
    g = S.gaussian_sum_gradient((200, 150), 12, seed=3, n_blobs=40, sigma=(3, 9))
    out.append(cases.Case("g2d_f64", "regular", 2, cases.MULTI, g, 1e6, [200, 150, 12]))
    g = S.gaussian_sum_gradient((130, 97), 9, seed=4, n_blobs=30, dtype=np.float32, sigma=(2, 6))
    U, V = np.ascontiguousarray(g[..., 0]), np.ascontiguousarray(g[..., 1])
    sc = np.random.default_rng(5).standard_normal(U.shape).astype(np.float32)
    out.append(cases.Case("g2d_f32_sep_offset", "regular", 2, cases.SEPARATE, [U, V], 1e6,
                          [120, 90, 8], [5, 4, 1], [130, 97, 9], scalar=sc))
    g = S.gaussian_sum_gradient((34, 33, 35), 5, seed=11, n_blobs=20)
    comps = [np.ascontiguousarray(g[..., j]) for j in range(3)]
    out.append(cases.Case("g3d_sep_offset", "regular", 3, cases.SEPARATE, comps, 2.0 ** 20,
                          [30, 29, 31, 4], [2, 3, 1, 1], [34, 33, 35, 5]))
    return out


@pytest.mark.parametrize("case", _medium_cases(), ids=lambda c: c.name)
def test_medium_vs_restatement(ctx, case):
    g = gpu_run(ctx, case)
    o = oracle_run(case)
    assert len(o.track_id) > 0
    assert_identical(g, o)
    assert g.n_simplices == o.n_tested
    ctx.set_option(api.OPT_DISABLE_TMA, 1)
    try:
        p = gpu_run(ctx, case)
    finally:
        ctx.set_option(api.OPT_DISABLE_TMA, 0)
    assert_identical(p, o)


def test_tma_used_when_aligned_and_skipped_when_not(ctx):
    g = S.gaussian_sum_gradient((40, 36, 32), 4, seed=2, n_blobs=10)
    # aligned multicomponent float64 array: TMA staging
    gpu_run(ctx, cases.Case("a", "regular", 3, cases.MULTI, g, 2.0 ** 20, [40, 36, 32, 4]))
    assert ctx.get_option(api.INFO_LAST_TMA) == 1
    # odd x offset: a box would start 24 bytes into a 16-byte line, so the
    # kernel falls back to plain loads, with identical results
    case = cases.Case("b", "regular", 3, cases.MULTI, g, 2.0 ** 20, [36, 30, 28, 3], [3, 1, 2, 1],
                      [40, 36, 32, 4])
    r = gpu_run(ctx, case)
    assert ctx.get_option(api.INFO_LAST_TMA) == 0
    assert_identical(r, oracle_run(case))


def test_device_input_matches_host_input(ctx):
    torch = pytest.importorskip("torch")
    g = S.gaussian_sum_gradient((40, 40, 40), 5, seed=13, n_blobs=24)
    keep: list = []
    mesh = api.regular_mesh_desc([40, 40, 40, 5])
    host = ctx.extract(mesh, api.field_desc(g, api.LAYOUT_MULTICOMPONENT, 3, keep=keep),
                       api.params(2.0 ** 20))
    dev = torch.from_numpy(g).cuda()
    devr = ctx.extract(mesh, api.field_desc(dev, api.LAYOUT_MULTICOMPONENT, 3, keep=keep),
                       api.params(2.0 ** 20))
    assert_identical(host, devr)
    again = ctx.extract(mesh, api.field_desc(dev, api.LAYOUT_MULTICOMPONENT, 3, keep=keep),
                        api.params(2.0 ** 20))
    assert_identical(devr, again)


def test_graph_replay_and_eager_agree(ctx):
    case = cases.GOLDEN_CASES["f32_3d_noise_offset"]()
    a = gpu_run(ctx, case)
    b = gpu_run(ctx, case)          # replayed graph
    ctx.set_option(api.OPT_USE_GRAPHS, 0)
    try:
        c = gpu_run(ctx, case)      # eager launches
    finally:
        ctx.set_option(api.OPT_USE_GRAPHS, 1)
    assert_identical(a, b)
    assert_identical(a, c)


def test_overflow_retry(ctx):
    case = cases.c1_analytic_2d()
    ctx.set_option(api.OPT_FEATURE_CAPACITY, 100)  # far below the 3697 features
    try:
        g = gpu_run(ctx, case)
    finally:
        ctx.set_option(api.OPT_FEATURE_CAPACITY, 0)
    z = np.load(os.path.join(GOLDEN, "c1_analytic_2d.npz"))
    assert np.array_equal(g.simplices, z["simplices"])
    assert np.array_equal(g.edges, z["edges"])


@pytest.mark.parametrize("tchunk", [1, 3])
def test_time_chunking_is_invisible(ctx, tchunk):
    case = cases.GOLDEN_CASES["gauss3d_16"]()
    base = gpu_run(ctx, case)
    ctx.set_option(api.OPT_TIME_CHUNK, tchunk)
    try:
        g = gpu_run(ctx, case)
    finally:
        ctx.set_option(api.OPT_TIME_CHUNK, 0)
    assert_identical(base, g)


def check_invariants(r):
    n = len(r.track_id)
    # canonical order: strictly increasing tuples (Simplex::operator<)
    s = r.simplices
    if n > 1:
        a, b = s[:-1], s[1:]
        diff = a != b
        first = diff.argmax(axis=1)
        rows = np.arange(n - 1)
        assert diff.any(axis=1).all()
        assert (a[rows, first] < b[rows, first]).all()
    assert (np.diff(s, axis=1) > 0).all()              # sorted vertex ids
    # track ids: root of the component = smallest member, idempotent
    t = r.track_id.astype(np.int64)
    assert (t <= np.arange(n)).all()
    assert (t[t] == t).all()
    # edges: sorted, unique, lo < hi, endpoints in one track
    e = r.edges.astype(np.int64)
    if len(e):
        assert (e[:, 0] < e[:, 1]).all()
        key = e[:, 0] * (n + 1) + e[:, 1]
        assert (np.diff(key) > 0).all()
        assert (t[e[:, 0]] == t[e[:, 1]]).all()
    # barycentrics in range and summing to one
    assert (r.lam >= -1e-9).all() and (r.lam <= 1 + 1e-9).all()
    np.testing.assert_allclose(r.lam.sum(axis=1), 1.0, atol=1e-12)


def test_full_size_3d_config_invariants_and_windows(ctx):
    """128^3 x 16 float64 Gaussian-sum gradient (the 3D plain drop-in
    configuration): invariants at full size, and sub-box meshes of the same
    field identical to the restatement."""
    torch = pytest.importorskip("torch")
    from ftk2_b200 import generate
    dev = generate.gaussian_field_device((128, 128, 128), 16, seed=1234, n_blobs=32,
                                         dtype=torch.float64)
    keep: list = []
    mesh = api.regular_mesh_desc([128, 128, 128, 16])
    r = ctx.extract(mesh, api.field_desc(dev, api.LAYOUT_MULTICOMPONENT, 3, keep=keep),
                    api.params(2.0 ** 20))
    assert len(r.track_id) > 100
    check_invariants(r)
    host = dev.cpu().numpy()
    rng = np.random.default_rng(0)
    for _ in range(2):
        lo = [int(rng.integers(0, 128 - 40)) for _ in range(3)] + [int(rng.integers(0, 8))]
        local = [40, 40, 40, 8]
        case = cases.Case("win", "regular", 3, cases.MULTI, host, 2.0 ** 20, local, lo,
                          [128, 128, 128, 16])
        g = gpu_run(ctx, case)
        o = oracle_run(case)
        assert_identical(g, o)


def test_refined_precision_same_set_smaller_error(ctx):
    g32 = S.gaussian_sum_gradient((40, 36, 32), 5, seed=7, n_blobs=24, dtype=np.float32, noise=1e-3,
                                  sigma=(3, 8))
    case = cases.Case("p", "regular", 3, cases.MULTI, g32, 2.0 ** 20, [40, 36, 32, 5])
    exact = gpu_run(ctx, case)
    refined = gpu_run(ctx, case, precision=api.PRECISION_REFINED)
    # the accepted set, tracks and stored float barycentrics are unchanged
    assert np.array_equal(exact.simplices, refined.simplices)
    assert np.array_equal(exact.track_id, refined.track_id)
    assert np.array_equal(exact.bary, refined.bary)
    # position error against an FP64 solve of the promoted values
    case64 = cases.Case("p64", "regular", 3, cases.MULTI, g32.astype(np.float64), 2.0 ** 20,
                        [40, 36, 32, 5])
    o64 = oracle_run(case64)
    idx = {tuple(s): i for i, s in enumerate(o64.simplices.tolist())}
    common = [(i, idx[tuple(s)]) for i, s in enumerate(refined.simplices.tolist()) if tuple(s) in idx]
    assert len(common) > 0.9 * len(refined.simplices)
    a = np.array([refined.lam[i] for i, _ in common])
    b = np.array([o64.lam[j] for _, j in common])
    c = np.array([exact.lam[i] for i, _ in common])
    err_ref = np.abs(a - b).max()
    err_f32 = np.abs(c - b).max()
    assert err_ref <= 1e-9 or err_ref < 1e-3 * err_f32, (err_ref, err_f32)


def test_graph_cache_alternating_workloads(ctx):
    # several workloads in turn on one context: each replays its own cached
    # graphs and still gives its own exact result
    cs = _medium_cases()[:3]
    first = [gpu_run(ctx, c) for c in cs]
    for _ in range(2):
        for c, f in zip(cs, first):
            assert_identical(gpu_run(ctx, c), f)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_cull_modes_agree_with_restatement(ctx, mode):
    # mode 0: per-vertex cull words only; mode 1: tile statistics first;
    # mode 2: the faster of the two per workload shape, timed once
    ctx.set_option(api.OPT_CULL_MODE, mode)
    try:
        for case in _medium_cases()[:4]:
            assert_identical(gpu_run(ctx, case), oracle_run(case))
    finally:
        ctx.set_option(api.OPT_CULL_MODE, 2)


def test_tile_cull_edge_fields(ctx):
    # whole tiles that the tile statistics drop (one-signed component, values
    # below the pivot floor) next to tiles that they must keep
    base = S.gaussian_sum_gradient((70, 44, 38), 4, seed=21, n_blobs=16)
    shifted = base.copy()
    shifted[..., 0] += 5.0                      # component 0 positive everywhere
    tiny = base * 1e-14                          # every |v| below 4e-13
    mixed = base.copy()
    mixed[:, :, :, :30, :] *= 1e-14              # tiny on one side only
    mixed[:, :, :, 50:, 1] -= 3.0                # one-signed on the other
    for name, f, q in (("shifted", shifted, 2.0 ** 20), ("tiny", tiny, 2.0 ** 20),
                       ("mixed", mixed, 2.0 ** 20), ("tiny_q", tiny, 1e15)):
        case = cases.Case(name, "regular", 3, cases.MULTI, np.ascontiguousarray(f), q, [70, 44, 38, 4])
        g, o = gpu_run(ctx, case), oracle_run(case)
        assert_identical(g, o)
        if name in ("shifted", "tiny"):
            assert len(o.track_id) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tile_cull_partial_rows(ctx, dtype):
    # sub-meshes of aligned arrays (so the tile statistics stream 16-byte
    # vectors) whose rows end inside a vector: the tail elements are copied
    # one by one and nothing beyond the local mesh is read
    g = S.gaussian_sum_gradient((40, 36, 32), 5, seed=17, n_blobs=24, dtype=dtype, noise=1e-3, sigma=(3, 8))
    for dims, off in (([35, 30, 27, 4], [4, 2, 1, 1]), ([35, 33, 31, 5], [0, 3, 1, 0]),
                      ([21, 36, 32, 5], [16, 0, 0, 0])):
        case = cases.Case(f"part_{dims[0]}", "regular", 3, cases.MULTI, g, 2.0 ** 20, dims, off, [40, 36, 32, 5])
        o = oracle_run(case)
        for mode in (0, 1):
            ctx.set_option(api.OPT_CULL_MODE, mode)
            try:
                r = gpu_run(ctx, case)
            finally:
                ctx.set_option(api.OPT_CULL_MODE, 2)
            assert ctx.get_option(api.INFO_LAST_TMA) == 1
            assert_identical(r, o)


def test_cull_autotuner_keeps_its_choice(ctx):
    # the first extraction of a shape times both modes; later ones of the
    # same shape run the mode it chose, with identical results
    case = _medium_cases()[2]
    ctx.set_option(api.OPT_CULL_MODE, 2)
    first = gpu_run(ctx, case)
    mode = ctx.get_option(api.INFO_LAST_CULL_MODE)
    assert mode in (0, 1)
    for _ in range(2):
        assert_identical(gpu_run(ctx, case), first)
        assert ctx.get_option(api.INFO_LAST_CULL_MODE) == mode
    assert_identical(first, oracle_run(case))


def test_short_and_radix_post_chains_agree(ctx):
    # feature capacities up to 16384 run the short post-extraction chain (rank
    # sort, star edges, one-block union-find), larger ones the radix-sort chain
    for case in _medium_cases()[:3] + [cases.c1_analytic_2d()]:
        short = gpu_run(ctx, case)
        ctx.set_option(api.OPT_FEATURE_CAPACITY, 20000)
        try:
            radix = gpu_run(ctx, case)
        finally:
            ctx.set_option(api.OPT_FEATURE_CAPACITY, 0)
        assert_identical(short, radix)
        assert_identical(short, oracle_run(case))


def test_many_features_grow_past_the_short_chain():
    # a noise field with more features than the short chain holds: the first
    # attempt overflows its capacity and the retry runs the radix-sort chain
    rng = np.random.default_rng(3)
    g = np.ascontiguousarray(rng.standard_normal((3, 18, 20, 24, 3)).astype(np.float32))
    case = cases.Case("noise", "regular", 3, cases.MULTI, g, 2.0 ** 20, [24, 20, 18, 3])
    with api.Context(0) as c:
        r = gpu_run(c, case)
        assert c.get_option(api.OPT_FEATURE_CAPACITY) > 16384
    assert len(r.track_id) > 16384
    assert_identical(r, oracle_run(case))


@pytest.mark.parametrize("staging", ["tma", "bulk"])
def test_bounded_wait_runs_out_and_context_recovers(staging):
    """Failure path without a fault: with the stall option every cull block,
    once its first slice has landed, waits a few polls on an mbarrier that
    nothing completes, leaves through the bounded-wait path (the other copy in
    flight waited for) and the call reports FTK2B_TIMEOUT; the same context
    then gives the restatement's result."""
    case = _medium_cases()[0]
    with api.Context(0) as c:
        c.set_option(api.OPT_DISABLE_TMA, 1 if staging == "bulk" else 0)
        c.set_option(api.OPT_TEST_STALL_POLLS, 64)
        with pytest.raises(api.Ftk2bError) as e:
            gpu_run(c, case)
        assert e.value.status == api.TIMEOUT
        c.set_option(api.OPT_TEST_STALL_POLLS, 0)
        assert_identical(gpu_run(c, case), oracle_run(case))
        assert c.get_option(api.INFO_LAST_TMA) == (1 if staging == "tma" else 0)

