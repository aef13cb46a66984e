"""Time streams (ftk2b_stream_*): timesteps pushed one at a time give exactly
the one-shot result over the same timesteps (the reference's streaming
drivers are defective, engine.hpp:214-270, 601-819, so the oracle for a
stream is execute() + get_complex() on the whole spacetime mesh, which the
one-shot path matches bit for bit against the restatement)."""
import numpy as np
import pytest

from ftk2_b200 import api
from ftk2_b200 import synthetic as S
from oracle import bridge
import cases

pytestmark = pytest.mark.gpu


def assert_identical(g, o, cls=False):
    assert g.simplices.shape == o.simplices.shape, (g.simplices.shape, o.simplices.shape)
    assert np.array_equal(g.simplices, o.simplices)
    assert np.array_equal(g.track_id, o.track_id)
    assert np.array_equal(g.edges, o.edges)
    assert np.array_equal(g.bary, o.bary)
    assert np.array_equal(g.lam, o.lam)
    assert np.array_equal(g.scalar, o.scalar)
    assert g.n_tracks == len(np.unique(o.track_id))
    if cls:
        assert np.array_equal(g.cp_class, o.cp_class)


def steps_of(case, t):
    if case.layout == cases.MULTI:
        return case.arrays[t]
    return [a[t] for a in case.arrays]


def one_shot(ctx, case, nt, classify):
    keep: list = []
    d = len(case.local_dims)
    ld = list(case.local_dims[:-1]) + [nt]
    off = list(case.offset) if case.offset else None
    gd = list(case.global_dims[:-1]) + [nt] if case.global_dims else None
    mesh = api.regular_mesh_desc(ld, off, gd)
    arrs = case.arrays[:nt] if case.layout == cases.MULTI else [a[:nt] for a in case.arrays]
    fld = api.field_desc(arrs, case.layout, case.ncomp, keep=keep)
    return ctx.extract(mesh, fld, api.params(case.sos_q, classify=classify))


def stream_case(ctx, case, classify=False, device=False, check_every=False):
    keep: list = []
    nt = case.local_dims[-1]
    mesh = api.regular_mesh_desc(case.local_dims, case.offset, case.global_dims)
    tmpl = api.field_desc(steps_of(case, 0), case.layout, case.ncomp, keep=keep)
    prm = api.params(case.sos_q, classify=classify)
    if device:
        import torch
    with api.Stream(ctx, mesh, tmpl, prm) as st:
        total = 0
        for t in range(nt):
            step = steps_of(case, t)
            if device:
                step = (torch.from_numpy(np.ascontiguousarray(step)).cuda() if case.layout == cases.MULTI
                        else [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in step])
                keep.append(step)
            total += st.push(api.field_desc(step, case.layout, case.ncomp, keep=keep))
            if check_every or t == nt - 1:
                r = st.result()
                assert len(r.track_id) == total
                assert_identical(r, one_shot(ctx, case, t + 1, classify), cls=classify)
        assert st.info()[:2] == (nt, total)
        return r


def _cases():
    out = [cases.c1_analytic_2d()]
    g = S.gaussian_sum_gradient((48, 40, 36), 6, seed=1, n_blobs=24)
    out.append(cases.Case("g3d_f64", "regular", 3, cases.MULTI, g, 2.0 ** 20, [48, 40, 36, 6]))
    g = S.gaussian_sum_gradient((40, 36, 32), 5, seed=7, n_blobs=24, dtype=np.float32, noise=1e-3,
                                sigma=(3, 8))
    out.append(cases.Case("g3d_f32_noise", "regular", 3, cases.MULTI, g, 2.0 ** 20, [40, 36, 32, 5]))
    g = S.gaussian_sum_gradient((130, 97), 9, seed=4, n_blobs=30, dtype=np.float32, sigma=(2, 6))
    U, V = np.ascontiguousarray(g[..., 0]), np.ascontiguousarray(g[..., 1])
    out.append(cases.Case("g2d_f32_sep_offset", "regular", 2, cases.SEPARATE, [U, V], 1e6,
                          [120, 90, 9], [5, 4, 0], [130, 97, 9]))
    g = S.gaussian_sum_gradient((34, 33, 35), 5, seed=11, n_blobs=20)
    comps = [np.ascontiguousarray(g[..., j]) for j in range(3)]
    out.append(cases.Case("g3d_sep_offset", "regular", 3, cases.SEPARATE, comps, 2.0 ** 20,
                          [30, 29, 31, 5], [2, 3, 1, 0], [34, 33, 35, 5]))
    g = S.gaussian_sum_gradient((20, 18), 6, seed=3, n_blobs=8, sigma=(2, 4))
    out.append(cases.Case("offset2d_multi", "regular", 2, cases.MULTI, g, 1e6, [16, 14, 6], [2, 1, 0],
                          [20, 18, 6]))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c.name)
def test_stream_equals_one_shot(ctx, case):
    stream_case(ctx, case)


def test_stream_every_prefix_and_classes(ctx):
    stream_case(ctx, _cases()[2], classify=True, check_every=True)
    stream_case(ctx, cases.c1_analytic_2d(), classify=True, check_every=True)


def test_stream_device_steps(ctx):
    stream_case(ctx, _cases()[1], device=True)


def test_stream_matches_restatement(ctx):
    case = _cases()[2]
    r = stream_case(ctx, case)
    keep: list = []
    om, of = cases.oracle_inputs(case, keep)
    o = bridge.run_restatement(om, of)
    assert_identical(r, o)


def test_two_streams_on_two_contexts_interleaved():
    a_case, b_case = _cases()[0], _cases()[1]
    with api.Context(0) as ca, api.Context(0) as cb:
        keep: list = []
        sa = api.Stream(ca, api.regular_mesh_desc(a_case.local_dims),
                        api.field_desc(steps_of(a_case, 0), a_case.layout, 2, keep=keep), api.params(a_case.sos_q))
        sb = api.Stream(cb, api.regular_mesh_desc(b_case.local_dims),
                        api.field_desc(steps_of(b_case, 0), b_case.layout, 3, keep=keep), api.params(b_case.sos_q))
        for t in range(max(a_case.local_dims[-1], b_case.local_dims[-1])):
            if t < a_case.local_dims[-1]:
                sa.push(api.field_desc(steps_of(a_case, t), a_case.layout, 2, keep=keep))
            if t < b_case.local_dims[-1]:
                sb.push(api.field_desc(steps_of(b_case, t), b_case.layout, 3, keep=keep))
        assert_identical(sa.result(), one_shot(ca, a_case, a_case.local_dims[-1], False))
        assert_identical(sb.result(), one_shot(cb, b_case, b_case.local_dims[-1], False))
        sa.close()
        sb.close()


def test_stream_rejects_mismatched_step(ctx):
    case = _cases()[1]
    keep: list = []
    with api.Stream(ctx, api.regular_mesh_desc(case.local_dims),
                    api.field_desc(steps_of(case, 0), case.layout, 3, keep=keep), api.params(case.sos_q)) as st:
        bad = np.zeros((10, 10, 10, 3))
        with pytest.raises(api.Ftk2bError) as e:
            st.push(api.field_desc(bad, cases.MULTI, 3, keep=keep))
        assert e.value.status == api.INVALID_ARG
        st.push(api.field_desc(steps_of(case, 0), case.layout, 3, keep=keep))


# ---------------------------------------------------------------------------
# extruded meshes (the serving stream of a triangulated plane extruded into tets)

def ext_one_shot(ctx, case, nt):
    keep: list = []
    nv = case.coords.shape[0]
    mesh = api.extruded_mesh_desc(nv, case.cells, nt - 1, keep)
    fld = api.field_desc([np.ascontiguousarray(a[: nt * nv]) for a in case.arrays], case.layout, case.ncomp,
                         keep=keep)
    return ctx.extract(mesh, fld, api.params(case.sos_q))


def ext_stream_case(ctx, case, check_every=False, device=False):
    keep: list = []
    nv = case.coords.shape[0]
    nt = case.n_layers + 1
    mesh = api.extruded_mesh_desc(nv, case.cells, case.n_layers, keep)
    step = lambda t: [np.ascontiguousarray(a[t * nv:(t + 1) * nv]) for a in case.arrays]
    tmpl = api.field_desc(step(0), case.layout, case.ncomp, keep=keep)
    if device:
        import torch
    with api.Stream(ctx, mesh, tmpl, api.params(case.sos_q)) as st:
        total = 0
        for t in range(nt):
            arrs = step(t)
            if device:
                arrs = [torch.from_numpy(a).cuda() for a in arrs]
                keep.append(arrs)
            total += st.push(api.field_desc(arrs, case.layout, case.ncomp, keep=keep))
            if check_every or t == nt - 1:
                r = st.result()
                assert len(r.track_id) == total
                assert_identical(r, ext_one_shot(ctx, case, t + 1))
        return r


def _ext_cases():
    out = [cases.GOLDEN_CASES["extruded_3d_s0"](), cases.GOLDEN_CASES["extruded_2d"]()]
    coords, tets = S.extruded_tet_mesh(24, 22, 9, seed=1)
    vals = S.gaussian_sum_gradient_at(coords, 7, seed=201, n_blobs=24, sigma=(1.0, 3.0), drift=0.6,
                                      dtype=np.float32)
    out.append(cases.Case("ext3d_f32_7", "extruded", 3, cases.PER_VERTEX, [vals[0], vals[1], vals[2]],
                          2.0 ** 20, coords=coords, cells=tets, n_layers=6))
    return out


@pytest.mark.parametrize("case", _ext_cases(), ids=lambda c: c.name)
def test_extruded_stream_every_prefix(ctx, case):
    ext_stream_case(ctx, case, check_every=True)


def test_extruded_stream_matches_reference_fixture(ctx):
    import os
    case = cases.GOLDEN_CASES["extruded_3d_s4"]()
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "extruded_3d_s4.npz"))
    r = ext_stream_case(ctx, case, device=True)
    ref = bridge.CPResult(simplices=z["simplices"], bary=z["bary"], lam=z["lam"], track_id=z["track_id"],
                          type=z["type"], scalar=z["scalar"], edges=z["edges"])
    assert_identical(r, ref)


@pytest.mark.parametrize("cut", [1, 3])
@pytest.mark.parametrize("which", [2, 3], ids=["g3d_f32_noise", "g2d_f32_sep_offset"])
def test_stream_checkpoint_resume(ctx, which, cut):
    """A stream checkpointed after `cut` pushes, closed, restored on another
    context and fed the remaining timesteps gives the one-shot result."""
    case = _cases()[which]
    keep: list = []
    nt = case.local_dims[-1]
    mesh = api.regular_mesh_desc(case.local_dims, case.offset, case.global_dims)
    tmpl = api.field_desc(steps_of(case, 0), case.layout, case.ncomp, keep=keep)
    prm = api.params(case.sos_q)
    with api.Stream(ctx, mesh, tmpl, prm) as st:
        for t in range(cut):
            st.push(api.field_desc(steps_of(case, t), case.layout, case.ncomp, keep=keep))
        blob = st.checkpoint()
    with api.Context(0) as ctx2, api.Stream.restore(ctx2, blob) as st2:
        assert st2.info()[0] == cut
        for t in range(cut, nt):
            st2.push(api.field_desc(steps_of(case, t), case.layout, case.ncomp, keep=keep))
        assert_identical(st2.result(), one_shot(ctx, case, nt, False))
        # a checkpoint of the restored stream equals the original's layout
        assert len(st2.checkpoint()) >= len(blob)


def test_extruded_stream_checkpoint_resume(ctx):
    case = _ext_cases()[2]
    keep: list = []
    nv = case.coords.shape[0]
    nt = case.n_layers + 1
    mesh = api.extruded_mesh_desc(nv, case.cells, case.n_layers, keep)
    step = lambda t: [np.ascontiguousarray(a[t * nv:(t + 1) * nv]) for a in case.arrays]
    tmpl = api.field_desc(step(0), case.layout, case.ncomp, keep=keep)
    with api.Stream(ctx, mesh, tmpl, api.params(case.sos_q)) as st:
        for t in range(3):
            st.push(api.field_desc(step(t), case.layout, case.ncomp, keep=keep))
        blob = st.checkpoint()
    with api.Stream.restore(ctx, blob) as st2:
        for t in range(3, nt):
            st2.push(api.field_desc(step(t), case.layout, case.ncomp, keep=keep))
        assert_identical(st2.result(), ext_one_shot(ctx, case, nt))


def test_stream_restore_rejects_damaged_blobs(ctx):
    case = _cases()[2]
    keep: list = []
    mesh = api.regular_mesh_desc(case.local_dims, case.offset, case.global_dims)
    tmpl = api.field_desc(steps_of(case, 0), case.layout, case.ncomp, keep=keep)
    with api.Stream(ctx, mesh, tmpl, api.params(case.sos_q)) as st:
        st.push(api.field_desc(steps_of(case, 0), case.layout, case.ncomp, keep=keep))
        blob = st.checkpoint()
    for bad in (blob[:-1], b"XXXXXXXX" + blob[8:], blob[:64], blob + b"\0"):
        with pytest.raises(api.Ftk2bError) as e:
            api.Stream.restore(ctx, bad)
        assert e.value.status == api.INVALID_ARG
