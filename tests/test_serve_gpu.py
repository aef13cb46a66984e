"""Serving loop (ftk2b_server_*): requests admitted as worker slots and HBM
budget free up, their device work overlapping; every result equals the same
request run alone, bit for bit (the path is deterministic, so the stated
tolerance is zero)."""
import numpy as np
import pytest

from ftk2_b200 import api
from ftk2_b200 import synthetic as S
import cases

pytestmark = pytest.mark.gpu


def identical(a, b):
    return (a.simplices.shape == b.simplices.shape and np.array_equal(a.simplices, b.simplices)
            and np.array_equal(a.track_id, b.track_id) and np.array_equal(a.edges, b.edges)
            and np.array_equal(a.lam, b.lam) and np.array_equal(a.bary, b.bary))


def mixed_requests(seed=0):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(10):
        if i % 2 == 0:
            n = int(rng.integers(128, 513))
            g = S.gaussian_sum_gradient((n, n), 2, seed=100 + i, n_blobs=int(rng.integers(8, 65)),
                                        dtype=np.float32, sigma=(3, 12))
            reqs.append(cases.Case(f"2d_{n}", "regular", 2, cases.MULTI, g, 1e6, [n, n, 2]))
        else:
            n = int(rng.integers(32, 97))
            g = S.gaussian_sum_gradient((n, n, n), 2, seed=200 + i, n_blobs=int(rng.integers(8, 65)),
                                        dtype=np.float32, sigma=(3, 10))
            reqs.append(cases.Case(f"3d_{n}", "regular", 3, cases.MULTI, g, 2.0 ** 20, [n, n, n, 2]))
    return reqs


def ext_case():
    coords, tets = S.extruded_tet_mesh(20, 18, 7, seed=5)
    vals = S.gaussian_sum_gradient_at(coords, 6, seed=55, n_blobs=16, sigma=(1.0, 3.0), drift=0.6)
    return cases.Case("ext", "extruded", 3, cases.PER_VERTEX, [vals[0], vals[1], vals[2]], 2.0 ** 20,
                      coords=coords, cells=tets, n_layers=5)


def alone(ctx, case):
    keep: list = []
    mesh, fld = cases.gpu_inputs(case, keep)
    return ctx.extract(mesh, fld, api.params(case.sos_q))


def run_mix(server, reqs, ext):
    keep: list = []
    nv = ext.coords.shape[0]
    sid = server.open_stream(api.extruded_mesh_desc(nv, ext.cells, ext.n_layers, keep),
                             api.field_desc([a[:nv] for a in ext.arrays], ext.layout, 3, keep=keep),
                             api.params(ext.sos_q))
    tickets = []
    for t in range(ext.n_layers + 1):
        # interleave stream pushes with the extraction requests
        if t < len(reqs):
            k: list = []
            mesh, fld = cases.gpu_inputs(reqs[t], k)
            tickets.append(("x", t, server.submit_extract(mesh, fld, api.params(reqs[t].sos_q), keep=k)))
        k = []
        step = api.field_desc([np.ascontiguousarray(a[t * nv:(t + 1) * nv]) for a in ext.arrays],
                              ext.layout, 3, keep=k)
        tickets.append(("p", t, server.submit_push(sid, step, keep=k)))
    for t in range(ext.n_layers + 1, len(reqs)):
        k = []
        mesh, fld = cases.gpu_inputs(reqs[t], k)
        tickets.append(("x", t, server.submit_extract(mesh, fld, api.params(reqs[t].sos_q), keep=k)))
    results = {}
    for kind, t, tk in tickets:
        res, st = server.wait(tk, timeout=120.0)
        assert st["status"] == 0 and st["latency_ms"] >= st["run_ms"] >= 0
        if kind == "x":
            results[t] = res
    sres = server.stream_result(sid)
    server.close_stream(sid)
    return results, sres


def test_mix_equals_alone(ctx):
    reqs = mixed_requests()
    ext = ext_case()
    with api.Server(0, n_slots=4) as sv:
        results, sres = run_mix(sv, reqs, ext)
        stats = sv.stats()
    for t, case in enumerate(reqs):
        assert identical(results[t], alone(ctx, case)), case.name
    assert identical(sres, alone(ctx, ext))
    assert stats["completed"] == len(reqs) + ext.n_layers + 1 and stats["failed"] == 0
    assert 0 < stats["p50_ms"] <= stats["p99_ms"] <= stats["max_ms"]
    assert stats["max_in_flight"] >= 2  # work of several requests overlapped


def test_budget_serialises_and_keeps_results(ctx):
    reqs = mixed_requests(seed=1)[:4]
    ext = ext_case()
    with api.Server(0, n_slots=4, hbm_budget=1) as sv:
        results, sres = run_mix(sv, reqs, ext)
        stats = sv.stats()
    assert stats["max_in_flight"] == 1  # nothing fits next to another request
    for t, case in enumerate(reqs):
        assert identical(results[t], alone(ctx, case))
    assert identical(sres, alone(ctx, ext))


def test_queue_limit_rejects_with_busy():
    g = S.gaussian_sum_gradient((96, 96, 96), 3, seed=3, n_blobs=32, dtype=np.float32, sigma=(3, 10))
    case = cases.Case("b", "regular", 3, cases.MULTI, g, 2.0 ** 20, [96, 96, 96, 3])
    busy = 0
    tickets = []
    with api.Server(0, n_slots=1, queue_limit=1) as sv:
        for _ in range(12):
            k: list = []
            mesh, fld = cases.gpu_inputs(case, k)
            try:
                tickets.append(sv.submit_extract(mesh, fld, api.params(case.sos_q), keep=k))
            except api.Ftk2bError as e:
                assert e.status == api.BUSY
                busy += 1
        for tk in tickets:
            sv.wait(tk, timeout=120.0, want_result=False)
        st = sv.stats()
    assert busy >= 1 and st["rejected"] == busy and st["completed"] == len(tickets)


def test_warm_runs_on_every_slot_and_stays_out_of_stats(ctx):
    case = mixed_requests(seed=2)[1]
    with api.Server(0, n_slots=3) as sv:
        k: list = []
        mesh, fld = cases.gpu_inputs(case, k)
        sv.warm(mesh, fld, api.params(case.sos_q))
        st = sv.stats()
        assert st["completed"] == 0 and st["submitted"] == 0
        t = sv.submit_extract(mesh, fld, api.params(case.sos_q), keep=k)
        res, s = sv.wait(t)
        assert s["phase_ms"][1] < 50.0  # replayed a cached graph, no capture of note
    assert identical(res, alone(ctx, case))
