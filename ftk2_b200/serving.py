"""Serving workload: a Poisson request stream through the ftk2b server.

Requests arrive with exponential inter-arrival times at ``rate`` per second:
with probability ``p_push`` the next timestep of a long-running extruded-mesh
stream (a jittered 100 x 100 triangulated plane extruded into 40 layers of
tets, about 400k vertices, one timestep per push, its previous timestep and
union-find state resident on the device), otherwise a one-shot extraction of
a two-timestep slab, 2D with sides U[256, 2048] or 3D with sides U[64, 192]
(float32 Gaussian-sum gradients, 8-64 blobs, from pinned host memory, so the
host-to-device copy is part of each request's latency).

Inputs are drawn from pre-generated pools (``pool`` fields per kind, stream
timesteps cycling through ``n_steps`` generated ones) so that generation does
not compete with serving.  Latency = submission -> completion, reported per
kind and overall as p50 / p99.
"""
from __future__ import annotations

import statistics
import threading
import time

import numpy as np

from . import api, generate, synthetic


def _pct(v, p):
    if not v:
        return None
    s = sorted(v)
    k = max(1, int(np.ceil(p * len(s))))
    return s[k - 1]


def make_pools(seed: int = 5, pool: int = 6, n_steps: int = 16, plane=(100, 100, 40)):
    import torch
    rng = np.random.default_rng(seed)
    slabs = []
    for i in range(pool):
        n = int(rng.integers(256, 2049))
        f = generate.gaussian_field_device((n, n), 2, seed=1000 + i, n_blobs=int(rng.integers(8, 65)),
                                           dtype=torch.float32, sigma=(8.0, 64.0))
        slabs.append(("2d", [n, n, 2], 2, 1e6, f.cpu().pin_memory()))
        del f
    for i in range(pool):
        n = int(rng.integers(64, 193))
        f = generate.gaussian_field_device((n, n, n), 2, seed=2000 + i, n_blobs=int(rng.integers(8, 65)),
                                           dtype=torch.float32, sigma=(4.0, 16.0))
        slabs.append(("3d", [n, n, n, 2], 3, 2.0 ** 20, f.cpu().pin_memory()))
        del f
    coords, tets = synthetic.extruded_tet_mesh(*plane, seed=seed)
    nv = coords.shape[0]
    vals = generate.gaussian_at_device(coords, n_steps, seed=3000, n_blobs=48, sigma=(3.0, 9.0), drift=0.8,
                                       dtype=torch.float32)
    steps = []
    for t in range(n_steps):
        steps.append([vals[j, t * nv:(t + 1) * nv].cpu().pin_memory() for j in range(3)])
    torch.cuda.synchronize()
    return slabs, (coords, tets, steps)


def run(duration_s: float = 5.0, rate: float = 200.0, p_push: float = 0.2, n_slots: int = 4,
        seed: int = 5, pools=None, device: int = 0, warm_pushes: int = 17):
    """Runs the request stream for ``duration_s`` seconds of arrivals and
    returns a summary dict (latencies in ms).  Before the timed region every
    pool field is extracted once on every slot and the stream takes
    ``warm_pushes`` timesteps, one full cycle of the generated steps (its
    first push prepares the base mesh on the device; the warm-up push
    latencies are reported as ``stream_setup_ms``)."""
    slabs, (coords, tets, steps) = pools if pools is not None else make_pools(seed)
    nv = coords.shape[0]
    rng = np.random.default_rng(seed + 1)
    lat = {"2d": [], "3d": [], "push": []}
    detail: list = []  # (submit offset s, kind, latency ms, queue ms, slot, host phases ms)
    simplices = [0]
    errors: list = []
    with api.Server(device, n_slots=n_slots) as sv:
        keep: list = []
        mesh = api.extruded_mesh_desc(nv, tets, 1, keep)
        tmpl = api.field_desc([s.numpy() for s in steps[0]], api.LAYOUT_PER_VERTEX, 3, keep=keep)
        sid = sv.open_stream(mesh, tmpl, api.params(2.0 ** 20))
        # every pool shape once on every slot (buffers and cached graphs), and
        # the stream, before the timed region (not counted)
        # largest first: buffers reach their final size before any graph is
        # cached over them (a later regrowth would drop the cached graphs)
        for kind, dims, m, q, f in sorted(slabs, key=lambda e: -e[4].numel()):
            k: list = []
            sv.warm(api.regular_mesh_desc(dims), api.field_desc(f.numpy(), api.LAYOUT_MULTICOMPONENT, m, keep=k),
                    api.params(q))
        setup_ms = []
        step_i = 0
        for _ in range(warm_pushes):
            k = []
            fd = api.field_desc([s.numpy() for s in steps[step_i % len(steps)]], api.LAYOUT_PER_VERTEX, 3, keep=k)
            step_i += 1
            _, st = sv.wait(sv.submit_push(sid, fd, keep=k), want_result=False)
            setup_ms.append(st["latency_ms"])
        pending: list = []
        cv = threading.Condition()
        done_submitting = [False]

        def waiter():
            while True:
                with cv:
                    while not pending and not done_submitting[0]:
                        cv.wait()
                    if not pending:
                        return
                    kind, tk, t_sub = pending.pop(0)
                try:
                    _, st = sv.wait(tk, want_result=False)
                    lat[kind].append(st["latency_ms"])
                    detail.append((round(t_sub, 4), kind, st["latency_ms"], st["queue_ms"], st["slot"],
                                   [round(x, 3) for x in st["phase_ms"]]))
                    simplices[0] += st["n_simplices"]
                except api.Ftk2bError as e:
                    errors.append(str(e))

        th = threading.Thread(target=waiter, daemon=True)
        th.start()
        base = sv.stats()["completed"]
        t0 = time.perf_counter()
        t_next = 0.0
        n_sub = 0
        while t_next < duration_s:
            now = time.perf_counter() - t0
            if t_next > now:
                time.sleep(t_next - now)
            if rng.random() < p_push:
                k = []
                fd = api.field_desc([s.numpy() for s in steps[step_i % len(steps)]], api.LAYOUT_PER_VERTEX, 3,
                                    keep=k)
                step_i += 1
                tk = sv.submit_push(sid, fd, keep=k)
                kind = "push"
            else:
                kind, dims, m, q, f = slabs[int(rng.integers(0, len(slabs)))]
                k = []
                tk = sv.submit_extract(api.regular_mesh_desc(dims),
                                       api.field_desc(f.numpy(), api.LAYOUT_MULTICOMPONENT, m, keep=k),
                                       api.params(q), keep=k)
            n_sub += 1
            with cv:
                pending.append((kind, tk, time.perf_counter() - t0))
                cv.notify()
            t_next += float(rng.exponential(1.0 / rate))
        with cv:
            done_submitting[0] = True
            cv.notify()
        th.join()
        wall = time.perf_counter() - t0
        stats = sv.stats()
        stream_res = sv.stream_result(sid)
        sv.close_stream(sid)
    everything = lat["2d"] + lat["3d"] + lat["push"]
    out = {
        "offered_rate_req_s": rate, "duration_s": duration_s, "slots": n_slots, "submitted": n_sub,
        "completed": stats["completed"] - base, "failed": stats["failed"], "errors": errors[:3],
        "throughput_req_s": len(everything) / wall, "wall_s": wall,
        "p50_ms": _pct(everything, 0.50), "p99_ms": _pct(everything, 0.99), "max_ms": max(everything),
        "mean_ms": statistics.mean(everything),
        "by_kind": {k: {"n": len(v), "p50_ms": _pct(v, 0.5), "p99_ms": _pct(v, 0.99)} for k, v in lat.items()},
        "extract_simplices_per_s": simplices[0] / wall,
        "max_in_flight": stats["max_in_flight"], "hbm_reserved_peak_bytes": stats["hbm_reserved_peak"],
        "slowest": sorted(detail, key=lambda r: -r[2])[:5],
        "stream_first_push_ms": setup_ms[0] if setup_ms else None,
        "stream_warm_pushes": len(setup_ms),
        "stream": {"timesteps": step_i, "features": int(len(stream_res.track_id)),
                   "tracks": int(stream_res.n_tracks), "vertices_per_step": nv},
    }
    return out


def sweep(rates=(200, 500, 1000, 2000, 4000, 8000), duration_s: float = 1.5, n_slots: int = 4,
          one_slot_rates=(1000, 4000), seed: int = 5, device: int = 0):
    """Offered-rate sweep: throughput and p50 / p99 latency per Poisson rate
    (the same request mix and pools), until the server saturates; plus the
    same load on one worker slot at some rates, which shows what admitting
    requests into free slots while others run buys over a single queue."""
    pools = make_pools(seed)
    rows = []

    def row(rate, slots):
        r = run(duration_s=duration_s, rate=rate, n_slots=slots, seed=seed, pools=pools, device=device,
                warm_pushes=2)
        return {"offered_req_s": rate, "slots": slots, "served_req_s": round(r["throughput_req_s"], 1),
                "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "failed": r["failed"],
                "max_in_flight": r["max_in_flight"]}

    for rate in rates:
        rows.append(row(rate, n_slots))
    for rate in one_slot_rates:
        rows.append(row(rate, 1))
    best = max((x for x in rows if x["slots"] == n_slots), key=lambda x: x["served_req_s"])
    return {"duration_s_per_rate": duration_s, "rows": rows, "capacity_req_s": best["served_req_s"]}


if __name__ == "__main__":
    import json
    import sys
    d = float(sys.argv[1]) if len(sys.argv) > 1 else 5.0
    print(json.dumps(run(duration_s=d), indent=1))
