"""Benchmark of the critical-point tracking path (one JSON line on rank 0).

Workload: 3D flow critical points, plain drop-in -- a 128^3 x 16 float64
3-component Gaussian-sum gradient field (32 seeded blobs, sigma U[4,12]
voxels, drift U[-0.5,0.5] voxel/step), tetrahedra of the 4D Kuhn spacetime mesh
tested with the exact integer SoS at Q = 2^20, then canonical ordering, star
edges and trajectories.

A step = one full extraction (execute + get_complex equivalent) of the field.
  value : simplices/s with the field resident in HBM (ftk2b_cp_run), device
          timed with CUDA events on the context's stream, max over ranks.
  e2e   : the same through ftk2b_cp_extract with pinned host input and host
          output (H2D + D2H inside the timed region).
The field (805 MB) is larger than L2 (126 MB), so no flush is needed.

--impl reference times the reference's own CPU engine (oracle/_ref, built from
the reference's headers) on 32^3 x 2-vertex sub-boxes of the same field, one
per step, and reports the exact C restatement's all-core rate beside it.
With --gpus N > 1 every rank runs an independent replica on its own field
(weak scaling); there is no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D CP tracking simplices/s & HBM GB/s, batched vs plain; serve p50/p99 ms"
UNIT = "simplices/s"
DIMS = (128, 128, 128)
NT = 16
SOS_Q = 2.0 ** 20
CONFIG = {"workload": "3D flow critical points, plain drop-in: 128^3 x 16 float64 3-component "
                      "Gaussian-sum gradient (32 blobs), 4D Kuhn tets, SoS Q=2^20",
          "grid": [128, 128, 128, 16], "ncomp": 3, "field_dtype": "float64", "sos_q": SOS_Q,
          "units": "tets = every 3-face of the 4D Kuhn top cells, upper-boundary faces included "
                   "(the set the reference's phase 1 + phase 2 test): 1,860,189,828 at 128^3 x 16",
          "l2": "inputs larger than L2 (805 MB field vs 126 MB L2)"}
# the reference's CPU engine runs on spatial sub-boxes of this size, one time
# step of hypercubes each (a 32^3 x 2-vertex RegularSimplicialMesh sub-box)
REF_SUB = (32, 32, 32, 2)


def kuhn_chains(d: int, m: int):
    """Vertex masks 1..m of every m-simplex type of the Kuhn d-cube (strictly
    growing chains of corner masks), mesh.hpp:123-237."""
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


def kuhn_simplex_count(dims, m: int) -> int:
    """m-simplices of the Kuhn triangulation of a regular grid of ``dims``
    vertices, upper-boundary faces included: one per (corner vertex, chain)
    whose top mask stays inside the grid.  Pure Python, so the reference arm
    loads none of this repository's libraries."""
    total = 0
    for ch in kuhn_chains(len(dims), m):
        c = 1
        for k, n in enumerate(dims):
            c *= n - 1 if (ch[-1] >> k) & 1 else n
        total += c
    return total


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """SM clocks and throttle reasons sampled through NVML every few
    milliseconds while the timed region runs (read-only queries)."""

    def __init__(self, gpu: int, period_s: float = 0.001):
        self.gpu = gpu
        self.period = period_s
        self.samples: list[tuple[float, int]] = []
        self.max_mhz = None
        self._stop = threading.Event()
        self.ok = False

    def __enter__(self):
        try:
            import pynvml as N
            N.nvmlInit()
            self.N = N
            self.h = N.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = float(N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM))
            self.ok = True
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
        except Exception:
            self.ok = False
        return self

    def _poll(self):
        N = self.N
        while not self._stop.is_set():
            try:
                mhz = float(N.nvmlDeviceGetClockInfo(self.h, N.NVML_CLOCK_SM))
                reasons = int(N.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((mhz, reasons))
            except Exception:
                pass
            self._stop.wait(self.period)

    def __exit__(self, *a):
        self._stop.set()
        if self.ok:
            self.t.join(timeout=2)

    def summary(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"], "samples": 0}
        N = self.N
        bits = {"hw_slowdown": N.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": N.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": N.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": N.nvmlClocksEventReasonSwPowerCap}
        seen = set()
        for _, r in self.samples:
            for nm, b in bits.items():
                if r & b:
                    seen.add(nm)
        mhz = [m for m, _ in self.samples]
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(seen), "samples": len(mhz)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_launch():
    """DRAM bytes of one extraction launch from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "extract_regular_c2_traffic.json")
    try:
        return float(json.load(open(p))["dram_bytes_per_launch"])
    except Exception:
        return None


def ref_sub_box(rng, corner=DIMS, nt=NT):
    """A random REF_SUB sub-box (offset) inside a grid of ``corner`` x nt."""
    return [int(rng.integers(0, corner[i] - REF_SUB[i] + 1)) for i in range(3)] + \
        [int(rng.integers(0, nt - REF_SUB[3] + 1))]


def run_reference_sub_box(lo, seed=1234):
    """The reference's CPU engine (oracle/_ref) on one REF_SUB sub-box of the
    headline field at offset ``lo``; the sub-box's values are generated on the
    host from the same blob draws and handed to the engine as a mesh of its
    own (multicomponent arrays are read at global coordinates, so an offset
    mesh would need the whole field).  Returns (simplices, seconds)."""
    from oracle import bridge
    from ftk2_b200 import synthetic
    f = synthetic.gaussian_sum_gradient(REF_SUB[:3], REF_SUB[3], seed=seed, n_blobs=32, box=DIMS,
                                        origin=lo[:3], t0=lo[3])
    keep: list = []
    mesh = bridge.make_regular_mesh(list(REF_SUB))
    fld = bridge.make_field(f, bridge.LAYOUT_MULTI, 3, sos_q=SOS_Q, keep=keep)
    t = time.perf_counter()
    bridge.run_reference(mesh, fld)
    return kuhn_simplex_count(REF_SUB, 3), time.perf_counter() - t


def cpu_baseline_sample(budget_s=20.0):
    """The reference's CPU engine on REF_SUB sub-boxes of the headline field
    until ~budget_s seconds have been spent; returns (simplices/s, sample)."""
    import numpy as np
    rng = np.random.default_rng(0)
    total_s, total_n, boxes = 0.0, 0, 0
    while total_s < budget_s and boxes < 16:
        n, t = run_reference_sub_box(ref_sub_box(rng))
        total_s += t
        total_n += n
        boxes += 1
    sample = (f"{boxes} sub-boxes of {REF_SUB[0]}x{REF_SUB[1]}x{REF_SUB[2]}x{REF_SUB[3]} vertices "
              f"(one time step of 31^3 hypercubes) of the same field, reference engine (oracle/_ref) "
              f"execute+get_complex, {total_s:.1f} s")
    return total_n / total_s, sample


def restatement_rate(budget_s=10.0):
    """The exact multithreaded C restatement (oracle/cp_oracle.c, every host
    core) on 64^3 x 4 sub-boxes of the headline field: simplices/s."""
    import numpy as np
    from oracle import bridge
    from ftk2_b200 import synthetic
    sub = (64, 64, 64, 4)
    rng = np.random.default_rng(2)
    total_s, total_n, boxes = 0.0, 0, 0
    while total_s < budget_s and boxes < 8:
        lo = [int(rng.integers(0, DIMS[i] - sub[i] + 1)) for i in range(3)] + [int(rng.integers(0, NT - sub[3] + 1))]
        f = synthetic.gaussian_sum_gradient(sub[:3], sub[3], seed=1234, n_blobs=32, box=DIMS,
                                            origin=lo[:3], t0=lo[3])
        keep: list = []
        mesh = bridge.make_regular_mesh(list(sub))
        fld = bridge.make_field(f, bridge.LAYOUT_MULTI, 3, sos_q=SOS_Q, keep=keep)
        t = time.perf_counter()
        bridge.run_restatement(mesh, fld)
        total_s += time.perf_counter() - t
        total_n += kuhn_simplex_count(sub, 3)
        boxes += 1
    return {"value": total_n / total_s, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
            "sample": f"{boxes} sub-boxes of {sub[0]}x{sub[1]}x{sub[2]}x{sub[3]} vertices, the exact C "
                      f"restatement on every host core, {total_s:.1f} s"}


def _positions(simplices, lam, dims):
    """Barycentric positions sum_i lambda_i p_i in grid units (x, y, z, t)."""
    import numpy as np
    ids = simplices.astype(np.int64)
    coords = []
    rest = ids
    for n in dims:
        coords.append(rest % n)
        rest = rest // n
    P = np.stack(coords, -1).astype(np.float64)  # (n, m+1, 4)
    return (lam[:, :, None] * P).sum(1)


def precision_c4(ctx, steps=5):
    """Precision workload: 256^3 x 8 float32 Gaussian-sum gradient (64 blobs)
    plus 1e-3 noise.  The refined-FP32 path (exact int64 SoS, float solve for
    acceptance, reported positions from an FP32 solve plus one FP64 refinement
    step) against the plain FP64 drop-in on the same field promoted to
    float64, on the same GPU; positions compared on the simplices both accept."""
    import numpy as np
    import torch
    from ftk2_b200 import api, generate
    dims = [256, 256, 256, 8]
    f32 = generate.c4_field()
    torch.cuda.synchronize()
    keep: list = []
    mesh = api.regular_mesh_desc(dims)
    nsimp = api.simplex_count(mesh, 3)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr)

    def timed(fd, prm):
        for _ in range(3):
            ctx.run(mesh, fd, prm)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        xs = []
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(steps):
            ctx.run(mesh, fd, prm)
            xs.append(ctx.last_timing()[0])
        ev1.record(stream)
        torch.cuda.synchronize()
        modes.append(ctx.get_option(api.INFO_LAST_CULL_MODE))
        return ev0.elapsed_time(ev1) / steps, statistics.mean(xs), ctx.fetch()

    modes: list = []  # cull mode the autotuner chose per timed form

    fd32 = api.field_desc(f32, api.LAYOUT_MULTICOMPONENT, 3, keep=keep)
    ms_r, x_r, res_r = timed(fd32, api.params(SOS_Q, precision=api.PRECISION_REFINED))
    ms_e32, x_e32, res_e32 = timed(fd32, api.params(SOS_Q))
    f64 = f32.double()
    del keep[:]
    del f32
    fd64 = api.field_desc(f64, api.LAYOUT_MULTICOMPONENT, 3, keep=keep)
    ms_64, x_64, res_64 = timed(fd64, api.params(SOS_Q))
    del keep[:]
    del f64
    torch.cuda.empty_cache()

    def rows(a):
        return {tuple(r): i for i, r in enumerate(a.tolist())}

    r64 = rows(res_64.simplices)
    common = [(i, r64[tuple(r)]) for i, r in enumerate(res_r.simplices.tolist()) if tuple(r) in r64]
    ia = np.array([c[0] for c in common], dtype=np.int64)
    ib = np.array([c[1] for c in common], dtype=np.int64)
    pos64 = _positions(res_64.simplices[ib], res_64.lam[ib], dims)
    err_r = np.abs(_positions(res_r.simplices[ia], res_r.lam[ia], dims) - pos64).max(1)
    err_e = np.abs(_positions(res_e32.simplices[ia], res_e32.lam[ia], dims) - pos64).max(1)
    peak, _ = measured_peak()
    alg32 = 3 * 4 * 256 ** 3 * 8
    return {
        "workload": "256^3 x 8 float32, 64 blobs + 1e-3 noise, Q=2^20",
        "simplices": int(nsimp),
        "refined_fp32": {"simplices_per_s": nsimp / (ms_r / 1e3), "ms_per_step": ms_r, "extract_ms": x_r,
                         "features": int(len(res_r.track_id)), "cull_mode": modes[0],
                         "hbm_frac_extract": alg32 / (x_r / 1e3) / 1e9 / peak},
        "exact_fp32": {"simplices_per_s": nsimp / (ms_e32 / 1e3), "ms_per_step": ms_e32},
        "plain_fp64": {"simplices_per_s": nsimp / (ms_64 / 1e3), "ms_per_step": ms_64, "extract_ms": x_64,
                       "features": int(len(res_64.track_id)), "cull_mode": modes[2]},
        "speedup_refined_vs_fp64": ms_64 / ms_r,
        "position_error_grid_units": {
            "compared": int(len(ia)), "refined_max": float(err_r.max()) if len(ia) else None,
            "refined_mean": float(err_r.mean()) if len(ia) else None,
            "refined_frac_le_1e-9": float((err_r <= 1e-9).mean()) if len(ia) else None,
            "fp32_unrefined_max": float(err_e.max()) if len(ia) else None,
            "fp32_unrefined_mean": float(err_e.mean()) if len(ia) else None},
        "sets": {"fp32_only": int(len(res_r.track_id) - len(ia)), "fp64_only": int(len(res_64.track_id) - len(ia)),
                 "note": "acceptance follows the reference per precision: the float engine solves in float, "
                         "the double engine in double (zero_crossing.hpp with T = float / double)"},
    }


def run_reference_arm(args, rank, world):
    """The reference's own CPU engine (oracle/_ref, built from its headers,
    execute + get_complex) on REF_SUB sub-boxes of the headline field, one
    sub-box per step, with the std::thread workers it starts itself.  Loads
    none of this repository's CUDA code: simplex counts are pure Python."""
    if rank != 0:
        return 0
    from oracle import bridge
    import numpy as np
    if not bridge.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference engine build oracle/_ref missing"}))
        return 0
    rng = np.random.default_rng(1)
    for _ in range(args.warmup):
        run_reference_sub_box(ref_sub_box(rng))
    tot_n, tot_t = 0, 0.0
    for _ in range(args.steps):
        n, t = run_reference_sub_box(ref_sub_box(rng))
        tot_n += n
        tot_t += t
    value = tot_n / tot_t
    cores = os.cpu_count() or 1
    sample = (f"one {REF_SUB[0]}x{REF_SUB[1]}x{REF_SUB[2]}x{REF_SUB[3]}-vertex sub-box (31^3 hypercubes, "
              f"one time step) of the workload field per step through the reference engine "
              f"(std::thread parallel_for; phase 1 serial)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": dict(CONFIG, parallelism=f"replicas{world}"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "restatement": restatement_rate()}
    print(json.dumps(line))
    return 0


def contour_c2(ctx, steps=3):
    """Level sets (ContourPredicate) of the 3D plain drop-in generator's scalar,
    128^3 x 16 float64, threshold 0, Q = 2^20: device pipeline time per call
    (CUDA events inside ftk2b_contour_extract) and mesh edges per second; the
    result copy to the host is outside it and reported as wall time."""
    import numpy as np
    import torch
    from ftk2_b200 import api, generate
    dims, nt = (128, 128, 128), 16
    pot = generate.gaussian_potential_device(dims, nt, seed=1234, n_blobs=32)
    torch.cuda.synchronize()
    mesh = api.regular_mesh_desc([*dims, nt])
    r = ctx.contour(mesh, pot, 0.0, 2.0 ** 20)  # warm-up (buffers, first launches)
    dev_ms, wall_ms = [], []
    for _ in range(steps):
        t = time.perf_counter()
        r = ctx.contour(mesh, pot, 0.0, 2.0 ** 20)
        wall_ms.append((time.perf_counter() - t) * 1e3)
        dev_ms.append(r.device_ms)
    ms = float(np.median(dev_ms))
    nbytes = pot.numel() * 8
    del pot
    out = {"workload": "level set of the 128^3 x 16 f64 Gaussian-sum potential (32 blobs), threshold 0",
           "mesh_edges": int(r.n_simplices), "features": int(len(r.track_id)), "cells": int(len(r.cells)),
           "tracks": int(r.n_tracks), "device_ms": ms, "edges_per_s": r.n_simplices / (ms * 1e-3),
           "field_read_gbs": nbytes / (ms * 1e-3) / 1e9, "wall_ms_with_result_copy": float(np.median(wall_ms))}
    # the reference's level-set engine on the host cores, on a bounded sample:
    # its own moving-sphere test field (32^3 x 10 float32)
    try:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import contour_cases
        from oracle import bridge
        case = contour_cases.moving_sphere()
        keep: list = []
        rmesh = bridge.make_regular_mesh(case["local_dims"])
        rfld = bridge.make_field([case["field"]], bridge.LAYOUT_SEPARATE, 1, sos_q=case["q"], keep=keep)
        t = time.perf_counter()
        ref, _ = bridge.run_reference_contour(rmesh, rfld, 0.0, one_thread=False)
        secs = time.perf_counter() - t
        dims = case["local_dims"]
        edges = 0
        for e in range(1, 16):
            c = 1
            for k in range(4):
                c *= dims[k] - 1 if (e >> k) & 1 else dims[k]
            edges += c
        out["cpu_baseline"] = {"value": edges / secs, "unit": "edges/s", "cores": os.cpu_count() or 1,
                               "kind": "reference", "features": int(len(ref.track_id)),
                               "sample": f"the reference's moving-sphere level set, 32^3 x 10 float32 ({edges} edges), "
                                         f"reference engine execute+get_complex, {secs:.1f} s"}
    except Exception as e:  # the reference build travels prebuilt; report its absence
        out["cpu_baseline"] = {"unavailable": str(e)[:200]}
    return out


def fiber_surface_bench(ctx, steps=3):
    """Fiber surfaces (FiberPredicate on 3D+t) of two Gaussian-sum potentials,
    96^3 x 8 float64 (seeds 1234, 4321), thresholds at 0: device time per call
    and mesh triangles per second."""
    import numpy as np
    import torch
    from ftk2_b200 import api, generate
    dims, nt = (96, 96, 96), 8
    f = generate.gaussian_potential_device(dims, nt, seed=1234, n_blobs=32)
    g = generate.gaussian_potential_device(dims, nt, seed=4321, n_blobs=32)
    torch.cuda.synchronize()
    keep: list = []
    mesh = api.regular_mesh_desc([*dims, nt])
    fd = api.field_desc([f, g], api.LAYOUT_SEPARATE, 2, keep=keep)
    r = ctx.fiber_surface(mesh, fd, (0.0, 0.0), 2.0 ** 20)
    dev_ms = []
    for _ in range(steps):
        r = ctx.fiber_surface(mesh, fd, (0.0, 0.0), 2.0 ** 20)
        dev_ms.append(r.device_ms)
    ms = float(np.median(dev_ms))
    del f, g, fd
    keep.clear()
    return {"workload": "fiber surface of two 96^3 x 8 f64 Gaussian-sum potentials (32 blobs each), thresholds 0",
            "mesh_triangles": int(r.n_simplices), "features": int(len(r.track_id)), "triangles": int(len(r.cells)),
            "tracks": int(r.n_tracks), "device_ms": ms, "mesh_triangles_per_s": r.n_simplices / (ms * 1e-3)}


def batched_c3(ctx, steps=5, check=True):
    """Batched workload: 256 independent float32 fields (2D sides U[32,512],
    3D sides U[16,96], nt U[2,8], 8-64 blobs), device-resident.  Plain = one
    extraction call per field; batched = one ftk2b_cp_run_batch call for all
    of them.  With check, every field's batched result is compared with its
    plain result."""
    import numpy as np
    import torch
    from ftk2_b200 import api, generate
    t0 = time.perf_counter()
    fields = generate.c3_batch()
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    keep: list = []
    meshes = [api.regular_mesh_desc(d) for d, _, _ in fields]
    fds = [api.field_desc(f, api.LAYOUT_MULTICOMPONENT, m, keep=keep) for _, m, f in fields]
    prms = [api.params(SOS_Q) for _ in fields]
    nsimp = sum(api.simplex_count(md, len(d) - 1) for md, (d, _, _) in zip(meshes, fields))
    nbytes = sum(f.numel() * f.element_size() for _, _, f in fields)
    n2 = sum(1 for d, _, _ in fields if len(d) == 3)

    def plain_pass():
        nf = 0
        for md, fd, p in zip(meshes, fds, prms):
            nf += ctx.run(md, fd, p)[0]
        return nf

    for _ in range(2):
        plain_pass()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(steps):
        nf_plain = plain_pass()
    ms_plain = (time.perf_counter() - t) * 1e3 / steps
    for _ in range(3):
        ctx.run_batch(meshes, fds, prms)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    xs = []
    torch.cuda.synchronize()
    t = time.perf_counter()
    ev0.record(stream)
    for _ in range(steps):
        nf_batch = ctx.run_batch(meshes, fds, prms)
        xs.append(ctx.last_timing())
    ev1.record(stream)
    torch.cuda.synchronize()
    ms_batch_wall = (time.perf_counter() - t) * 1e3 / steps
    ms_batch = ev0.elapsed_time(ev1) / steps
    cull_ms = statistics.mean(x[0] for x in xs)
    out = {
        "workload": "256 fields: 2D sides U[32,512] / 3D sides U[16,96], nt U[2,8], 8-64 blobs, float32, Q=2^20",
        "fields": len(fields), "fields_2d": n2, "fields_3d": len(fields) - n2, "simplices": int(nsimp),
        "input_bytes": int(nbytes), "generate_s": gen_s, "features": int(nf_batch),
        "plain": {"ms_per_pass": ms_plain, "simplices_per_s": nsimp / (ms_plain / 1e3), "calls": len(fields)},
        "batched": {"ms_per_pass": ms_batch, "ms_per_pass_wall": ms_batch_wall,
                    "simplices_per_s": nsimp / (ms_batch / 1e3), "cull_ms": cull_ms,
                    "cull_hbm_gbs": nbytes / (cull_ms / 1e3) / 1e9},
        "speedup_batched_vs_plain": ms_plain / ms_batch,
    }
    if check:
        batch = ctx.fetch_batch()
        same = 0
        for md, fd, p, b in zip(meshes, fds, prms, batch):
            r = ctx.extract(md, fd, p)
            same += int(np.array_equal(r.simplices, b.simplices) and np.array_equal(r.track_id, b.track_id)
                        and np.array_equal(r.edges, b.edges) and np.array_equal(r.lam, b.lam)
                        and np.array_equal(r.bary, b.bary))
        out["identical_to_plain"] = f"{same}/{len(batch)}"
        out["features_plain"] = int(nf_plain)
    del fds, keep, fields
    return out


def targets_summary(line):
    """The targets of the workload set in one short object, printed last on
    the line: HBM roofline fractions of the plain FP64 drop-in (128^3 x 16)
    and of the 256^3 x 8 float32 workload (extraction kernels alone and whole
    step), the refined-FP32 form against the plain FP64 drop-in on the same
    field, its position error, the batch and serving figures."""
    peak = line["roofline"]["peak"]
    p = line.get("precision", {})
    b = line.get("batched", {})
    sv = line.get("serve", {})
    alg32 = 3 * 4 * 256 ** 3 * 8
    r32 = p.get("refined_fp32", {})
    out = {
        "peak_gbs": peak,
        "c2_extract_frac": line["roofline"]["frac"],
        "c2_step_frac": line["roofline"]["algorithmic_bytes"] / (line["ms_per_step"] / 1e3) / 1e9 / peak,
        "c4_extract_frac": r32.get("hbm_frac_extract"),
        "c4_step_frac": alg32 / (r32["ms_per_step"] / 1e3) / 1e9 / peak if r32 else None,
        "c4_refined_vs_fp64_same_field": p.get("speedup_refined_vs_fp64"),
        "c4_refined_max_pos_err": p.get("position_error_grid_units", {}).get("refined_max"),
        "c4_sets_differ": (p.get("sets", {}).get("fp32_only"), p.get("sets", {}).get("fp64_only")),
        "c3_cull_frac": b.get("batched", {}).get("cull_hbm_gbs", 0.0) / peak if b else None,
        "c3_batched_vs_plain": b.get("speedup_batched_vs_plain"),
        "c3_identical": b.get("identical_to_plain"),
        "serve_p50_p99_ms": (sv.get("p50_ms"), sv.get("p99_ms")),
        "serve_req_s": sv.get("throughput_req_s"),
        "serve_capacity_req_s": line.get("serve_sweep", {}).get("capacity_req_s"),
    }
    return {k: (float(f"{v:.4g}") if isinstance(v, float) else v) for k, v in out.items()}


def run_sharded(args, rank, world, local):
    """The headline field split into time slabs, one per rank (each rank
    generates and holds only its slab, as separate component arrays indexed
    from the slab's offset), each slab extracted on its GPU and the exchange
    of ftk2_b200.sharded run over NCCL; a step = the slab extractions plus the
    exchange, timed on the device, max over ranks.  value = simplices of the
    whole mesh per second (strong scaling)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from ftk2_b200 import api, generate, sharded
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        import socket
        sk = socket.socket()
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
        sk.close()
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    dims = list(DIMS) + [NT]
    bounds = sharded.slab_bounds(NT, world)
    ctx = api.Context(local)
    keep: list = []
    fd = mesh = None
    if rank < len(bounds):
        t0, t1 = bounds[rank]
        f = generate.gaussian_field_device(DIMS, t1 - t0 + 1, seed=1234, n_blobs=32, dtype=torch.float64, t0=t0)
        comps = [f[..., j].contiguous() for j in range(3)]
        del f
        fd = api.field_desc(comps, api.LAYOUT_SEPARATE, 3, keep=keep)
        mesh = sharded.slab_mesh(dims, t0, t1)
    prm = api.params(SOS_Q)

    def extractor(m, a, b):
        return ctx.extract(mesh, fd, prm)

    for _ in range(max(args.warmup, 3)):
        sharded.extract_sharded(dims, None, 3, extractor=extractor)
    torch.cuda.synchronize()
    dist.barrier()
    t = time.perf_counter()
    for _ in range(args.steps):
        shard = sharded.extract_sharded(dims, None, 3, extractor=extractor)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t) * 1e3 / args.steps
    tt = torch.tensor([ms], dtype=torch.float64, device="cuda" if world > 1 else "cpu")
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    ms = float(tt.item())
    nsimp = kuhn_simplex_count(dims, 3)
    nfeat = torch.tensor([len(shard.track_id)], dtype=torch.int64, device="cuda" if world > 1 else "cpu")
    if world > 1:
        dist.all_reduce(nfeat)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": nsimp / (ms / 1e3), "unit": UNIT, "n_gpus": world,
                          "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": dict(CONFIG, parallelism=f"time-slabs{world}"),
                          "result": {"features": int(nfeat.item()), "simplices": nsimp},
                          "timing": "host wall clock around the slab extractions and the exchange, max over ranks"}),
              flush=True)
    ctx.close()
    dist.barrier()
    dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ftk2b", choices=["ftk2b", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="only the headline workload (no precision / serving measurements)")
    ap.add_argument("--serve-seconds", type=float, default=5.0)
    ap.add_argument("--shard", action="store_true",
                    help="split the headline field into time slabs across the ranks (strong scaling) "
                         "instead of one replica per rank")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.shard:
        return run_sharded(args, rank, world, local)

    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist
    from ftk2_b200 import api, generate

    ctx = api.Context(local)
    # independent replica per rank: seed offset by rank
    field = generate.gaussian_field_device(DIMS, NT, seed=1234 + rank, n_blobs=32,
                                           dtype=torch.float64)
    torch.cuda.synchronize()
    keep: list = []
    mesh = api.regular_mesh_desc(list(DIMS) + [NT])
    fdev = api.field_desc(field, api.LAYOUT_MULTICOMPONENT, 3, keep=keep)
    prm = api.params(SOS_Q)
    nsimp = api.simplex_count(mesh, 3)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr)

    for _ in range(max(args.warmup, 3)):
        ctx.run(mesh, fdev, prm)
    _, _, launches0 = ctx.last_timing()

    # ---- device-resident timed region
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    extract_ms = []
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            nf, ne = ctx.run(mesh, fdev, prm)
            xms, _, _ = ctx.last_timing()
            extract_ms.append(xms)
        ev1.record(stream)
        torch.cuda.synchronize()
    _, _, launches1 = ctx.last_timing()
    cull_mode = ctx.get_option(api.INFO_LAST_CULL_MODE)
    ms_total = ev0.elapsed_time(ev1)
    if pg:
        t = torch.tensor([ms_total], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_step = ms_total / args.steps
    value = world * nsimp / (ms_step / 1000.0)

    # ---- end to end through the public API with host buffers
    host = field.cpu().numpy()
    pinned = torch.from_numpy(host).pin_memory()
    fhost = api.field_desc(pinned.numpy(), api.LAYOUT_MULTICOMPONENT, 3, keep=keep)
    res = ctx.extract(mesh, fhost, prm)  # warm the host path
    # bytes ftk2b_cp_fetch copies back: vertex ids, float barycentrics, four
    # double lambdas, scalar and track id per feature, plus the edge list
    nfe = len(res.track_id)
    d2h = nfe * (8 * 4 + 4 * 4 + 8 * 4 + 4 + 8) + res.edges.nbytes
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e2e_steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        res = ctx.extract(mesh, fhost, prm)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if pg:
        t = torch.tensor([e2e_s], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * nsimp / e2e_s

    # ---- roofline of the dominant kernel (fused extraction)
    peak, peak_kind = measured_peak()
    alg_bytes = 3 * 8 * DIMS[0] * DIMS[1] * DIMS[2] * NT
    xms = statistics.mean(extract_ms)
    achieved = alg_bytes / (xms / 1000.0) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic_per_launch(),
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else "fallback 6650 GB/s",
            "kernel": "extract_regular_kernel<double,4>" if cull_mode == 0
            else "plane_stats_stream_kernel + tile_runs_kernel + run_cull_kernel <double,4>",
            "cull_mode": cull_mode,
            "kernel_ms": xms, "algorithmic_bytes": alg_bytes}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG, parallelism=f"replicas{world}"),
            "result": {"features": int(nf), "edges": int(ne), "simplices": int(nsimp)},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(host.nbytes),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_s * 1000.0},
            "roofline": roof, "clocks": clocks.summary(),
            "gpu_launches": int(launches1 - launches0)}
    del pinned, host
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sample = cpu_baseline_sample()
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1,
                                "kind": "reference", "sample": sample}
    # the extra lines are one-GPU measurements (and their CPU baselines belong
    # to rank 0 at N = 1): with several ranks only the replica line is timed
    if not args.no_extra and world == 1:
        del field, fdev
        keep.clear()
        torch.cuda.empty_cache()
        line["precision"] = precision_c4(ctx)
        # refined FP32 (c4) against the plain FP64 drop-in workload (c2, this line's value)
        line["precision"]["refined_fp32_vs_plain_fp64_c2"] = line["precision"]["refined_fp32"]["simplices_per_s"] / value
        torch.cuda.empty_cache()
        line["batched"] = batched_c3(ctx)
        torch.cuda.empty_cache()
        from ftk2_b200 import serving
        line["serve"] = serving.run(duration_s=args.serve_seconds, device=local)
        line["serve"].pop("slowest", None)
        torch.cuda.empty_cache()
        line["serve_sweep"] = serving.sweep(device=local)
        torch.cuda.empty_cache()
        line["contour"] = contour_c2(ctx)
        torch.cuda.empty_cache()
        line["fiber_surface"] = fiber_surface_bench(ctx)
        line["targets"] = targets_summary(line)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
