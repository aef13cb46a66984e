"""Named workloads of the critical-point path, runnable from the command line
(used for profiling runs; the field is generated on the device):

    python -m ftk2_b200.workloads --case c2 --steps 3
    python -m ftk2_b200.workloads --case c2_small --steps 2 --no-tma

c2        3D flow CPs, plain drop-in: 128^3 x 16 float64, 32 blobs, Q = 2^20
c2_small  the same field definition on 128^3 x 4 (200 MB, larger than L2)
c4        precision workload: 256^3 x 8 float32 with 1e-3 noise
c4_small  the same on 256^3 x 2
c1        2D analytic 64 x 64 x 10 float64, Q = 1e6
c3        batch of 256 float32 fields (2D and 3D, uneven sizes), one batched call per step
contour   level set (threshold 0, Q = 2^20) of the 128^3 x 16 float64 Gaussian-sum potential
          whose gradient is c2
contour_small  the same potential on 128^3 x 8 (134 MB, larger than L2)
"""
from __future__ import annotations

import argparse
import time

from . import api, generate, synthetic


def make(case: str):
    import torch
    if case == "c2":
        return generate.c2_field(), [128, 128, 128, 16], 3, 2.0 ** 20
    if case == "c2_small":
        f = generate.gaussian_field_device((128, 128, 128), 4, seed=1234, n_blobs=32,
                                           dtype=torch.float64)
        return f, [128, 128, 128, 4], 3, 2.0 ** 20
    if case == "c4":
        return generate.c4_field(), [256, 256, 256, 8], 3, 2.0 ** 20
    if case == "c4_small":
        f = generate.gaussian_field_device((256, 256, 256), 2, seed=4321, n_blobs=64,
                                           dtype=torch.float32, noise=1e-3, sigma=(16.0, 48.0),
                                           scale=256.0)
        return f, [256, 256, 256, 2], 3, 2.0 ** 20
    if case == "c1":
        f = torch.from_numpy(synthetic.analytic_2d()).cuda()
        return f, [64, 64, 10], 2, 1e6
    raise ValueError(case)


def run_batch_case(args):
    """c3: the 256-field batch, one ftk2b_cp_run_batch per step."""
    import torch
    fields = generate.c3_batch(n=args.nfields)
    if args.field_dims:
        fields = [f for f in fields if len(f[0]) - 1 == args.field_dims]
    torch.cuda.synchronize()
    with api.Context(0) as ctx:
        if args.no_graphs:
            ctx.set_option(api.OPT_USE_GRAPHS, 0)
        if args.no_tma:
            ctx.set_option(api.OPT_DISABLE_TMA, 1)
        if args.tchunk:
            ctx.set_option(api.OPT_BATCH_TIME_CHUNK, args.tchunk)
        keep: list = []
        meshes = [api.regular_mesh_desc(d) for d, _, _ in fields]
        fds = [api.field_desc(f, api.LAYOUT_MULTICOMPONENT, m, keep=keep) for _, m, f in fields]
        prms = [api.params(2.0 ** 20) for _ in fields]
        for i in range(args.steps):
            t = time.perf_counter()
            n = ctx.run_batch(meshes, fds, prms)
            x, tot, _ = ctx.last_timing()
            print(f"step {i}: {n} features  cull {x:.3f} ms  pipeline {tot:.3f} ms  "
                  f"host {1e3 * (time.perf_counter() - t):.3f} ms  "
                  f"candidates={ctx.get_option(api.INFO_LAST_CANDIDATES)}  "
                  f"tested={ctx.get_option(api.INFO_LAST_TESTED)}", flush=True)


def run_contour_case(args):
    """contour: one ftk2b_contour_extract per step on the device-resident potential."""
    import torch
    dims, nt = (128, 128, 128), (16 if args.case == "contour" else 8)
    pot = generate.gaussian_potential_device(dims, nt, seed=1234, n_blobs=32)
    torch.cuda.synchronize()
    mesh = api.regular_mesh_desc([*dims, nt])
    with api.Context(0) as ctx:
        for i in range(args.steps):
            t = time.perf_counter()
            r = ctx.contour(mesh, pot, 0.0, 2.0 ** 20)
            print(f"step {i}: {len(r.track_id)} features {len(r.cells)} cells {r.n_tracks} tracks  "
                  f"device {r.device_ms:.3f} ms  host {1e3 * (time.perf_counter() - t):.3f} ms", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="c2_small")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--no-tma", action="store_true")
    ap.add_argument("--refined", action="store_true")
    ap.add_argument("--tchunk", type=int, default=0, help="time steps per extraction block (0 = all)")
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--nfields", type=int, default=256, help="c3: fields in the batch")
    ap.add_argument("--field-dims", type=int, default=0, choices=(0, 2, 3),
                    help="c3: keep only the batch's 2D or 3D fields (0: all)")
    ap.add_argument("--cull-mode", type=int, default=2,
                    help="0: per-vertex cull words only; 1: tile statistics first; 2: the faster, timed once (default)")
    args = ap.parse_args()
    import torch
    if args.case == "c3":
        return run_batch_case(args)
    if args.case in ("contour", "contour_small"):
        return run_contour_case(args)
    field, dims, m, q = make(args.case)
    torch.cuda.synchronize()
    with api.Context(0) as ctx:
        if args.no_tma:
            ctx.set_option(api.OPT_DISABLE_TMA, 1)
        if args.tchunk:
            ctx.set_option(api.OPT_TIME_CHUNK, args.tchunk)
        if args.no_graphs:
            ctx.set_option(api.OPT_USE_GRAPHS, 0)
        ctx.set_option(api.OPT_CULL_MODE, args.cull_mode)
        keep: list = []
        mesh = api.regular_mesh_desc(dims)
        fd = api.field_desc(field, api.LAYOUT_MULTICOMPONENT, m, keep=keep)
        prm = api.params(q, precision=api.PRECISION_REFINED if args.refined else api.PRECISION_EXACT)
        for i in range(args.steps):
            t = time.perf_counter()
            n, ne = ctx.run(mesh, fd, prm)
            x, tot, _ = ctx.last_timing()
            print(f"step {i}: {n} features {ne} edges  extract {x:.3f} ms  pipeline {tot:.3f} ms  "
                  f"host {1e3 * (time.perf_counter() - t):.3f} ms  tma={ctx.get_option(api.INFO_LAST_TMA)}  "
                  f"cull_mode={ctx.get_option(api.INFO_LAST_CULL_MODE)}  "
                  f"candidates={ctx.get_option(api.INFO_LAST_CANDIDATES)}  "
                  f"tested={ctx.get_option(api.INFO_LAST_TESTED)}", flush=True)


if __name__ == "__main__":
    main()
