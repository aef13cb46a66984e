"""Extraction cases run through both library builds by tests/test_checked_gpu.py:
the normal one in the test process and the build with the device bounds
checks compiled in (FTK2B_CHECKED=1) in a child process, which runs this file
as a script and saves every result to the .npz named on its command line."""
from __future__ import annotations

import sys

import numpy as np

from ftk2_b200 import api
from ftk2_b200 import synthetic as S


def cases():
    """(name, mesh dims, field array, components, Q) of every single-field case."""
    rng = np.random.default_rng(7)
    noise3 = rng.standard_normal((4, 20, 18, 16, 3)).astype(np.float64)  # many features: the general post chain
    return [
        ("c1_2d", [64, 64, 10], S.analytic_2d(64, 64, 10), 2, 1e6),
        ("gauss3d_f64", [40, 36, 32, 6], S.gaussian_sum_gradient((40, 36, 32), 6, seed=5, n_blobs=12), 3, 2.0 ** 20),
        ("gauss3d_f32", [40, 36, 32, 6],
         S.gaussian_sum_gradient((40, 36, 32), 6, seed=6, n_blobs=12).astype(np.float32), 3, 2.0 ** 20),
        ("noise3d", [16, 18, 20, 4], noise3, 3, 2.0 ** 20),
    ]


def run_all(ctx) -> dict:
    out = {}
    for name, dims, field, m, q in cases():
        r = ctx.extract(api.regular_mesh_desc(dims), api.field_desc(field, api.LAYOUT_MULTICOMPONENT, m),
                        api.params(q))
        out[f"{name}.simplices"] = r.simplices
        out[f"{name}.lam"] = r.lam
        out[f"{name}.track"] = r.track_id
        out[f"{name}.edges"] = r.edges
    cs = cases()[:2]  # one dtype per batch: the 2D and the 3D+t float64 fields
    res = ctx.extract_batch([api.regular_mesh_desc(d) for _, d, _, _, _ in cs],
                            [api.field_desc(f, api.LAYOUT_MULTICOMPONENT, m) for _, _, f, m, _ in cs],
                            [api.params(q) for _, _, _, _, q in cs])
    for (name, *_), r in zip(cs, res):
        out[f"batch.{name}.simplices"] = r.simplices
        out[f"batch.{name}.lam"] = r.lam
        out[f"batch.{name}.track"] = r.track_id
        out[f"batch.{name}.edges"] = r.edges
    return out


if __name__ == "__main__":
    with api.Context(0) as ctx:
        np.savez(sys.argv[1], **run_all(ctx))
