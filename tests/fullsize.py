"""Full-size workloads of the critical-point path and digests of their results.

Shared by tests/golden/make_fullsize_digests.py (which runs the exact C
restatement once on each workload and records digests of its output) and by
tests/test_fullsize_gpu.py (which runs the CUDA path on the same workloads and
compares).  The fields are generated on the device exactly as the benchmark
generates them, so the digest of the field's bytes is recorded too: when a
regenerated field does not hash to the recorded value (another torch build,
another GPU), the test runs the restatement live instead of trusting the
recorded result digests.

Workloads (the benchmark's configurations, full size):

* ``c2``: 3D flow critical points, 128^3 x 16 float64 Gaussian-sum gradient
  (32 blobs, seed 1234), Q = 2^20;
* ``c4``: 256^3 x 8 float32 Gaussian-sum gradient (64 blobs of width
  U[16,48], gradient per box length) plus 1e-3 N(0,1) noise, Q = 2^20, the
  float engine's acceptance;
* ``c3``: 256 independent float32 fields (2D sides U[32,512], 3D sides
  U[16,96], nt U[2,8], 8-64 blobs), one batched call.
"""
from __future__ import annotations

import hashlib

import numpy as np

Q = 2.0 ** 20

# dtypes the digests are taken in (the restatement's and the library's
# result arrays are converted to these first)
DIGEST_DTYPES = {"simplices": np.uint64, "lam": np.float64, "bary": np.float32,
                 "track_id": np.uint64, "edges": np.uint32, "scalar": np.float32, "type": np.uint32}


def result_digest(r) -> dict:
    """Number of features and edges and a SHA-256 of every result array:
    vertex ids, lambda and float barycentric bits, track ids, edges, scalars,
    types."""
    out = {"features": int(len(r.track_id)), "edges": int(len(r.edges))}
    for name, dt in DIGEST_DTYPES.items():
        a = np.ascontiguousarray(np.asarray(getattr(r, name)).astype(dt, copy=False))
        out[name] = hashlib.sha256(a.tobytes()).hexdigest()
    return out


def bytes_digest(arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def c2_field():
    from ftk2_b200 import generate
    return [128, 128, 128, 16], 3, generate.c2_field()


def c4_field():
    from ftk2_b200 import generate
    return [256, 256, 256, 8], 3, generate.c4_field()


def c3_fields():
    from ftk2_b200 import generate
    return generate.c3_batch()


def positions(simplices: np.ndarray, lam: np.ndarray, dims) -> np.ndarray:
    """sum_i lambda_i p_i in grid units (x, y, z, t) of each feature."""
    rest = simplices.astype(np.int64)
    coords = []
    for n in dims:
        coords.append(rest % n)
        rest = rest // n
    P = np.stack(coords, -1).astype(np.float64)
    return (lam[:, :, None] * P).sum(1)
