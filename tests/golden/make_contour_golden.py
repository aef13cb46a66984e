"""Generate tests/golden/contour/*.npz, tests/golden/fiber/*.npz and
tests/golden/fiber_surface/*.npz, tests/golden/contour_extruded/*.npz and
tests/golden/fiber_extruded/*.npz and tests/golden/fiber_surface_extruded/*.npz
(the one-worker engine, whose numbering of the triangles found while patching
is deterministic) by running
the reference's own CPU engine with ContourPredicate<T> (one worker thread,
oracle/_ref/libftk2ref1t.so) and FiberPredicate<T> (oracle/_ref/libftk2ref.so),
built from the reference headers by oracle/Makefile, on the seeded inputs of
tests/contour_cases.py.

Each fixture stores the sha256 of the input bytes and, per output array
(simplices, bary, lam, track_id, scalar, cells), its sha256 and shape; the
small cases also store the arrays themselves.

Run here, where the reference tree exists:  python tests/golden/make_contour_golden.py
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import bridge  # noqa: E402
import contour_cases  # noqa: E402

FULL_ARRAYS_BELOW = 20000  # features


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run(case):
    keep: list = []
    mesh = bridge.make_regular_mesh(case["local_dims"], case["offset"], case["global_dims"])
    fld = bridge.make_field([case["field"]], bridge.LAYOUT_SEPARATE, 1, sos_q=case["q"], keep=keep)
    r, cells = bridge.run_reference_contour(mesh, fld, case["threshold"])
    return {"simplices": r.simplices, "bary": r.bary, "lam": r.lam, "track_id": r.track_id,
            "scalar": r.scalar, "cells": cells}


def run_fiber(case):
    keep: list = []
    mesh = bridge.make_regular_mesh(case["local_dims"], case["offset"], case["global_dims"])
    fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep)
    r = bridge.run_reference_fiber(mesh, fld, case["thresholds"])
    return {"simplices": r.simplices, "bary": r.bary, "lam": r.lam, "track_id": r.track_id,
            "scalar": r.scalar, "edges": r.edges}


def main_fiber(names=None):
    out_dir = os.path.join(HERE, "fiber")
    os.makedirs(out_dir, exist_ok=True)
    for name, make in contour_cases.FIBER_CASES.items():
        if names and name not in names:
            continue
        case = make()
        t = time.time()
        res = run_fiber(case)
        dt = time.time() - t
        rec = {"input_sha256": np.array(digest(np.concatenate([a.reshape(-1) for a in case["fields"]]))),
               "reference_seconds": np.array(dt)}
        rec.update(res)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **rec)
        print(f"{name}: {len(res['track_id'])} features, {len(set(res['track_id'].tolist()))} tracks, "
              f"{len(res['edges'])} edges, reference {dt:.1f}s")


def main_extruded(names=None):
    out_dir = os.path.join(HERE, "contour_extruded")
    os.makedirs(out_dir, exist_ok=True)
    for name, make in contour_cases.EXTRUDED_CASES.items():
        if names and name not in names:
            continue
        case = make()
        keep: list = []
        mesh = bridge.make_extruded_mesh(case["coords"], case["cells"], case["n_layers"], keep)
        fld = bridge.make_field([case["field"]], bridge.LAYOUT_SEPARATE, 1, sos_q=case["q"], keep=keep)
        t = time.time()
        r, cells = bridge.run_reference_contour(mesh, fld, case["threshold"])
        dt = time.time() - t
        rec = {"input_sha256": np.array(digest(case["field"])), "reference_seconds": np.array(dt),
               "simplices": r.simplices, "bary": r.bary, "lam": r.lam, "track_id": r.track_id,
               "scalar": r.scalar, "cells": cells}
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **rec)
        print(f"{name}: {len(r.track_id)} features, {len(set(r.track_id.tolist()))} tracks, "
              f"{len(cells)} cells, reference {dt:.1f}s")


def main_fiber_extruded(names=None):
    out_dir = os.path.join(HERE, "fiber_extruded")
    os.makedirs(out_dir, exist_ok=True)
    for name, make in contour_cases.FIBER_EXTRUDED_CASES.items():
        if names and name not in names:
            continue
        case = make()
        keep: list = []
        mesh = bridge.make_extruded_mesh(case["coords"], case["cells"], case["n_layers"], keep)
        fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep)
        t = time.time()
        r = bridge.run_reference_fiber(mesh, fld, case["thresholds"])
        dt = time.time() - t
        rec = {"input_sha256": np.array(digest(np.concatenate([a.reshape(-1) for a in case["fields"]]))),
               "reference_seconds": np.array(dt), "simplices": r.simplices, "bary": r.bary, "lam": r.lam,
               "track_id": r.track_id, "scalar": r.scalar, "edges": r.edges}
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **rec)
        print(f"{name}: {len(r.track_id)} features, {len(set(r.track_id.tolist()))} tracks, "
              f"{len(r.edges)} edges, reference {dt:.1f}s")


def main_fiber_surface(names=None):
    out_dir = os.path.join(HERE, "fiber_surface")
    os.makedirs(out_dir, exist_ok=True)
    for name, make in contour_cases.FIBER_SURFACE_CASES.items():
        if names and name not in names:
            continue
        case = make()
        keep: list = []
        mesh = bridge.make_regular_mesh(case["local_dims"], case["offset"], case["global_dims"])
        fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep)
        t = time.time()
        r, cells = bridge.run_reference_fiber_surface(mesh, fld, case["thresholds"])
        dt = time.time() - t
        rec = {"input_sha256": np.array(digest(np.concatenate([a.reshape(-1) for a in case["fields"]]))),
               "reference_seconds": np.array(dt), "simplices": r.simplices, "bary": r.bary, "lam": r.lam,
               "track_id": r.track_id, "scalar": r.scalar, "cells": cells}
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **rec)
        print(f"{name}: {len(r.track_id)} features, {len(set(r.track_id.tolist()))} tracks, "
              f"{len(cells)} triangles, reference {dt:.1f}s")


def main_fiber_surface_extruded(names=None):
    out_dir = os.path.join(HERE, "fiber_surface_extruded")
    os.makedirs(out_dir, exist_ok=True)
    for name, make in contour_cases.FIBER_SURFACE_EXTRUDED_CASES.items():
        if names and name not in names:
            continue
        case = make()
        keep: list = []
        mesh = bridge.make_extruded_mesh(case["coords"], case["cells"], case["n_layers"], keep)
        fld = bridge.make_field(list(case["fields"]), bridge.LAYOUT_SEPARATE, 2, sos_q=case["q"], keep=keep)
        t = time.time()
        r, cells = bridge.run_reference_fiber_surface(mesh, fld, case["thresholds"], one_thread=True)
        dt = time.time() - t
        rec = {"input_sha256": np.array(digest(np.concatenate([a.reshape(-1) for a in case["fields"]]))),
               "reference_seconds": np.array(dt), "simplices": r.simplices, "bary": r.bary, "lam": r.lam,
               "track_id": r.track_id, "scalar": r.scalar, "cells": cells}
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **rec)
        print(f"{name}: {len(r.track_id)} features, {len(set(r.track_id.tolist()))} tracks, "
              f"{len(cells)} triangles, reference {dt:.1f}s")


def main(names=None):
    out_dir = os.path.join(HERE, "contour")
    os.makedirs(out_dir, exist_ok=True)
    for name, make in contour_cases.CASES.items():
        if names and name not in names:
            continue
        case = make()
        t = time.time()
        res = run(case)
        dt = time.time() - t
        rec = {"input_sha256": np.array(digest(case["field"])), "reference_seconds": np.array(dt)}
        for k, v in res.items():
            rec[k + "_sha256"] = np.array(digest(v))
            rec[k + "_shape"] = np.array(v.shape, dtype=np.int64)
            if len(res["track_id"]) < FULL_ARRAYS_BELOW:
                rec[k] = v
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **rec)
        print(f"{name}: {len(res['track_id'])} features, {len(set(res['track_id'].tolist()))} tracks, "
              f"{len(res['cells'])} cells, reference {dt:.1f}s")


if __name__ == "__main__":
    main(sys.argv[1:])
    main_fiber(sys.argv[1:])
    main_fiber_surface(sys.argv[1:])
    main_extruded(sys.argv[1:])
    main_fiber_extruded(sys.argv[1:])
    main_fiber_surface_extruded(sys.argv[1:])
