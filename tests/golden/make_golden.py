"""Generate the golden fixtures under tests/golden/ by running the reference's
own CPU engine (oracle/_ref/libftk2ref.so, built from the reference headers by
oracle/Makefile) on the seeded inputs of tests/cases.py.

Each fixture stores the reference's FeatureComplex flattened (sorted simplex
vertex ids, float barycentrics, track ids, scalars, edges), the solver's
lambdas in the field precision (side channel of oracle/ref_driver.cpp), and
the sha256 of the input bytes so that generator drift is detected.

Run here, where the reference tree exists:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import bridge  # noqa: E402
import cases  # noqa: E402


def main(names=None):
    for name, make in cases.GOLDEN_CASES.items():
        if names and name not in names:
            continue
        case = make()
        keep: list = []
        mesh, fld = cases.oracle_inputs(case, keep)
        t = time.time()
        r = bridge.run_reference(mesh, fld)
        dt = time.time() - t
        out = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(out, simplices=r.simplices, bary=r.bary, lam=r.lam,
                            track_id=r.track_id, type=r.type, scalar=r.scalar, edges=r.edges,
                            input_sha256=np.array(case.input_digest()),
                            reference_seconds=np.array(dt))
        print(f"{name}: {len(r.track_id)} features, {len(set(r.track_id.tolist()))} tracks, "
              f"{len(r.edges)} edges, reference {dt:.1f}s -> {os.path.basename(out)}")


if __name__ == "__main__":
    main(sys.argv[1:])
