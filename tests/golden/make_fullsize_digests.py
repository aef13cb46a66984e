"""Record the exact C restatement's results on the full-size workloads.

For each workload of tests/fullsize.py (c2 128^3 x 16 f64, c4 256^3 x 8 f32 +
noise, the 256 fields of c3) the field is generated on the GPU exactly as the
benchmark generates it, copied to the host, hashed, and run through the C
restatement (oracle/cp_oracle.c, every host core).  The digests of its output
go to tests/golden/fullsize_digests.json; for c4 the restatement also runs on
the field promoted to float64, and the features of that FP64 run are stored
in tests/golden/c4_fp64_oracle.npz (the position-error oracle of the refined
FP32 mode).

Needs a CUDA device (the generators run there) and the built restatement:
    python tests/golden/make_fullsize_digests.py [--out DIR] [c2] [c4] [c3]
(--out writes the two files to DIR instead of tests/golden/.)
"""
from __future__ import annotations

import json
import os
import platform
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import bridge  # noqa: E402
import fullsize  # noqa: E402

OUT_DIR = HERE


def restate(dims, m, host, q=fullsize.Q):
    keep: list = []
    mesh = bridge.make_regular_mesh(dims)
    fld = bridge.make_field(host, bridge.LAYOUT_MULTI, m, sos_q=q, keep=keep)
    return bridge.run_restatement(mesh, fld)


def main(args):
    import torch
    out_dir = OUT_DIR
    if args[:1] == ["--out"]:
        out_dir, args = args[1], args[2:]
    os.makedirs(out_dir, exist_ok=True)
    OUT = os.path.join(out_dir, "fullsize_digests.json")
    C4_FP64 = os.path.join(out_dir, "c4_fp64_oracle.npz")
    names = args or ["c2", "c4", "c3"]
    rec = json.load(open(OUT)) if os.path.exists(OUT) else {}
    rec["generated_on"] = {"torch": torch.__version__, "device": torch.cuda.get_device_name(0),
                           "host_cores": os.cpu_count(), "python": platform.python_version()}
    for name in names:
        t0 = time.time()
        if name in ("c2", "c4"):
            dims, m, dev = fullsize.c2_field() if name == "c2" else fullsize.c4_field()
            torch.cuda.synchronize()
            host = dev.cpu().numpy()
            del dev
            torch.cuda.empty_cache()
            entry = {"dims": dims, "field_sha256": fullsize.bytes_digest([host])}
            r = restate(dims, m, host)
            entry["result"] = fullsize.result_digest(r)
            entry["oracle_seconds"] = time.time() - t0
            if name == "c4":
                r64 = restate(dims, m, host.astype(np.float64))
                np.savez_compressed(C4_FP64, simplices=r64.simplices, lam=r64.lam,
                                    field_sha256=np.array(entry["field_sha256"]))
                entry["fp64_features"] = int(len(r64.track_id))
            rec[name] = entry
            print(f"{name}: {entry['result']['features']} features, {entry['result']['edges']} edges, "
                  f"{time.time() - t0:.1f} s", flush=True)
        elif name == "c3":
            fields = fullsize.c3_fields()
            torch.cuda.synchronize()
            hosts = [(d, m, f.cpu().numpy()) for d, m, f in fields]
            del fields
            torch.cuda.empty_cache()
            entry = {"fields": len(hosts), "fields_sha256": fullsize.bytes_digest([h for _, _, h in hosts]),
                     "results": []}
            for d, m, h in hosts:
                entry["results"].append(fullsize.result_digest(restate(d, m, h)))
            entry["oracle_seconds"] = time.time() - t0
            rec[name] = entry
            print(f"c3: {sum(r['features'] for r in entry['results'])} features over {len(hosts)} fields, "
                  f"{time.time() - t0:.1f} s", flush=True)
        json.dump(rec, open(OUT, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:])
