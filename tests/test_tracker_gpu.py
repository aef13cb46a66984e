"""The high-level tracker (include/ftk2b/feature_tracker.hpp) driven from a
YAML configuration, against the reference high-level flow: the reference's
engine on ExtrudedSimplicialMesh(RegularSimplicialMesh(spatial dims), nt - 1)
with the same multicomponent field and attribute specs
(feature_tracker.cpp:255-363, 480-520; engine.hpp:1143-1199).  Features,
float barycentrics, track ids, edges and attributes are identical, and the
text and JSON outputs are the reference's write_results format."""
import json
import os
import struct
import subprocess
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from ftk2_b200 import build as fb
from ftk2_b200 import synthetic as S
from oracle import bridge

pytestmark = pytest.mark.gpu


def f32bits(x):
    return struct.unpack("<I", struct.pack("<f", float(x)))[0]


def parse_dump(path):
    feats, edges = [], []
    for line in open(path):
        if line.startswith("F"):
            vs, bs, tr, at = line[1:].split("|")
            feats.append(([int(v) for v in vs.split()], [int(b, 16) for b in bs.split()], int(tr),
                          [int(a, 16) for a in at.split()]))
        elif line.startswith("E"):
            _, a, b = line.split()
            edges.append((int(a), int(b)))
    return feats, np.array(edges, dtype=np.uint32).reshape(-1, 2)


def write_config(path, out_dir, precision, attrs_yaml, vtp=True):
    path.write_text(
        "tracking:\n"
        "  feature: critical_points\n"
        "  input:\n"
        "    type: vector\n"
        "    variables: [V]\n"
        "  data:\n"
        "    source: arrays\n"
        "  mesh:\n"
        "    type: regular\n"
        "  execution:\n"
        "    backend: cuda\n"
        f"    precision: {precision}\n"
        "  output:\n"
        f"    trajectories: {out_dir}/traj.txt\n"
        f"    statistics: {out_dir}/stats.json\n"
        + (f"    format: vtp\n    filename: {out_dir}/traj.vtp\n" if vtp else "    format: text\n")
        + "    attributes:\n" + attrs_yaml)


def run_tracker(tmp_path, vec, extra, attrs_yaml, attrs_ref, precision):
    """vec: C-order (nt, [nz,] ny, nx, m); extra: name -> C-order array."""
    exe = fb.build_tracker_test()
    dt = "f64" if vec.dtype == np.float64 else "f32"
    args = []
    for name, a in [("V", vec)] + list(extra.items()):
        fp = tmp_path / f"{name}.bin"
        a.tofile(fp)
        args.append(f"{name}={fp}:{dt}:" + ",".join(str(d) for d in a.shape[::-1]))
    cfg = tmp_path / "cfg.yaml"
    write_config(cfg, tmp_path, precision, attrs_yaml)
    r = subprocess.run([exe, str(cfg), "--dump", str(tmp_path / "dump.txt")] + args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    feats, edges = parse_dump(tmp_path / "dump.txt")
    ref, ref_attrs = bridge.run_reference_tracked(vec, attrs_ref)
    return feats, edges, ref, ref_attrs


def expected_text(ref, ref_attrs, names):
    lines = ["# FTK2 Feature Complex", "# Feature: critical_points", f"# Num vertices: {len(ref.track_id)}"]
    if names:
        lines.append("# Attributes: " + ", ".join(names))
    lines += ["", "# Feature Elements:"]
    for i in range(len(ref.track_id)):
        s = f"{i}: track_id={int(ref.track_id[i])} type={int(ref.type[i])} scalar={float(ref.scalar[i]):g}"
        if names:
            s += " attrs=[" + ", ".join(f"{float(ref_attrs[i, j]):g}" for j in range(len(names))) + "]"
        lines.append(s)
    return "\n".join(lines) + "\n"


def check(tmp_path, feats, edges, ref, ref_attrs, n_attr):
    assert len(feats) == len(ref.track_id) > 0
    for i, (vs, bs, tr, at) in enumerate(feats):
        assert vs == [int(v) for v in ref.simplices[i]]
        assert bs == [f32bits(b) for b in ref.bary[i]]
        assert tr == int(ref.track_id[i])
        assert at[:n_attr] == [f32bits(a) for a in ref_attrs[i, :n_attr]], i
    assert np.array_equal(edges, ref.edges)


ATTRS_YAML = ("      - temperature\n"
              "      - name: vmag\n        source: V\n        type: magnitude\n"
              "      - name: vx\n        source: V\n        type: scalar\n        component: 0\n")


def test_tracker_2d_double_matches_reference_flow(tmp_path):
    v = S.analytic_2d(24, 20, 5)                                          # (nt, ny, nx, 2)
    temp = np.random.default_rng(3).standard_normal((5, 20, 24))          # Fortran [24, 20, 5]
    feats, edges, ref, ref_attrs = run_tracker(
        tmp_path, v, {"temperature": temp}, ATTRS_YAML, [(temp, False, -1), (v, True, -1), (v, False, 0)], "double")
    check(tmp_path, feats, edges, ref, ref_attrs, 3)
    # the reference's output files
    assert open(tmp_path / "traj.txt").read() == expected_text(ref, ref_attrs, ["temperature", "vmag", "vx"])
    st = json.load(open(tmp_path / "stats.json"))
    assert st == {"feature": "critical_points", "dimension": 2, "num_vertices": len(ref.track_id),
                  "precision": "double", "backend": "cuda"}
    root = ET.parse(tmp_path / "traj.vtp").getroot()
    piece = root.find("PolyData/Piece")
    assert int(piece.get("NumberOfPoints")) == len(ref.track_id)
    assert int(piece.get("NumberOfLines")) == len(ref.edges)


def test_tracker_3d_float_matches_reference_flow(tmp_path):
    g = S.gaussian_sum_gradient((13, 11, 9), 4, seed=5, n_blobs=10, dtype=np.float32, sigma=(2, 5))  # (4,9,11,13,3)
    temp = np.random.default_rng(4).standard_normal((4, 9, 11, 13)).astype(np.float32)
    feats, edges, ref, ref_attrs = run_tracker(
        tmp_path, g, {"temperature": temp}, ATTRS_YAML, [(temp, False, -1), (g, True, -1), (g, False, 0)], "float")
    check(tmp_path, feats, edges, ref, ref_attrs, 3)
    assert json.load(open(tmp_path / "stats.json"))["precision"] == "float"
