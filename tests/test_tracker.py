"""Configuration reader of the high-level tracker (include/ftk2b/
tracking_config.hpp), on the CPU: the reference's own example configurations
parse to the fields its TrackingConfig::from_yaml_node gives them
(tracking_config.cpp:167-401), the round trip through to_yaml reproduces the
file the reference wrote for its example, and invalid configurations are
rejected with the reference's messages."""
import os
import subprocess

import pytest
import yaml

from ftk2_b200 import build as fb

GOLD = os.path.join(os.path.dirname(__file__), "golden", "tracker")


@pytest.fixture(scope="module")
def exe():
    return fb.build_tracker_test()


def dump(exe, path):
    out = subprocess.run([exe, path, "--config-dump"], capture_output=True, text=True, check=True).stdout
    d = {}
    for line in out.splitlines():
        k, v = line.split("=", 1)
        d.setdefault(k, []).append(v)
    return d


def expected(path):
    """The fields the reference's from_yaml_node reads, from PyYAML."""
    t = yaml.safe_load(open(path))["tracking"]
    inp, data, mesh = t.get("input", {}), t.get("data", {}), t.get("mesh", {})
    exe_, out = t.get("execution", {}), t.get("output", {})
    attrs = []
    for a in out.get("attributes", []) or []:
        if isinstance(a, str):
            attrs.append(f"{a},{a},scalar,-1")
        else:
            name = a.get("name", "")
            attrs.append(f"{name},{a.get('source', name)},{a.get('type', 'scalar')},{a.get('component', -1)}")
    e = {
        "dimension": [str(t.get("dimension", 0))],
        "input.variable": list(inp.get("variables", [])),
        "input.field_type": [inp.get("field_type", "gradient")],
        "mesh.dimension": [str(x) for x in mesh.get("dimensions", [])],
        "execution.precision": [exe_.get("precision", "double")],
        "execution.threads": [str(exe_.get("threads", -1))],
        "output.trajectories": [out.get("trajectories", "")],
        "output.statistics": [out.get("statistics", "")],
        "output.format": [out.get("format", "auto")],
        "output.attribute": attrs,
        "data.inline_stream": ["1" if data.get("stream") else "0"],
    }
    return e


@pytest.mark.parametrize("name", ["high_level_example_config.yaml", "cp_with_attributes.yaml",
                                  "sujudi_haimes_highlevel.yaml"])
def test_reference_examples_parse_like_the_reference(exe, name):
    got = dump(exe, os.path.join(GOLD, name))
    for k, v in expected(os.path.join(GOLD, name)).items():
        assert got.get(k, []) == v, (k, got.get(k), v)


def test_round_trip_reproduces_the_reference_output(exe):
    # the reference's demo loads high_level_example_config.yaml and writes
    # config_roundtrip.yaml with TrackingConfig::to_yaml
    out = subprocess.run([exe, os.path.join(GOLD, "high_level_example_config.yaml"), "--config-only"],
                         capture_output=True, text=True, check=True).stdout
    assert out == open(os.path.join(GOLD, "config_roundtrip.yaml")).read()


def test_yaml_subset_edge_cases(exe, tmp_path):
    p = tmp_path / "c.yaml"
    p.write_text(
        "# leading comment\n"
        "tracking:\n"
        "  feature: CP   # alias, any case\n"
        "  dimension: 3\n"
        "  input:\n"
        "    type: gradient_vector\n"
        "    variables:\n"
        "    - \"u v\"\n"
        "    - 'w#1'\n"
        "    field_type: gradient\n"
        "  data: {}\n".replace("  data: {}\n", "  data:\n    source: arrays\n    stream: ~\n") +
        "  mesh:\n"
        "    dimensions: [8, 9, 10]\n"
        "  execution:\n"
        "    backend: GPU\n"
        "    precision: single\n"
        "  output:\n"
        "    trajectories: out.txt\n"
        "    attributes:\n"
        "      - name: a\n"
        "        component: 2\n"
        "      - b\n")
    d = dump(exe, str(p))
    assert d["feature"] == ["critical_points"]
    assert d["input.type"] == ["gradient_vector"]
    assert d["input.variable"] == ["u v", "w#1"]
    assert d["mesh.dimension"] == ["8", "9", "10"]
    assert d["execution.backend"] == ["cuda"]
    assert d["execution.precision"] == ["float"]
    assert d["data.inline_stream"] == ["0"]
    assert d["output.attribute"] == ["a,a,scalar,2", "b,b,scalar,-1"]


@pytest.mark.parametrize("bad,msg", [
    ("dimension: 5", "dimension must be 0 (auto-derive), 2, or 3"),
    ("feature: vortices", "Unknown feature type: vortices"),
])
def test_invalid_configurations_are_rejected(exe, tmp_path, bad, msg):
    p = tmp_path / "bad.yaml"
    p.write_text("tracking:\n  " + bad + "\n  input:\n    type: vector\n    variables: [v]\n"
                 "  output:\n    trajectories: x.txt\n")
    r = subprocess.run([exe, str(p), "--config-dump"], capture_output=True, text=True)
    assert r.returncode == 1 and msg in r.stderr
