"""Copies the reference's example tracking configurations and the round-trip
file its TrackingConfig::to_yaml wrote for one of them (its demo
examples/high_level_api_demo.cpp:53-57 loads high_level_example_config.yaml
and saves config_roundtrip.yaml) into tests/golden/tracker/, as fixtures for
the configuration reader of include/ftk2b/tracking_config.hpp.

    python tests/golden/make_tracker_fixtures.py REFERENCE_ROOT

REFERENCE_ROOT is the reference's source tree (the directory holding its
examples/ folder).
"""
import os
import shutil
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_tracker_fixtures.py REFERENCE_ROOT")
REF = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tracker")
FILES = ["high_level_example_config.yaml", "config_roundtrip.yaml", "cp_with_attributes.yaml",
         "sujudi_haimes_highlevel.yaml"]

if __name__ == "__main__":
    os.makedirs(OUT, exist_ok=True)
    for f in FILES:
        shutil.copyfile(os.path.join(REF, "examples", f), os.path.join(OUT, f))
        print("copied", f)
