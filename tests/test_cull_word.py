"""The per-vertex cull word of the fused cull (ftk2_b200/csrc/cp_cull.cuh),
compiled for the host and checked against a plain statement of its
definition on random and special high words (float and double, 2 and 3
components) -- no GPU needed."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cull_word_matches_its_definition(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    exe = str(tmp_path / "cull_word_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "cull_word_check.cu"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
