"""The build with the device bounds checks compiled in (-DFTK2B_CHECKED) on a
B200: every case of tests/checked_cases.py (2D and 3D+t, float and double, the
short and the general post chain, a batch) runs in a child process that loads
that build; no check may fail (a failure would make the call return
FTK2B_INTERNAL and the child exit non-zero), and every result must equal the
normal build's bit for bit."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))

pytestmark = pytest.mark.gpu


def test_checked_build_equals_normal_build(tmp_path):
    from ftk2_b200 import api
    import checked_cases

    if not os.path.exists(api.CHECKED_LIB_PATH):
        pytest.fail("checked build missing: run __graft_entry__.build()")
    out = str(tmp_path / "checked.npz")
    env = dict(os.environ, FTK2B_CHECKED="1", PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    proc = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_cases.py"), out], env=env,
                          capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    got = np.load(out)
    with api.Context(0) as ctx:
        want = checked_cases.run_all(ctx)
    assert sorted(got.files) == sorted(want)
    for k, v in want.items():
        g = got[k]
        assert g.shape == v.shape, k
        if v.dtype.kind == "f":
            assert np.array_equal(g.view(np.uint8), v.view(np.uint8)), k
        else:
            assert np.array_equal(g, v), k
    # the general post chain ran (more features than the short chain takes)
    assert len(want["noise3d.track"]) > 16384
