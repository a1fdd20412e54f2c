"""The checked build (libdgrain_checked.so, -DDGR_CHECKED): kernels that test every index
they gather from the connectivity before using it, recording an out-of-range one as
DGR_ERR_BAD_INDEX instead of reading or writing outside an array.  compute-sanitizer is
not available where these run, so this build plus exact comparison with the oracle on
small meshes stands in for it.  The parity and schedule tests run here once more against
the checked library, in a child process: they must pass unchanged (no index is out of
range, and the checks change no bits).
"""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_parity_suite_under_the_checked_build():
    sys.path.insert(0, os.path.join(ROOT, "dg-rain_b200"))
    import build

    lib = build.build_checked()
    assert os.path.exists(lib)
    env = dict(os.environ, DGRAIN_LIBRARY="checked")
    sel = ("compute2DL or limiter or single_step or run_bitexact or failure or nan_injection or extensions "
           "or large_mesh or schedules or ensemble_equals or failing_scenario or rk3_run")
    probe = ("import sys; sys.path.insert(0, 'dg-rain_b200'); import dgrain; print(dgrain._lib.LIB_PATH)")
    out = subprocess.run([sys.executable, "-c", probe], cwd=ROOT, env=env, capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip().endswith("libdgrain_checked.so"), out.stdout + out.stderr
    res = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-k", sel,
                          "tests/test_gpu_parity.py", "tests/test_gpu_ensemble.py", "tests/test_gpu_rk3.py"],
                         cwd=ROOT, env=env, capture_output=True, text=True)
    tail = (res.stdout + res.stderr)[-3000:]
    assert res.returncode == 0, tail
    assert " passed" in res.stdout, tail
