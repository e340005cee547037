"""The reference's own native parity suites, run live against this module.

The reference checks its native core with tests that skip unless the module
``blackhole_native`` imports (python/tests/test_native_sampler_parity.py:130-272,
python/tests/test_native_stokes_parity.py:38-46).  This test runs those files,
and the reference tests that report the native core's status
(test_benchmark.py, test_platform_probe.py), through the reference's own call
path -- native_loader.py imports ``blackhole_native`` by name and
native_kernels.py routes ``prefer_native=True`` calls to it with ``.tolist()``
copies -- with this package first on the path, on a GPU.

The reference's sources are not part of this repository: set
BHN_REFERENCE_PYTHON to a copy of the reference project's ``python/``
directory to run it; without it the test is skipped.
"""

from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
SUITES = ("test_native_sampler_parity.py", "test_native_stokes_parity.py", "test_benchmark.py",
          "test_platform_probe.py")
WHEN_INSTALLED = ("test_native_sample_brick_trilinear_matches_reference_when_installed",
                  "test_native_sample_and_step_stokes_matches_reference_when_installed",
                  "test_native_sample_and_step_stokes_invalid_policy_matches_reference_when_installed",
                  "test_native_stokes_rk2_brick_matches_reference_when_installed")

pytestmark = pytest.mark.gpu


def test_reference_native_suites_pass_unskipped():
    ref = os.environ.get("BHN_REFERENCE_PYTHON")
    if not ref:
        pytest.skip("BHN_REFERENCE_PYTHON (a copy of the reference's python/ directory) is not set")
    ref = Path(ref).resolve()
    files = [str(ref / "tests" / f) for f in SUITES if (ref / "tests" / f).exists()]
    assert len(files) == len(SUITES), f"reference test files missing under {ref / 'tests'}"
    env = dict(os.environ)
    # this package first, so ``import blackhole_native`` finds it; then the reference package
    env["PYTHONPATH"] = os.pathsep.join([str(REPO / "blackhole-sim_b200"), str(ref), env.get("PYTHONPATH", "")])
    env["PYTHONDONTWRITEBYTECODE"] = "1"
    # -p no:cacheprovider: nothing is written into the reference copy
    cmd = [sys.executable, "-m", "pytest", "-q", "-rA", "-p", "no:cacheprovider", "--rootdir", str(ref), *files]
    out = subprocess.run(cmd, capture_output=True, text=True, env=env, cwd=str(ref), timeout=900)
    report = out.stdout + out.stderr
    assert out.returncode == 0, report[-4000:]
    for name in WHEN_INSTALLED:
        assert re.search(rf"PASSED .*::{name}\b", report), f"{name} did not pass unskipped:\n{report[-4000:]}"
