"""The bounds-checked build (libvfb_checked.so) on the GPU, in a process of its own
(tests/bounds_check_run.py with VFB_LIBRARY=checked):

* with valid inputs it computes the same bits as the default build (the 10^3 cavity against the
  oracle) and records nothing;
* a fluid-node list or a BC list holding an index beyond the level's node count is caught by the
  kernels' own checks: the index is recorded (vfb_bounds_check_status) and replaced by the dummy
  node 0, so no access leaves the arrays; reading the record clears it.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def test_checked_build_matches_and_records_bad_indices(cuda):
    if not (ROOT / "virtualfluids_b200" / "libvfb_checked.so").exists():
        pytest.fail("libvfb_checked.so is missing: build it with python -m virtualfluids_b200.build --checked")
    env = dict(os.environ, VFB_LIBRARY="checked")
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "bounds_check_run.py")], capture_output=True, text=True,
                       env=env, cwd=str(ROOT), timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["checked"] == 1 and out["library"] == "libvfb_checked.so"
    assert out["bitwise_with_checks"]
    assert out["status_clean"] == [N.VFB_OK, 0, 0]
    st, bad, n = out["status_bad_fluid_index"]
    assert st == N.VFB_ERR_INVALID_ARGUMENT and n > 0 and bad == n + 5
    assert out["status_after_read"] == [N.VFB_OK, 0, 0]
    st, bad, n2 = out["status_bad_bc_index"]
    assert st == N.VFB_ERR_INVALID_ARGUMENT and n2 == n and bad == n + 11
