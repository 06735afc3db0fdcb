"""The reference-side binding (include/vfb_virtualfluids_adapter.hpp) compiles against the
reference's own headers: the KernelImp subclass registered for "K17CompressibleNavierStokes"
(Kernel/Kernel.h:44-51, KernelFactoryImp.cpp:92-139), the BoundaryConditionFactory functions and
its subclass (BoundaryConditionFactory.h:50-160) and the GridScalingFactory functions
(GridScalingFactory.h:46). Only spdlog, a network-fetched dependency of the reference, is a stub
(tests/reference_stubs). Needs the reference tree (VFB_REFERENCE_DIR); skipped where it is absent."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
REF = Path(os.environ.get("VFB_REFERENCE_DIR", "/root/reference"))


@pytest.mark.skipif(not (REF / "src" / "gpu" / "core" / "Kernel" / "KernelImp.h").exists(),
                    reason="the reference source tree is not present")
@pytest.mark.parametrize("double_accuracy", [True, False], ids=["real=double", "real=float"])
def test_adapter_compiles_against_reference_headers(double_accuracy):
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [cxx, "-std=c++17", "-fsyntax-only", "-Wall", "-Werror=return-type",
           f"-I{ROOT / 'tests' / 'reference_stubs'}", f"-I{ROOT / 'include'}",
           f"-I{REF / 'src'}", f"-I{REF / 'src' / 'basics'}", f"-I{REF / 'src' / 'gpu'}",
           f"-I{REF / 'src' / 'gpu' / 'core'}", f"-I{REF / 'src' / 'lbm'}", f"-I{REF / '3rdParty' / 'cuda_samples'}",
           "-I/usr/local/cuda/include", str(ROOT / "tests" / "adapter_compile_check.cpp")]
    if double_accuracy:
        cmd.insert(2, "-DVF_DOUBLE_ACCURACY")
    r = subprocess.run(cmd, capture_output=True, text=True)
    errors = [l for l in r.stderr.splitlines() if "error" in l and str(REF) not in l.split(":")[0]]
    assert r.returncode == 0, r.stderr[-4000:]
    assert not errors
