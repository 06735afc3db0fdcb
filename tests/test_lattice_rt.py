"""The run-time direction helpers of the link-parallel BC kernels (csrc/lattice.cuh: component
masks, shift_class_rt, order_rt, weight_rt, cdot_link) against the compile-time lattice
functions of the unrolled kernels. The check compiles tests/lattice_rt_check.cu as host code with
nvcc and runs it on the CPU; results must agree bit for bit, so a kernel that picks a direction at
run time computes what the unrolled kernels compute. It also checks the esoteric-twist plane map
and the direction numbering against the known answers of the reference's KernelUtilitiesTests.cpp
(getDistributionReferences27 on even and odd steps)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not Path(NVCC).exists(), reason="nvcc not available")
def test_run_time_direction_helpers_equal_compile_time_lattice(tmp_path):
    exe = tmp_path / "lattice_rt_check"
    subprocess.run([NVCC, "-std=c++17", "--expt-relaxed-constexpr", f"-I{ROOT / 'virtualfluids_b200' / 'csrc'}",
                    str(ROOT / "tests" / "lattice_rt_check.cu"), "-o", str(exe)], check=True, timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout
    assert out.stdout.strip() == "ok"
