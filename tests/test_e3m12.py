"""The E3M12 storage format (1 sign, 3 exponent, 12 significand bits for (f - w)/w; csrc/storage.cuh
Codec<e3m12_t>, virtualfluids_b200/formats.py).

CPU: the device codec compiled for the host (tests/e3m12_check.cu: exhaustive round trip, order,
unbiased stochastic rounding, saturation) and the numpy restatement of formats.py over every bit
pattern. GPU: a TGV run in E3M12 storage lands several times closer to FP64 than the same run in
IEEE half, a pool domain computes the same bits as the same box alone, and the step driver's list
path runs the format and decodes its populations on the host."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from virtualfluids_b200 import _native as N
from virtualfluids_b200.formats import MAX, decode, encode

ROOT = Path(__file__).resolve().parent.parent
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not Path(NVCC).exists(), reason="nvcc not available")
def test_device_codec_on_the_host(tmp_path):
    exe = tmp_path / "e3m12_check"
    subprocess.run([NVCC, "-std=c++17", "-O2", "--expt-relaxed-constexpr", f"-I{ROOT / 'virtualfluids_b200' / 'csrc'}",
                    str(ROOT / "tests" / "e3m12_check.cu"), "-o", str(exe)], check=True, timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout
    assert out.stdout.strip().endswith("ok")


def test_numpy_restatement_over_every_pattern():
    h = np.arange(65536, dtype=np.uint32).astype(np.uint16)
    g = decode(h)
    assert np.array_equal(encode(g.astype(np.float32)), h)
    assert np.array_equal(encode(g.astype(np.float32), 2047), h)
    assert g[0x7FFF] == MAX and g[1] == 2.0 ** -18 and g[0x1000] == 2.0 ** -6
    assert np.all(np.diff(g[:0x8000]) > 0)
    assert np.array_equal(encode(np.array([3.0, -3.0, np.inf], dtype=np.float32)), [0x7FFF, 0xFFFF, 0x7FFF])
    # 4x finer than IEEE half near the populations' typical magnitude 0.1: 2^-16 against 2^-14
    assert decode(encode(np.float32(0.1) + np.float32(2.0 ** -16))) - decode(encode(np.float32(0.1))) == 2.0 ** -16


def _tgv(n, u0=0.04):
    x = (np.arange(n) + 0.5) / n * 2 * np.pi - np.pi
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    rho = 3.0 * (u0 * u0 / 16.0) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    return [a.reshape(-1) for a in (rho, u0 * np.sin(X) * np.cos(Y) * np.cos(Z),
                                    -u0 * np.cos(X) * np.sin(Y) * np.cos(Z), np.zeros_like(X))]


def _l2(a, b):
    num = sum(np.sum((a[k].astype(np.float64) - b[k]) ** 2) for k in ("vx", "vy", "vz"))
    return np.sqrt(num / sum(np.sum(b[k] ** 2) for k in ("vx", "vy", "vz")))


@pytest.mark.gpu
def test_tgv_closer_to_fp64_than_half(cuda):
    """TGV 64^3, u0 = 0.04, Re 1600, 500 steps: relative L2 velocity error against FP64."""
    from virtualfluids_b200 import Box
    n, steps = 64, 500
    omega = 1.0 / (3 * 0.04 * n / (2 * np.pi * 1600) + 0.5)
    f = _tgv(n)
    ref = Box(n, n, n, omega, storage="f64")
    ref.init(*f)
    ref.step(steps)
    r = ref.fields()
    err = {}
    for st in ("f16", "e3m12"):
        b = Box(n, n, n, omega, storage=st)
        b.init(*(a.astype(np.float32) for a in f))
        b.step(steps)
        err[st] = _l2(b.fields(), r)
    print("relative L2 velocity error vs FP64:", err)
    assert err["e3m12"] < err["f16"] / 2.5
    assert err["e3m12"] < 6e-4


@pytest.mark.gpu
def test_list_path_runs_e3m12_and_decodes(cuda):
    """The drop-in step driver on a lid-driven cavity in E3M12: populations decoded on the host match
    the structured box of the same level within the storage rounding, after a few steps, and the
    cavity's flow follows the FP64 run."""
    from virtualfluids_b200 import BoundaryConditionFactory, ListGrid, Parameter, Simulation
    g = ListGrid(16, 16, 16)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    out = {}
    for st in (N.STORAGE_F64, N.STORAGE_E3M12):
        p = Parameter()
        p.set_viscosity_lb(0.05 * 16 / 100.0)
        p.configure_main_kernel("K17CompressibleNavierStokes")
        p.storage = st
        bcf = BoundaryConditionFactory()
        bcf.set_no_slip_boundary_condition(bcf.NoSlipBC.NoSlipBounceBack)
        bcf.set_velocity_boundary_condition(bcf.VelocityBC.VelocityBounceBack)
        sim = Simulation(p, g, bcf, device=cuda)
        sim.init()
        sim.run(200)
        out[st] = sim.macroscopic()
        if st == N.STORAGE_E3M12:
            pops = sim.populations()
            assert pops.dtype == np.float64 and np.isfinite(pops).all() and np.abs(pops).max() < MAX
        sim.close()
    fl = g.geo == N.GEO_FLUID
    a, b = out[N.STORAGE_E3M12], out[N.STORAGE_F64]
    scale = np.abs(b["vx"][fl]).max()
    assert np.abs(a["vx"][fl] - b["vx"][fl]).max() < 2e-3 * scale
