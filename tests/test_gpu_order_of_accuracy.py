"""Order of accuracy of the K17 time step on the reference's numerical test
(tests/numerical-tests/gpu/NumericalTests/configK17chim_nu10tm3.txt, PhiTest and NyTest with
MinOrderOfAccuracy 1.95): the Taylor-Green vortex advected along x (TGV-Ux, the reference's
Simulations/TaylorGreenVortexUx initial condition and analytic solution) on lx x 4 x 1.5 lx nodes for
lx = 32, 64, 128, viscosity 1e-3 in lattice units, diffusive scaling: 1000 (lx/32)^2 steps between
20 outputs and an advection velocity 0.096 * 32/lx, so that the vortex travels exactly three domain
lengths per output. On the y = 0 slice, the (1,1) Fourier mode of v_x (and of v_z) over outputs
11-20 gives the viscosity, from the slope of its log amplitude, and the phase error, from the slope
of its phase (FFTCalculator.cpp: amplitude 4 |F| / (lx lz), phase atan(Im/Re)). The errors
|nu - 1e-3| / 1e-3 and |phase slope| must fall with an order above 1.95 between successive
resolutions. The box runs the exact FP64 form, the reference's own arithmetic.
"""
import numpy as np
import pytest

from virtualfluids_b200 import Box

pytestmark = pytest.mark.gpu

L0, NU, AMP, UX0 = 32, 1e-3, 1e-3, 0.096
MIN_ORDER = 1.95


def _tgv_ux(lx):
    ly, lz = 4, lx * 3 // 2
    z, _, x = np.meshgrid(np.arange(lz), np.arange(ly), np.arange(lx), indexing="ij")
    kx, kz = 2 * np.pi * x / lx, 2 * np.pi * z / lz
    ux = UX0 * L0 / lx + AMP * L0 * np.cos(kz) * np.sin(kx) / lx
    uz = -AMP * L0 * lz * np.cos(kx) * np.sin(kz) / lx ** 2
    press = AMP * L0 ** 2 * (AMP * lz ** 2 * np.cos(kz) ** 2 - 4 * (lx ** 2 - lz ** 2) * UX0 * np.cos(kz) * np.sin(kx)
                             - AMP * lx ** 2 * np.sin(kx) ** 2) / (2 * lx ** 4)
    return (lx, ly, lz), [a.reshape(-1) for a in (3 * press, ux, np.zeros_like(ux), uz)]


def _slope(y):
    x = np.arange(len(y), dtype=np.float64)
    return float(np.sum((x - x.mean()) * (y - np.mean(y))) / np.sum((x - x.mean()) ** 2))


def _nu_and_phase(lx):
    (nx, ny, nz), fields = _tgv_ux(lx)
    steps = 1000 * (lx // L0) ** 2
    box = Box(nx, ny, nz, 1.0 / (3 * NU + 0.5), storage="f64", arith="exact")
    box.init(*fields)
    modes = {"vx": [], "vz": []}
    for out in range(1, 21):
        box.step(steps)
        if out < 11:
            continue
        f = box.fields()
        for key in modes:
            slice_y0 = f[key].reshape(nz, ny, nx)[:, 0, :]
            modes[key].append(np.fft.fft2(slice_y0)[1, 1])
    k2 = (2 * np.pi / nz) ** 2 + (2 * np.pi / nx) ** 2
    out = {}
    for key, m in modes.items():
        m = np.array(m)
        amp = 4.0 / (nx * nz) * np.abs(m)
        nu = -_slope(np.log(amp)) / (k2 * steps)
        phase = np.arctan(m.imag / m.real)
        out[key] = (abs(nu - NU) / NU, abs(_slope(phase)))
    return out


def test_tgv_ux_viscosity_and_phase_converge_at_second_order(cuda):
    res = {lx: _nu_and_phase(lx) for lx in (32, 64, 128)}
    for key in ("vx", "vz"):
        for a, b in ((32, 64), (64, 128)):
            for i, name in ((0, "viscosity"), (1, "phase")):
                ea, eb = res[a][key][i], res[b][key][i]
                order = np.log(ea / eb) / np.log(b / a)
                assert order > MIN_ORDER, (key, name, a, b, ea, eb, order)
