"""Generate the golden vectors of tests/golden/ from the reference's own arithmetic.

Runs the reference's K17, chimera, macroscopic and interpolation headers, compiled for the host from the
reference tree by oracle/Makefile (target `ref`), on seeded random inputs and stores inputs
and outputs. The committed .npz files let the oracle be pinned on machines that do not have
the reference tree. Usage:

    make -C oracle ref REF=<reference checkout>
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import pyoracle  # noqa: E402

W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
SEED = 20261203


def _cases(rng, n):
    """Populations near equilibrium at lattice Mach numbers up to ~0.1, and far from it."""
    out = []
    for i in range(n):
        rho = rng.uniform(-0.05, 0.05)
        u = rng.uniform(-0.1, 0.1, 3)
        cx = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
        cy = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1])
        cz = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1])
        cu = cx * u[0] + cy * u[1] + cz * u[2]
        feq = W * (rho + (1 + rho) * (3 * cu + 4.5 * cu * cu - 1.5 * (u @ u)))
        noise = rng.normal(0, 1e-3 if i % 3 else 2e-2, 27) * W
        out.append(feq + noise)
    return np.array(out)


def main():
    r64, r32 = pyoracle.ref64(), pyoracle.ref32()
    if r64 is None or r32 is None:
        raise SystemExit("reference pins missing: run `make -C oracle ref` first")
    rng = np.random.default_rng(SEED)
    n = 256
    f_in = _cases(rng, n)
    omega = rng.uniform(0.6, 1.99, n)
    lim = np.where(rng.random((n, 3)) < 0.5, 0.01, rng.uniform(1e-4, 1e-1, (n, 3)))
    force = np.where(rng.random((n, 1)) < 0.5, 0.0, rng.normal(0, 1e-5, (n, 3)))
    out64 = np.zeros((n, 27))
    mac64 = np.zeros((n, 4))
    out32 = np.zeros((n, 27), dtype=np.float32)
    mac32 = np.zeros((n, 4), dtype=np.float32)
    for i in range(n):
        a = f_in[i].copy()
        m = np.zeros(4)
        r64.ref_k17_f64(pyoracle.ptr(a), omega[i], pyoracle.ptr(lim[i].copy()), *force[i], pyoracle.ptr(m))
        out64[i], mac64[i] = a, m
        a = f_in[i].astype(np.float32)
        m = np.zeros(4, dtype=np.float32)
        r32.ref_k17_f32(pyoracle.ptr(a), np.float32(omega[i]), pyoracle.ptr(lim[i].astype(np.float32)),
                        *(np.float32(x) for x in force[i]), pyoracle.ptr(m))
        out32[i], mac32[i] = a, m
    np.savez_compressed(ROOT / "tests/golden/k17_reference.npz", f_in=f_in, omega=omega, lim=lim, force=force,
                        out64=out64, mac64=mac64, out32=out32, mac32=mac32)

    # chimera transforms: which in 0..3, (a, b, c, v, v2, kinv, k) -> (a, b, c)
    m = 128
    chim_in = rng.normal(0, 1, (m, 3))
    v = rng.uniform(-0.2, 0.2, m)
    kin = rng.choice([1.0, 3.0, 9.0, 36.0, 1.5, 4.5, 6.0, 18.0, 2.25], m)
    chim_out = np.zeros((4, m, 3))
    for which in range(4):
        for i in range(m):
            abc = chim_in[i].copy()
            r64.ref_chimera_f64(which, pyoracle.ptr(abc), v[i], v[i] * v[i], kin[i], 1.0 / kin[i])
            chim_out[which, i] = abc
    dens = np.array([r64.ref_density_f64(pyoracle.ptr(f.copy())) for f in f_in])
    macro = np.zeros((n, 4))
    for i in range(n):
        r64.ref_macro_compressible_f64(pyoracle.ptr(f_in[i].copy()), pyoracle.ptr(macro[i]))
    np.savez_compressed(ROOT / "tests/golden/chimera_macro_reference.npz", chim_in=chim_in, v=v, kinv=kin,
                        chim_out=chim_out, f_in=f_in, density=dens, macro=macro)

    # refinement interpolation: eight source nodes of a cell in the reference's visiting order
    # MMM, MMP, PMP, PMM, MPM, MPP, PPP, PPM; coefficients, coarse-to-fine populations of the eight
    # fine nodes at (+-1/4)^3 (oracle corner order c = ix + 2 iy + 4 iz) and the fine-to-coarse ones
    nc = 96
    f8 = np.zeros((nc, 8, 27))
    for i in range(nc):
        f8[i] = _cases(rng, 8) * (1.0 if i % 4 else 3.0)
    om = rng.uniform(1.2, 1.95, (nc, 2))
    offs = np.zeros((nc, 3))
    offs[1::3] = rng.choice([-0.5, 0.0, 0.5], (len(offs[1::3]), 3))
    offs[2::3] = rng.uniform(-0.5, 0.5, (len(offs[2::3]), 3))
    coef = np.zeros((nc, 46))
    cf = np.zeros((nc, 8, 27))
    fc = np.zeros((nc, 27))
    for i in range(nc):
        src = np.ascontiguousarray(f8[i][pyoracle.REF_CORNER_ORDER])
        r64.ref_interp_coefficients_f64(pyoracle.ptr(src), om[i, 0], *offs[i], pyoracle.ptr(coef[i]))
        for c in range(8):
            pos = [0.25 if (c >> a) & 1 else -0.25 for a in range(3)]
            r64.ref_interp_cf_f64(pyoracle.ptr(src), om[i, 0], om[i, 1], *offs[i], *pos, pyoracle.ptr(cf[i, c]))
        r64.ref_interp_fc_f64(pyoracle.ptr(src), om[i, 1], om[i, 0], *offs[i], pyoracle.ptr(fc[i]))
    np.savez_compressed(ROOT / "tests/golden/interpolation_reference.npz", f8=f8, omega=om, offset=offs,
                        coef=coef, cf=cf, fc=fc)
    print("wrote", ROOT / "tests/golden")


if __name__ == "__main__":
    main()
