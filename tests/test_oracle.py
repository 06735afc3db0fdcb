"""The oracle, pinned against the reference's own tests and golden vectors (CPU only)."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _chim(oracle, which, abc, v, v2, kinv, k):
    a = np.array(abc, dtype=np.float64)
    oracle.lib().orc_chimera_f64(which, oracle.ptr(a), v, v2, kinv, k)
    return a


# tests/unit-tests/lbm/ChimeraTests.cpp known answers
def test_chimera_known_answers(oracle):
    assert np.array_equal(_chim(oracle, 0, [1, 1, 1], 1.0, 1.0, 1.0, 1.0), [3.0, -4.0, 6.0])
    assert np.array_equal(_chim(oracle, 1, [3, -4, 6], 1.0, 1.0, 1.0, 1.0), [1.0, 1.0, 1.0])
    assert np.array_equal(_chim(oracle, 2, [1, 1, 1], 1.0, 1.0, 0, 0), [3.0, -3.0, 5.0])
    assert np.array_equal(_chim(oracle, 3, [3, -3, 5], 1.0, 1.0, 0, 0), [1.0, 1.0, 1.0])


# tests/unit-tests/lbm/MacroscopicQuantitiesTests.cpp known answers
def test_macroscopic_known_answers(oracle):
    L = oracle.lib()
    f = np.ones(27)
    assert L.orc_density_f64(oracle.ptr(f)) == 27.0
    out = [C.c_double() for _ in range(5)]
    L.orc_macro_compressible_f64(oracle.ptr(f), *(C.byref(o) for o in out))
    assert out[2].value == 0.0 and out[3].value == 0.0 and out[4].value == 0.0
    f[1] = 2.0  # dP00
    L.orc_macro_compressible_f64(oracle.ptr(f), *(C.byref(o) for o in out))
    assert out[0].value == 28.0
    assert out[2].value == pytest.approx(1.0 / 29.0, rel=1e-15)


def test_chimera_and_macros_match_reference_golden(oracle):
    g = np.load(GOLDEN / "chimera_macro_reference.npz")
    for which in range(4):
        for i in range(g["chim_in"].shape[0]):
            v, kinv = g["v"][i], g["kinv"][i]
            got = _chim(oracle, which, g["chim_in"][i], v, v * v, kinv, 1.0 / kinv)
            assert np.array_equal(got, g["chim_out"][which, i]), (which, i)
    L = oracle.lib()
    for i, f in enumerate(g["f_in"]):
        f = np.ascontiguousarray(f)
        assert L.orc_density_f64(oracle.ptr(f)) == g["density"][i]
        out = [C.c_double() for _ in range(5)]
        L.orc_macro_compressible_f64(oracle.ptr(f), *(C.byref(o) for o in out))
        assert [out[0].value, out[2].value, out[3].value, out[4].value] == list(g["macro"][i])


def test_k17_matches_reference_golden_bitwise(oracle):
    """K17CompressibleNavierStokes.h:88 run by the reference header on the host vs the oracle."""
    g = np.load(GOLDEN / "k17_reference.npz")
    for i in range(g["f_in"].shape[0]):
        out, mac = oracle.k17(g["f_in"][i], g["omega"][i], tuple(g["lim"][i]), tuple(g["force"][i]))
        assert np.array_equal(out, g["out64"][i]), i
        assert np.array_equal(mac, g["mac64"][i]), i
        out, mac = oracle.k17(g["f_in"][i], g["omega"][i], tuple(g["lim"][i]), tuple(g["force"][i]), dtype=np.float32)
        assert np.array_equal(out, g["out32"][i]), i
        assert np.array_equal(mac, g["mac32"][i]), i


def test_k17_matches_reference_header_live(oracle):
    """Same pin against the freshly built reference header, when the pins are present."""
    r64 = oracle.ref64()
    if r64 is None:
        pytest.skip("reference pins not built here (golden vectors cover this)")
    rng = np.random.default_rng(7)
    W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
    for i in range(2000):
        f = rng.normal(0, 5e-3, 27) * W
        om = rng.uniform(0.5, 1.99)
        a, ma = oracle.k17(f, om)
        b = f.copy()
        mb = np.zeros(4)
        r64.ref_k17_f64(oracle.ptr(b), om, oracle.ptr(np.full(3, 0.01)), 0.0, 0.0, 0.0, oracle.ptr(mb))
        assert np.array_equal(a, b) and np.array_equal(ma, mb)


def test_rest_state_is_a_fixed_point(oracle):
    out, mac = oracle.k17(np.zeros(27), 1.7)
    assert np.all(out == 0.0) and np.all(mac == 0.0)


def _ldc_grid(n, interpolated=False):
    from virtualfluids_b200.grid import ListGrid
    g = ListGrid(n, n, n)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    return g


def test_oracle_init_roundtrip_and_macros(oracle):
    """init writes the equilibrium of (rho, u); the macroscopic output reads (rho, u) back."""
    from virtualfluids_b200.grid import ListGrid
    g = ListGrid(6, 5, 4, periodic=(True, True, True))
    rng = np.random.default_rng(3)
    n = g.number_of_nodes
    rho, ux, uy, uz = (rng.uniform(-0.02, 0.02, n) for _ in range(4))
    lv = oracle.OracleLevel(g, omega=1.5)
    lv.init(rho, ux, uy, uz)
    m = lv.macroscopic()
    fl = g.fluid
    np.testing.assert_allclose(m["rho"][fl], rho[fl], rtol=0, atol=1e-15)
    np.testing.assert_allclose(m["vx"][fl], ux[fl], rtol=0, atol=1e-15)
    np.testing.assert_allclose(m["vz"][fl], uz[fl], rtol=0, atol=1e-15)


def smooth_fields(g, rng, amp_rho=1e-2, amp_u=0.03, modes=3):
    """Seeded smooth periodic fields: a few low Fourier modes per component."""
    x, y, z = (g.coords[a].astype(np.float64) for a in range(3))
    out = []
    for amp in (amp_rho, amp_u, amp_u, amp_u):
        f = np.zeros(g.number_of_nodes)
        for _ in range(modes):
            k = rng.integers(0, 2, 3) + np.array([1, 0, 0])
            ph = rng.uniform(0, 2 * np.pi, 3)
            f += np.cos(2 * np.pi * k[0] * x / g.nx + ph[0]) * np.cos(2 * np.pi * k[1] * y / g.ny + ph[1]) \
                * np.cos(2 * np.pi * k[2] * z / g.nz + ph[2])
        f *= amp / modes
        f[0] = 0.0
        out.append(f)
    return out


def test_oracle_periodic_mass_conservation(oracle):
    from virtualfluids_b200.grid import ListGrid
    g = ListGrid(8, 8, 8, periodic=(True, True, True))
    rng = np.random.default_rng(4)
    # omega = 1.8 (nu = 0.0185 < 1/42): K17's modified 4th-order equilibrium is linearly unstable for
    # large viscosities, which is why Parameter.cpp:424-445 warns above nu = 1/42
    lv = oracle.OracleLevel(g, omega=1.8)
    lv.init(*smooth_fields(g, rng))
    m0, e0 = lv.mass_energy()
    lv.run(50)
    m1, e1 = lv.mass_energy()
    assert abs(m1 - m0) < 1e-11 * m0
    assert e1 < e0  # viscous decay


def test_oracle_cavity_bounce_back_conserves_mass(oracle):
    g = _ldc_grid(8)
    lv = oracle.OracleLevel(g, omega=1.7)
    lv.init()
    m0, _ = lv.mass_energy()
    lv.run(100)
    m1, e1 = lv.mass_energy()
    assert abs(m1 - m0) < 1e-10 * m0   # velocity bounce-back with a tangential lid injects no mass
    assert e1 > 0.0                     # the lid drives the flow


def test_cpu_baseline_step_equals_oracle_step_bitwise(oracle):
    """The timed CPU baseline advances a level with the reference header's collision sweep (the
    parity build and the Release-flag build) and the oracle's boundary conditions; both give the
    oracle's own time step bit for bit, on a cavity with bounce-back and with interpolated BCs."""
    builds = [b for b in (oracle.ref64(), oracle.ref64_release()) if b is not None]
    if not builds:
        pytest.skip("reference pins not built here")
    for kind in (1, 2):
        g = _ldc_grid(10)
        want = oracle.OracleLevel(g, omega=1.7, velocity_kind=kind, noslip_kind=kind)
        want.init()
        want.run(25)
        for ref in builds:
            got = oracle.OracleLevel(g, omega=1.7, velocity_kind=kind, noslip_kind=kind)
            got.init()
            got.run_reference_collision(ref, 25, threads=2)
            assert got.is_even.value == want.is_even.value
            assert np.array_equal(got.f, want.f)


# refinement interpolation (InterpolationCoefficients.h, InterpolationCF.h, InterpolationFC.h).
# The oracle forms the same polynomial with its sums in another order, so the pin is a tolerance:
# per cell, the largest deviation relative to the largest population.
INTERP_TOL = 1e-13


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def test_interpolation_matches_reference_golden(oracle):
    g = np.load(GOLDEN / "interpolation_reference.npz")
    for i in range(g["f8"].shape[0]):
        f8, (oc, of), off = g["f8"][i], g["omega"][i], tuple(g["offset"][i])
        coef = oracle.interp_coefficients(f8, oc, off)
        ref = g["coef"][i][:42]
        assert np.abs(coef - ref).max() <= INTERP_TOL * np.abs(ref).max(), i
        assert _rel(oracle.interp_cf_cell(f8, oc, of, off), g["cf"][i]) <= INTERP_TOL, i
        assert _rel(oracle.interp_fc_cell(f8, of, oc, off), g["fc"][i]) <= INTERP_TOL, i


def test_interpolation_matches_reference_header_live(oracle):
    r64 = oracle.ref64()
    if r64 is None:
        pytest.skip("reference pins not built here (golden vectors cover this)")
    rng = np.random.default_rng(11)
    W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
    for i in range(300):
        f8 = rng.normal(0, 1e-2, (8, 27)) * W + rng.normal(0, 1e-2, (8, 1)) * W
        oc, of = rng.uniform(1.0, 1.99, 2)
        off = (0.0, 0.0, 0.0) if i % 2 else tuple(rng.uniform(-0.5, 0.5, 3))
        src = np.ascontiguousarray(f8[oracle.REF_CORNER_ORDER])
        mine = oracle.interp_cf_cell(f8, oc, of, off)
        for c in range(8):
            pos = [0.25 if (c >> a) & 1 else -0.25 for a in range(3)]
            out = np.zeros(27)
            r64.ref_interp_cf_f64(oracle.ptr(src), oc, of, *off, *pos, oracle.ptr(out))
            assert _rel(mine[c], out) <= INTERP_TOL, (i, c)
        out = np.zeros(27)
        r64.ref_interp_fc_f64(oracle.ptr(src), of, oc, *off, oracle.ptr(out))
        assert _rel(oracle.interp_fc_cell(f8, of, oc, off), out) <= INTERP_TOL, i


def test_interpolation_of_a_uniform_state_is_that_state(oracle):
    """A cell whose eight corners hold one resting state gives that state back on both sides
    (the strain rate is zero, so only the equilibrium survives)."""
    W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
    f8 = np.zeros((8, 27))
    assert np.abs(oracle.interp_cf_cell(f8, 1.7, 1.8)).max() == 0.0
    assert np.abs(oracle.interp_fc_cell(f8, 1.8, 1.7)).max() == 0.0
    rho = 0.01
    f8 = np.tile(W * rho, (8, 1))
    out = oracle.interp_cf_cell(f8, 1.7, 1.8)
    for c in range(8):
        assert np.allclose(out[c], W * rho, rtol=0, atol=1e-16)
    assert np.allclose(oracle.interp_fc_cell(f8, 1.8, 1.7), W * rho, rtol=0, atol=1e-16)
