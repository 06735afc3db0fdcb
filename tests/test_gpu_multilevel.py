"""The multi-level step driver (UpdateGrid27::updateGrid's recursion with Refinement_noExchange) on
the GPU, through the C ABI, against the oracle's multi-level driver on the same nested grids.

Exact arithmetic reproduces the oracle bit for bit on every level (periodic boxes, a cavity whose
walls and lid stay on the coarse level, three nested levels, a body force scaled by 2^-level);
FMA arithmetic stays within 1e-12 relative L-inf; the shear wave decays at the analytic rate on
both levels of a refined box.
"""
import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import GridScalingFactory, ListGrid, MultiLevelGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-12


def _para(nu, arith, storage=N.STORAGE_F64, forcing=(0.0, 0.0, 0.0)):
    p = Parameter()
    p.set_viscosity_lb(nu)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage, p.arith = storage, arith
    p.set_forcing(*forcing)
    return p


def _scaling():
    s = GridScalingFactory()
    s.set_scaling_factory(GridScalingFactory.GridScaling.ScaleCompressible)
    return s


def _fields(mgrid, level, seed, n_coarse, amp_rho=5e-3, amp_u=0.02):
    """Smooth seeded fields of the coarse box's periodic modes, sampled at the level's node positions."""
    rng = np.random.default_rng(seed)
    pos = mgrid.positions(level)
    out = []
    for amp in (amp_rho, amp_u, amp_u, amp_u):
        k = rng.integers(1, 3, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        f = amp * np.cos(2 * np.pi * k[0] * pos[0] / n_coarse + ph[0]) * np.cos(2 * np.pi * k[1] * pos[1] / n_coarse
                                                                               + ph[1]) \
            * np.cos(2 * np.pi * k[2] * pos[2] / n_coarse + ph[2])
        f[0] = 0.0
        out.append(f)
    return out


def _run_both(oracle, mgrid, nu, steps, arith, bcf=None, forcing=(0.0, 0.0, 0.0), vkind=1, nkind=1, seed=11,
              n_coarse=None):
    bcf = bcf or BCF()
    sim = Simulation(_para(nu, arith, forcing=forcing), mgrid, bcf, _scaling())
    orc = oracle.OracleMultiLevel(mgrid, nu, forces=forcing, velocity_kind=vkind, noslip_kind=nkind)
    n_coarse = n_coarse or mgrid.levels[0].nx
    for level in range(len(mgrid.levels)):
        f = _fields(mgrid, level, seed + level, n_coarse)
        sim.init(*f, level=level)
        orc.init(level, *f)
    sim.run(steps)
    orc.run(steps)
    return sim, orc


def _periodic(n, lo, hi, levels=2):
    m = MultiLevelGrid.uniform(ListGrid(n, n, n, periodic=(True, True, True)))
    for _ in range(levels - 1):
        m.refine(lo, hi)
    return m


@pytest.mark.parametrize("steps", [1, 4], ids=["one_step", "four_steps"])
def test_two_levels_exact_is_bitwise(oracle, cuda, steps):
    m = _periodic(16, (4, 4, 4), (12, 12, 12))
    sim, orc = _run_both(oracle, m, 0.01, steps, N.ARITH_EXACT)
    for level in range(2):
        assert np.array_equal(sim.populations(level), orc.levels[level].f), f"level {level}"
        assert sim.levels[level].level.is_even_timestep == orc.levels[level].is_even.value


def test_two_levels_with_force_exact_is_bitwise(oracle, cuda):
    m = _periodic(16, (3, 5, 4), (11, 12, 13))
    sim, orc = _run_both(oracle, m, 0.012, 3, N.ARITH_EXACT, forcing=(2e-5, -1e-5, 3e-6))
    for level in range(2):
        assert np.array_equal(sim.populations(level), orc.levels[level].f), f"level {level}"


def test_three_levels_exact_is_bitwise(oracle, cuda):
    m = _periodic(14, (3, 3, 3), (11, 11, 11), levels=3)
    assert [g.nx for g in m.levels] == [14, 16, 16]
    sim, orc = _run_both(oracle, m, 0.004, 2, N.ARITH_EXACT)
    for level in range(3):
        assert np.array_equal(sim.populations(level), orc.levels[level].f), f"level {level}"


@pytest.mark.parametrize("interpolated", [False, True], ids=["bounce_back", "interpolated"])
def test_refined_cavity_exact_is_bitwise(oracle, cuda, interpolated):
    """A lid-driven cavity whose centre is refined: walls and lid on the coarse level only."""
    g = ListGrid(18, 18, 18)
    for side in ("MX", "PX", "MY", "PY", "MZ"):
        g.add_side(side, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    m = MultiLevelGrid.uniform(g)
    m.refine((5, 5, 4), (13, 13, 12))
    bcf = BCF()
    if interpolated:
        bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
        bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    else:
        bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
        bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
    kind = 2 if interpolated else 1
    sim = Simulation(_para(0.01, N.ARITH_EXACT), m, bcf, _scaling())
    orc = oracle.OracleMultiLevel(m, 0.01, velocity_kind=kind, noslip_kind=kind)
    for level in range(2):
        sim.init(level=level)
        orc.init(level)
    sim.run(6)
    orc.run(6)
    for level in range(2):
        assert np.array_equal(sim.populations(level), orc.levels[level].f), f"level {level}"
    assert np.abs(sim.macroscopic(1)["vx"]).max() > 0.0     # the lid's flow has reached the fine level


def test_two_levels_fma_within_tolerance(oracle, cuda):
    m = _periodic(16, (4, 4, 4), (12, 12, 12))
    sim, orc = _run_both(oracle, m, 0.01, 10, N.ARITH_FAST)
    for level in range(2):
        got, want = sim.macroscopic(level), orc.levels[level].macroscopic()
        f = m.levels[level].fluid
        for key in ("rho", "vx", "vy", "vz"):
            scale = max(np.abs(want[key][f]).max(), 1e-300)
            assert np.abs(got[key][f] - want[key][f]).max() / scale < FAST_TOL, (level, key)


def test_refined_shear_wave_decays_at_the_analytic_rate(cuda):
    """u_x = U sin(k z) on a periodic 32^3 box refined over its centre half: after 200 coarse steps
    the amplitude on both levels is within 0.4 % of U exp(-nu k^2 t) (the uniform box: 0.32 %), and
    the flow stays a sine wave to 0.5 % of U."""
    n, U, nu, steps = 32, 0.02, 0.01, 200
    k = 2 * np.pi / n
    m = _periodic(n, (8, 8, 8), (24, 24, 24))
    sim = Simulation(_para(nu, N.ARITH_FAST), m, BCF(), _scaling())
    for level in range(2):
        z = m.positions(level)[2]
        sim.init(None, U * np.sin(k * (z + 0.5)), None, None, level=level)
    sim.run(steps)
    want = U * np.exp(-nu * k * k * steps)
    for level in range(2):
        f = m.levels[level].fluid
        s = np.sin(k * (m.positions(level)[2][f] + 0.5))
        ux = sim.macroscopic(level)["vx"][f]
        amp = (ux * s).sum() / (s * s).sum()
        assert abs(amp / want - 1.0) < 4e-3, (level, amp / want - 1.0)
        assert np.abs(ux - amp * s).max() < 5e-3 * U, level


def test_missing_scaling_factory_is_an_error(cuda):
    m = _periodic(16, (4, 4, 4), (12, 12, 12))
    with pytest.raises(N.VfbError) as e:
        Simulation(_para(0.01, N.ARITH_FAST), m, BCF())
    assert e.value.status == N.VFB_ERR_SCALING_UNSET
