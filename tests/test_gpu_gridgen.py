"""Grids built by the reference's own grid generator (oracle/_ref/libvfref_gridgen.so), imported with
virtualfluids_b200.gridgen and run on the GPU with exact arithmetic, against the oracle on the same
arrays: bit for bit on a cavity, on a channel with a velocity inlet, a pressure outlet and a
sphere (interpolated BCs with the builder's exact q), and on a two-level cavity whose fine box
lies on a wall, so that interpolation cells with non-zero offsets (ICellNeigh) take part."""
import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import GridScalingFactory, Parameter, Simulation
from virtualfluids_b200 import _native as N
from virtualfluids_b200.gridgen import import_levels

pytestmark = pytest.mark.gpu
BOX = (-0.5, -0.5, -0.5, 0.5, 0.5, 0.5)


@pytest.fixture(scope="module")
def ref(oracle):
    if oracle.refgg() is None:
        pytest.fail("oracle/_ref/libvfref_gridgen.so is missing: run `make -C oracle ref` where the reference is")
    return oracle


def _para(nu):
    p = Parameter()
    p.set_viscosity_lb(nu)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.arith = N.ARITH_EXACT
    return p


def test_imported_cavity_bitwise(ref, cuda):
    G = import_levels(*ref.reference_grid(BOX, 1 / 16, noslip=("PX", "MX", "PY", "MY", "MZ"),
                                          velocity=[("PZ", 0.05, 0.0, 0.0)]))
    g = G.levels[0]
    nu = 0.05 * 16 / 100
    bcf = BCF()
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim = Simulation(_para(nu), G, bcf)
    sim.init()
    sim.run(100)
    orc = ref.OracleLevel(g, omega=sim.para.omega, velocity_kind=1)
    orc.init()
    orc.run(100)
    assert np.array_equal(sim.populations(), orc.f)
    assert np.abs(orc.macroscopic()["vx"]).max() > 1e-3


def test_imported_channel_with_sphere_and_pressure_outlet_bitwise(ref, cuda):
    lev, ifs = ref.reference_grid((0.0, 0.0, 0.0, 2.0, 0.5, 0.5), 1 / 16,
                                  geometries=[("sphere", 0.6, 0.25, 0.25, 0.12)], periodic=(False, True, False),
                                  noslip=("MZ", "PZ"), velocity=[("MX", 0.02, 0.0, 0.0)], pressure=[("PX", 0.0)],
                                  geometry_noslip=True)
    G = import_levels(lev, ifs, periodic=(False, True, False))
    g = G.levels[0]
    bcf = BCF()
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    bcf.set_pressure_boundary_condition(BCF.PressureBC.PressureNonEquilibriumCompressible)
    bcf.set_geometry_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    sim = Simulation(_para(0.02), G, bcf)
    sim.init()
    sim.run(60)
    orc = ref.OracleLevel(g, omega=sim.para.omega, velocity_kind=2, geometry_kind=2)
    orc.init()
    orc.run(60)
    assert np.array_equal(sim.populations(), orc.f)
    assert np.abs(orc.macroscopic()["vx"]).max() > 1e-3


def test_imported_two_levels_with_wall_interface_cells_bitwise(ref, cuda):
    lev, ifs = ref.reference_grid(BOX, 1 / 12, refinements=[((-0.5, -0.25, -0.25, 0.0, 0.25, 0.25), 1)],
                                  noslip=("PX", "MX", "PY", "MY", "MZ"), velocity=[("PZ", 0.05, 0.0, 0.0)])
    G = import_levels(lev, ifs)
    assert np.count_nonzero(G.interfaces[0].offsets_cf) > 0
    nu = 0.05 * 12 / 100
    bcf = BCF()
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sf = GridScalingFactory()
    sf.set_scaling_factory(GridScalingFactory.GridScaling.ScaleCompressible)
    sim = Simulation(_para(nu), G, bcf, sf)
    orc = ref.OracleMultiLevel(G, nu)
    for level in range(2):
        sim.init(level=level)
        orc.init(level)
    sim.run(12)
    orc.run(12)
    for level in range(2):
        # every slot but the dummy node 0's: the fine level's missing neighbours all point there,
        # many nodes write its slots in one launch (their order decides the bits) and none reads
        # them as data
        n = G.levels[level].number_of_nodes
        real = np.arange(27 * n) % n != 0
        a, b = sim.populations(level), orc.levels[level].f
        assert np.array_equal(a[real], b[real]), level
    assert np.abs(orc.levels[1].macroscopic()["vx"]).max() > 1e-4
