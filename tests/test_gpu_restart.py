"""Restart files and field output on the GPU: a run saved at step t and restarted from the file
continues bit for bit as the uninterrupted run (uniform and two-level list levels, structured
boxes in FP64 and FP16 storage); the VTK output holds the macroscopic fields."""
import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import Box, GridScalingFactory, ListGrid, MultiLevelGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N
from virtualfluids_b200.output import read_vtk

pytestmark = pytest.mark.gpu


def _para(nu, storage=N.STORAGE_F64):
    p = Parameter()
    p.set_viscosity_lb(nu)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage = storage
    return p


def _mgrid(levels):
    m = MultiLevelGrid.uniform(ListGrid(16, 16, 16, periodic=(True, True, True)))
    if levels == 2:
        m.refine((4, 4, 4), (12, 12, 12))
    return m


def _make(levels, storage):
    m = _mgrid(levels)
    sf = GridScalingFactory()
    sf.set_scaling_factory(GridScalingFactory.GridScaling.ScaleCompressible)
    sim = Simulation(_para(0.01, storage), m, BCF(), sf)
    return m, sim


@pytest.mark.parametrize("levels", [1, 2])
@pytest.mark.parametrize("storage", [N.STORAGE_F64, N.STORAGE_F16], ids=["f64", "f16"])
def test_simulation_restart_continues_bitwise(cuda, tmp_path, levels, storage):
    m, a = _make(levels, storage)
    for level in range(levels):
        pos = m.positions(level)
        a.init(None, 0.02 * np.sin(2 * np.pi * pos[2] / 16), 0.01 * np.cos(2 * np.pi * pos[0] / 16), None,
               level=level)
    a.run(5)                                   # odd: the coarse level restarts at the odd parity
    a.save_restart(tmp_path / "chk")
    a.run(6)
    _, b = _make(levels, storage)
    b.load_restart(tmp_path / "chk", timestep=5)
    b.run(6)
    for level in range(levels):
        assert np.array_equal(a._raw(level), b._raw(level)), level
    a.write_vtk(tmp_path / "out.vtk", level=levels - 1)
    back = read_vtk(tmp_path / "out.vtk")
    mac = a.macroscopic(levels - 1)
    f = m.levels[levels - 1].fluid
    assert np.array_equal(back["velocity"][0], mac["vx"][f]) and np.array_equal(back["drho"], mac["rho"][f])


@pytest.mark.parametrize("storage", ["f64", "f16"])
def test_box_restart_continues_bitwise(cuda, tmp_path, storage):
    n = 12
    x = np.arange(n ** 3) % n
    a = Box(n, n, n, 1.8, storage=storage)
    a.init(np.zeros(n ** 3), 0.02 * np.sin(2 * np.pi * x / n), np.zeros(n ** 3), np.zeros(n ** 3))
    a.step(7)
    planes, even = a.read_populations()
    assert not even
    a.save_restart(tmp_path / "box")
    a.step(4)
    b = Box(n, n, n, 1.8, storage=storage)
    b.load_restart(tmp_path / "box", is_even=even)
    b.step(4)
    assert np.array_equal(a.read_populations()[0], b.read_populations()[0])
    a.write_vtk(tmp_path / "box.vtk")
    back = read_vtk(tmp_path / "box.vtk")
    assert back["dimensions"] == (n, n, n)
    assert np.array_equal(back["velocity"][0], a.fields()["vx"].astype(np.float64))


def test_simulation_vtu_output_holds_the_oracle_fields(cuda, oracle, tmp_path):
    """Simulation.write_vtu after an exact-arithmetic cavity run: the part file equals the one the
    same writer makes from the oracle's fields of the same run (so the file carries the reference's
    values), and the time series lists both written steps."""
    from virtualfluids_b200.output import FileWriter
    g = ListGrid(10, 10, 10)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    p = _para(0.05 * 10 / 100.0)
    p.arith = N.ARITH_EXACT
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim = Simulation(p, g, bcf)
    sim.init()
    w, first = sim.write_vtu(tmp_path / "sim", 0)
    sim.run(30)
    w, files = sim.write_vtu(tmp_path / "sim", 30, last=True, writer=w)
    orc = oracle.OracleLevel(g, omega=p.omega)
    orc.init()
    orc.run(30)
    m = orc.macroscopic()
    ref = FileWriter(tmp_path / "orc").write_timestep(
        30, [dict(coords=g.coords.astype(np.float64), spacing=1.0, geo=g.geo, neighbor=g.neighbor, **{
            "rho": m["rho"], "vx": m["vx"], "vy": m["vy"], "vz": m["vz"], "pressure": m["pressure"]})])
    from pathlib import Path
    assert Path(files[0]).read_bytes() == Path(ref[0]).read_bytes()
    pvd = Path([f for f in files if f.endswith(".pvd")][0]).read_text()
    assert 'timestep="0"' in pvd and 'timestep="30"' in pvd
