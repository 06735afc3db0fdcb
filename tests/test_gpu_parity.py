"""Parity of the CUDA path (through the C ABI) with the oracle, on the GPU.

Tolerances: the exact arithmetic variant (no FMA contraction) must reproduce the oracle bit for
bit; the default variant (FMA) must stay within 1e-12 relative L-inf in density and velocity
(relative to the field's maximum magnitude), the bar of the FP64 form.
"""
import ctypes as C

import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import ListGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-12


def smooth_fields(g, seed, amp_rho=1e-2, amp_u=0.03, modes=3):
    rng = np.random.default_rng(seed)
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


def make_para(omega, storage=N.STORAGE_F64, arith=N.ARITH_FAST, forcing=(0.0, 0.0, 0.0)):
    p = Parameter()
    p.set_viscosity_lb((1.0 / omega - 0.5) / 3.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage, p.arith = storage, arith
    p.set_forcing(*forcing)
    return p


def rel_linf(a, b, mask):
    scale = max(np.abs(b[mask]).max(), 1e-300)
    return np.abs(a[mask] - b[mask]).max() / scale


def run_both(oracle, grid, omega, steps, arith, bcf=None, fields=None, forcing=(0.0, 0.0, 0.0), vkind=1, nkind=1,
             threads=0):
    bcf = bcf or BCF()
    sim = Simulation(make_para(omega, N.STORAGE_F64, arith, forcing), grid, bcf)
    orc = oracle.OracleLevel(grid, omega=sim.para.omega, forces=forcing, velocity_kind=vkind, noslip_kind=nkind)
    fields = fields or [None] * 4
    sim.init(*fields)
    orc.init(*fields)
    sim.run(steps)
    orc.run(steps, threads=threads)
    return sim, orc


def cavity(n, velocity=(0.05, 0.0, 0.0)):
    g = ListGrid(n, n, n)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=velocity)
    return g


def test_periodic_exact_is_bitwise(oracle, cuda):
    g = ListGrid(12, 10, 8, periodic=(True, True, True))
    sim, orc = run_both(oracle, g, 1.8, 20, N.ARITH_EXACT, fields=smooth_fields(g, 1))
    assert np.array_equal(sim.populations(), orc.f)


def test_periodic_fast_within_tolerance(oracle, cuda):
    g = ListGrid(12, 10, 8, periodic=(True, True, True))
    sim, orc = run_both(oracle, g, 1.8, 20, N.ARITH_FAST, fields=smooth_fields(g, 1))
    a, b = sim.macroscopic(), orc.macroscopic()
    fl = g.geo == N.GEO_FLUID
    for k in ("rho", "vx", "vy", "vz"):
        assert rel_linf(a[k], b[k], fl) <= FAST_TOL, k


def test_forcing_exact_is_bitwise(oracle, cuda):
    g = ListGrid(10, 8, 6, periodic=(True, True, True))
    sim, orc = run_both(oracle, g, 1.9, 15, N.ARITH_EXACT, fields=smooth_fields(g, 2), forcing=(1e-5, -2e-6, 3e-6))
    assert np.array_equal(sim.populations(), orc.f)


def test_cavity_bounce_back_exact_is_bitwise(oracle, cuda):
    """NoSlipBounceBack + VelocityBounceBack, as apps/gpu/DrivenCavity/DrivenCavity.cpp:145-146."""
    g = cavity(12)
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim, orc = run_both(oracle, g, 1.7, 100, N.ARITH_EXACT, bcf=bcf)
    assert np.array_equal(sim.populations(), orc.f)


def _randomise_q(g, seed):
    rng = np.random.default_rng(seed)
    for b in g.bcs:
        cut = b.q >= 0
        b.q[cut] = rng.uniform(0.05, 0.95, cut.sum())


def test_cavity_interpolated_exact_is_bitwise(oracle, cuda):
    """NoSlipInterpolatedCompressible + VelocityInterpolatedCompressible with q in (0,1)."""
    g = cavity(12)
    _randomise_q(g, 5)
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    sim, orc = run_both(oracle, g, 1.7, 100, N.ARITH_EXACT, bcf=bcf, vkind=2, nkind=2)
    assert np.array_equal(sim.populations(), orc.f)


def test_channel_pressure_outlet_exact_is_bitwise(oracle, cuda):
    """Velocity inlet (interpolated), PressureNonEquilibriumCompressible outlet, no-slip walls."""
    g = ListGrid(16, 8, 8, periodic=(False, True, False))
    g.add_side("MZ", "noslip")
    g.add_side("PZ", "noslip")
    g.add_side("MX", "velocity", velocity=(0.02, 0.0, 0.0))
    g.add_side("PX", "pressure", rho=0.001)
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    bcf.set_pressure_boundary_condition(BCF.PressureBC.PressureNonEquilibriumCompressible)
    sim, orc = run_both(oracle, g, 1.8, 120, N.ARITH_EXACT, bcf=bcf, vkind=2, nkind=2)
    assert np.array_equal(sim.populations(), orc.f)
    m = sim.macroscopic()
    assert np.abs(m["vx"]).max() > 1e-3


def test_mass_energy_and_macros_match_oracle(oracle, cuda):
    g = cavity(10)
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim, orc = run_both(oracle, g, 1.7, 50, N.ARITH_EXACT, bcf=bcf)
    a, b = sim.macroscopic(), orc.macroscopic()
    for k in ("rho", "vx", "vy", "vz", "pressure"):
        assert np.array_equal(a[k], b[k]), k
    (m1, e1), (m2, e2) = sim.mass_energy(), orc.mass_energy()
    assert abs(m1 - m2) <= 1e-13 * m2 and abs(e1 - e2) <= 1e-12 * e2


@pytest.mark.parametrize("arith", [N.ARITH_EXACT, N.ARITH_FAST])
def test_lid_driven_cavity_64_2000_steps(oracle, cuda, arith):
    """The 64^3 lid-driven cavity: lid u=0.05 in +x, Re=100, FP64, 2000 steps, bounce-back walls and lid.

    Exact arithmetic reproduces the oracle bit for bit (so within any tolerance, 1e-12 included).
    With FMA contraction the result differs from the oracle by the amplified rounding: the oracle
    itself built with contraction drifts from the uncontracted oracle by ~1e-8 (relative L-inf of
    the secondary velocity) after 2000 steps on this flow, so the FMA variant is held to 1e-6."""
    n = 64
    nu = 0.05 * n / 100.0
    omega = 1.0 / (3.0 * nu + 0.5)
    g = cavity(n)
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim, orc = run_both(oracle, g, omega, 2000, arith, bcf=bcf)
    a, b = sim.macroscopic(), orc.macroscopic()
    fl = g.geo == N.GEO_FLUID
    errs = {k: rel_linf(a[k], b[k], fl) for k in ("rho", "vx", "vy", "vz")}
    print("64^3 cavity relative L-inf vs oracle:", "exact" if arith == N.ARITH_EXACT else "fma", errs)
    (m1, _), (m2, _) = sim.mass_energy(), orc.mass_energy()
    assert np.abs(b["vx"][fl]).max() > 0.01  # the flow is developed
    if arith == N.ARITH_EXACT:
        assert np.array_equal(sim.populations(), orc.f)
        assert max(errs.values()) == 0.0
        assert abs(m1 - m2) <= 1e-13 * m2
    else:
        assert max(errs.values()) <= 1e-6, errs
        assert abs(m1 - m2) <= 1e-12 * m2


def _cube_channel(n=(24, 12, 12)):
    """Channel with an interpolated velocity inlet, a pressure outlet, no-slip walls in z and a
    box obstacle on the bottom wall whose faces lie between nodes (exact-geometry q)."""
    g = ListGrid(*n, periodic=(False, True, False))
    g.add_side("MZ", "noslip")
    g.add_side("PZ", "noslip")
    g.add_side("MX", "velocity", velocity=(0.02, 0.0, 0.0))
    g.add_side("PX", "pressure", rho=0.0)
    g.add_box_obstacle((7.3, 3.6, -0.5), (11.6, 7.8, 4.4))
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    bcf.set_pressure_boundary_condition(BCF.PressureBC.PressureNonEquilibriumCompressible)
    bcf.set_geometry_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    return g, bcf


@pytest.mark.parametrize("arith", [N.ARITH_EXACT, N.ARITH_FAST])
def test_obstacle_geometry_bc_and_drag_lift(oracle, cuda, arith):
    """Geometry BC (interpolated bounce-back on an obstacle) and the FP64 drag/lift of every step
    (DragLiftPost27 / DragLiftPre27 / calcDragLift). Exact arithmetic gives bit-identical
    populations; the per-step force is an FP64 sum formed in another order on the device, held to
    1e-12 of its magnitude (exact) and to the FMA tolerance of the flow (fast)."""
    g, bcf = _cube_channel()
    steps = 60
    sim = Simulation(make_para(1.8, N.STORAGE_F64, arith), g, bcf)
    orc = oracle.OracleLevel(g, omega=sim.para.omega, velocity_kind=2, noslip_kind=2, geometry_kind=2, drag_lift=True)
    sim.init()
    orc.init()
    sim.enable_drag_lift(history_steps=steps)
    sim.run(steps)
    orc.run(steps)
    got = sim.drag_lift_history()
    want = np.array(orc.drag_history)
    assert got.shape == want.shape == (steps, 3)
    assert want[-1, 0] > 0.0  # drag along the flow
    scale = np.abs(want).max(axis=0)
    if arith == N.ARITH_EXACT:
        assert np.array_equal(sim.populations(), orc.f)
        assert np.all(np.abs(got - want) <= 1e-12 * scale)
    else:
        assert np.all(np.abs(got - want) <= 1e-9 * scale)


def test_sphere_geometry_bc_and_drag_exact_is_bitwise(oracle, cuda):
    """A sphere in a channel with the exact q of Sphere::getIntersection on every cut link, the
    interpolated geometry BC and the FP64 drag of every step: bitwise against the oracle."""
    g = ListGrid(26, 14, 14, periodic=(False, True, True))
    g.add_side("MX", "velocity", velocity=(0.03, 0.0, 0.0))
    g.add_side("PX", "pressure", rho=0.0)
    g.add_sphere_obstacle((9.4, 6.7, 6.2), 3.3)
    bcf = BCF()
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    bcf.set_pressure_boundary_condition(BCF.PressureBC.PressureNonEquilibriumCompressible)
    bcf.set_geometry_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    steps = 40
    sim = Simulation(make_para(1.85, N.STORAGE_F64, N.ARITH_EXACT), g, bcf)
    orc = oracle.OracleLevel(g, omega=sim.para.omega, velocity_kind=2, noslip_kind=2, geometry_kind=2, drag_lift=True)
    sim.init()
    orc.init()
    sim.enable_drag_lift(history_steps=steps)
    sim.run(steps)
    orc.run(steps)
    assert np.array_equal(sim.populations(), orc.f)
    got, want = sim.drag_lift_history(), np.array(orc.drag_history)
    assert want[-1, 0] > 0.0
    assert np.all(np.abs(got - want) <= 1e-12 * np.abs(want).max(axis=0))


def test_drag_lift_history_ring_keeps_the_last_steps(oracle, cuda):
    g, bcf = _cube_channel()
    sim = Simulation(make_para(1.8, N.STORAGE_F64, N.ARITH_EXACT), g, bcf)
    orc = oracle.OracleLevel(g, omega=sim.para.omega, velocity_kind=2, noslip_kind=2, geometry_kind=2, drag_lift=True)
    sim.init()
    orc.init()
    sim.enable_drag_lift(history_steps=7)
    sim.run(10)
    sim.run(5)
    orc.run(15)
    got = sim.drag_lift_history()
    want = np.array(orc.drag_history)[-7:]
    assert np.all(np.abs(got - want) <= 1e-12 * np.abs(want).max(axis=0))


def test_box_with_boundary_conditions_matches_the_list_path(oracle, cuda):
    """Box.from_grid: the same level as a structured box with BC lists in box indices computes the
    list path's fields and drag bit for bit (exact arithmetic)."""
    from virtualfluids_b200 import Box
    g, bcf = _cube_channel()
    steps = 40
    sim = Simulation(make_para(1.8, N.STORAGE_F64, N.ARITH_EXACT), g, bcf)
    sim.init()
    sim.enable_drag_lift(history_steps=steps)
    sim.run(steps)
    box = Box.from_grid(g, sim.para.omega, bcf, storage="f64", arith="exact")
    Dx, Dy, Dz = g.dims
    z = np.zeros(Dx * Dy * Dz)
    box.init(z, z, z, z)
    box.enable_drag_lift(history_steps=steps)
    box.step(steps)
    f = box.fields()
    m = sim.macroscopic()
    fl = g.geo[1:] == N.GEO_FLUID
    for key in ("rho", "vx", "vy", "vz"):
        assert np.array_equal(f[key][fl], m[key][1:][fl]), key
    assert np.array_equal(box.drag_lift_history(), sim.drag_lift_history())


def test_box_inlet_perturbation_is_seeded(cuda):
    from virtualfluids_b200 import Box
    g, bcf = _cube_channel()
    runs = []
    for seed in (7, 7, 8):
        box = Box.from_grid(g, 1.8, bcf, storage="f32")
        Dx, Dy, Dz = g.dims
        z = np.zeros(Dx * Dy * Dz)
        box.init(z, z, z, z)
        box.set_velocity_perturbation(seed, 0.01)
        box.step(30)
        runs.append(box.fields()["vx"])
    assert np.array_equal(runs[0], runs[1])
    assert not np.array_equal(runs[0], runs[2])
    assert np.abs(runs[0] - runs[2]).max() < 1e-3


@pytest.mark.parametrize("storage,arith,align", [(N.STORAGE_F64, N.ARITH_EXACT, 1), (N.STORAGE_F64, N.ARITH_EXACT, 32),
                                                 (N.STORAGE_F32, N.ARITH_EXACT, 1), (N.STORAGE_F64, N.ARITH_FAST, 1),
                                                 (N.STORAGE_F32, N.ARITH_FAST, 32)])
def test_periodic_box_levels_take_box_addressing_with_the_same_bits(cuda, storage, arith, align):
    """An F64 or F32 level whose fluid list is a whole periodic box (reference numbering from node 1,
    or aligned from node 32) is collided by the box kernel over the reference layout: the same bits
    as the neighborX/Y/Z chain, with forcing, in both arithmetics; a level with walls, and a 16-bit
    level, keep the list kernel."""
    g = ListGrid(20, 9, 7, periodic=(True, True, True), align=align)
    out, used = [], []
    for tables in (0, 1):
        p = make_para(1.85, storage, arith, forcing=(2e-6, -1e-6, 5e-7))
        sim = Simulation(p, g, BCF(), neighbor_tables=tables)
        sim.init(*smooth_fields(g, 6))
        sim.run(9)
        out.append(sim.populations())
        flag = C.c_int32()
        N.check(N.lib().vfb_simulation_level_box_addressing(sim._sim, 0, C.byref(flag)))
        used.append(flag.value)
        sim.close()
    assert used == [0, 1]
    assert np.array_equal(out[0], out[1])
    for grid, st in ((ListGrid(12, 10, 9), N.STORAGE_F64), (g, N.STORAGE_F16)):
        sim = Simulation(make_para(1.8, st), grid, BCF())
        flag = C.c_int32()
        N.check(N.lib().vfb_simulation_level_box_addressing(sim._sim, 0, C.byref(flag)))
        assert flag.value == 0
        sim.close()


@pytest.mark.parametrize("storage,dims", [(N.STORAGE_F64, (12, 10, 9)), (N.STORAGE_F16, (12, 10, 9)),
                                          (N.STORAGE_F64, (96, 40, 36)), (N.STORAGE_F32, (90, 37, 33))],
                         ids=["f64", "f16", "f64-loop", "f32-loop"])
def test_neighbor_slot_tables_change_nothing(cuda, storage, dims):
    """The driver's neighbour slot tables, loaded directly or staged by bulk copies, give the same bits
    as the neighborX/Y/Z chain. The larger grids give the staged kernel's persistent warps several
    tiles each."""
    g = ListGrid(*dims)
    for side in ("MX", "PX", "MY", "PY", "MZ"):
        g.add_side(side, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.01, 0.0))
    bcf = BCF()
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    out = []
    for tables in (0, 1, 2):
        sim = Simulation(make_para(1.8, storage), g, bcf, neighbor_tables=tables)
        sim.init(*smooth_fields(g, 5))
        sim.run(7)
        out.append(sim.populations())
        st = C.c_int32()
        N.check(N.lib().vfb_simulation_status(sim._sim, C.byref(st), None))
        assert st.value == 0
        sim.close()
    assert all(np.array_equal(out[0], o) for o in out[1:])


@pytest.mark.parametrize("periodic,storage,arith", [((True, True, True), N.STORAGE_F64, N.ARITH_EXACT),
                                                    ((True, True, True), N.STORAGE_F32, N.ARITH_FAST),
                                                    ((False, True, False), N.STORAGE_F64, N.ARITH_EXACT),
                                                    ((True, True, True), N.STORAGE_F16, N.ARITH_FAST)],
                         ids=["periodic-f64", "periodic-f32-fma", "walls-f64", "periodic-f16"])
def test_k17_plans_match_the_stateless_entry_point(cuda, periodic, storage, arith):
    """vfb_k17_plan_run (the adapter's runOnIndices) against vfb_k17_run_on_indices over the chain:
    the same populations and macroscopic outputs, alternating the Default and WriteMacroVars
    templates, with box addressing exactly for the regular F64/F32 levels."""
    g = ListGrid(20, 9, 7, periodic=periodic)
    lib = N.lib()
    results, flags = [], []
    for use_plan in (False, True):
        sim = Simulation(make_para(1.85, storage, arith, forcing=(1e-6, 0.0, -2e-6)), g, BCF(), neighbor_tables=0)
        sim.init(*smooth_fields(g, 4))
        L = sim.levels[0].level
        fluid, n = C.c_void_p(sim.fluid.data_ptr()), int(g.fluid.size)
        plan = C.c_void_p()
        if use_plan:
            N.check(lib.vfb_k17_plan_create(C.byref(L), fluid, n, C.byref(plan)))
            flag = C.c_int32()
            N.check(lib.vfb_k17_plan_box_addressing(plan, C.byref(flag)))
            flags.append(flag.value)
        for step in range(8):
            tmpl = (N.COLLISION_DEFAULT, N.COLLISION_WRITE_MACRO_VARS)[step % 2]
            if use_plan:
                N.check(lib.vfb_k17_plan_run(plan, C.byref(L), tmpl, None))
            else:
                N.check(lib.vfb_k17_run_on_indices(C.byref(L), fluid, n, tmpl, None))
            L.is_even_timestep = 1 - L.is_even_timestep
        N.check(lib.vfb_synchronize(None))
        S = sim.levels[0]
        results.append([sim.populations()] + [x.double().cpu().numpy() for x in (S.rho, S.vx, S.vy, S.vz)])
        if use_plan:
            N.check(lib.vfb_k17_plan_destroy(plan))
        sim.close()
    regular = all(periodic) and storage in (N.STORAGE_F64, N.STORAGE_F32)
    assert flags == [1 if regular else 0]
    for a, b in zip(*results):
        assert np.array_equal(a, b)


def test_box_addressing_needs_every_neighbour_entry_regular(cuda):
    """One neighbour entry out of the box pattern (still a valid node), or a fluid list with a node
    left out, keeps the list kernel; the untouched grid takes box addressing."""
    def flag_of(grid):
        sim = Simulation(make_para(1.8), grid, BCF())
        f = C.c_int32()
        N.check(N.lib().vfb_simulation_level_box_addressing(sim._sim, 0, C.byref(f)))
        sim.close()
        return f.value

    g = ListGrid(10, 6, 5, periodic=(True, True, True))
    assert flag_of(g) == 1
    k = int(g.fluid[37])
    bad = ListGrid(10, 6, 5, periodic=(True, True, True))
    bad.neighbor[2][k] = bad.neighbor[2][int(bad.fluid[38])]      # a wrong +z neighbour
    assert flag_of(bad) == 0
    short = ListGrid(10, 6, 5, periodic=(True, True, True))
    short.fluid = short.fluid[:-1].copy()                          # the last node left out
    assert flag_of(short) == 0
