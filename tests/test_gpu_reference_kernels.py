"""The library's kernels against the reference's own CUDA kernels, run on the same GPU.

oracle/_ref/libvfref_gpu64.so holds the reference's kernels of the hot path (runCollision with
K17, the no-slip / velocity / pressure boundary kernels, initialisation, macroscopic output,
the coarse/fine scaling kernels and the drag/lift kernels), compiled in FP64 without FMA
contraction from the reference tree by oracle/Makefile (target `ref`). Both sides run the same
step sequence on the same device data. Bars: the library's exact arithmetic reproduces the
reference kernels bit for bit; the scaling kernels, whose coefficient sums are formed in another
order, agree to 1e-13 of the largest population.
"""
import ctypes as C

import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import InterpolationCells, ListGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N
from virtualfluids_b200 import scale_coarse_to_fine, scale_fine_to_coarse
from virtualfluids_b200.grid import SIDE_DIR

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(oracle):
    L = oracle.refgpu()
    if L is None:
        pytest.fail("oracle/_ref/libvfref_gpu64.so is missing: run `make -C oracle ref` where the reference tree is")
    assert L.refgpu_real_bytes() == 8
    return L


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


class RefLevel:
    """One level on the device, advanced by the reference's kernels in UpdateGrid27 order."""

    def __init__(self, grid, omega, vkind, nkind, gkind=0, forces=(0.0, 0.0, 0.0), pkind=0, correction=0.0):
        import torch
        dev = torch.device("cuda", 0)
        self.t = torch
        self.g = grid
        self.n = grid.number_of_nodes
        self.omega = float(omega)
        self.dist = torch.zeros(27 * self.n, dtype=torch.float64, device=dev)
        self.nb = [torch.from_numpy(grid.neighbor[a].astype(np.int32)).to(dev) for a in range(3)]
        self.geo = torch.from_numpy(grid.geo.astype(np.int32)).to(dev)
        self.fluid = torch.from_numpy(grid.fluid.astype(np.int32)).to(dev)
        self.forces = torch.tensor(forces, dtype=torch.float64, device=dev)
        self.lim = torch.full((3,), 0.01, dtype=torch.float64, device=dev)
        self.is_even = 1
        self.bcs = {}
        for kind in ("velocity", "noslip", "geometry"):
            m = grid.merged(kind)
            if m is None:
                continue
            k, q, vel = m
            self.bcs[kind] = (torch.from_numpy(k.astype(np.int32)).to(dev), torch.from_numpy(q.reshape(-1).copy()).to(dev),
                              [torch.from_numpy(vel[a].copy()).to(dev) for a in range(3)], k.size)
        self.pressure = []
        for b in grid.bcs:
            if b.kind == "pressure":
                self.pressure.append((torch.from_numpy(b.k.astype(np.int32)).to(dev),
                                      torch.from_numpy(b.k_neighbor.astype(np.int32)).to(dev),
                                      torch.full((b.k.size,), float(b.rho), dtype=torch.float64, device=dev),
                                      b.k.size, SIDE_DIR[b.side]))
        self.vkind, self.nkind, self.gkind, self.pkind, self.correction = vkind, nkind, gkind, pkind, correction

    def init(self, ref, rho=None, ux=None, uy=None, uz=None):
        z = np.zeros(self.n)
        arrs = [self.t.from_numpy(np.ascontiguousarray(a if a is not None else z, dtype=np.float64)).cuda()
                for a in (rho, ux, uy, uz)]
        nb = [_p(x) for x in self.nb]
        for ev in (0, 1):
            assert ref.refgpu_init(*nb, _p(self.geo), *(_p(a) for a in arrs), self.n, _p(self.dist), ev) == 0
        self.is_even = 1

    def _noslip(self, ref, bc, kind):
        k, q, _, nbc = bc
        nb = [_p(x) for x in self.nb]
        if kind == 1:
            assert ref.refgpu_noslip_bounce_back(_p(self.dist), _p(k), _p(q), nbc, *nb, self.n, self.is_even) == 0
        elif kind == 2:
            assert ref.refgpu_noslip_interpolated(_p(self.dist), _p(k), _p(q), nbc, self.omega, *nb, self.n,
                                                  self.is_even) == 0
        elif kind == 3:
            assert ref.refgpu_noslip_interpolated_incompressible(_p(self.dist), _p(k), _p(q), nbc, self.omega, *nb,
                                                                 self.n, self.is_even) == 0

    def step(self, ref, drag=None):
        nb = [_p(x) for x in self.nb]
        assert ref.refgpu_k17(_p(self.dist), self.n, *nb, _p(self.fluid), self.fluid.numel(), self.is_even, self.omega,
                              _p(self.forces), _p(self.lim), 1.0) == 0
        if "velocity" in self.bcs:
            k, q, v, nbc = self.bcs["velocity"]
            if self.vkind == 1:
                assert ref.refgpu_velocity_bounce_back(*(_p(a) for a in v), _p(self.dist), _p(k), _p(q), nbc, *nb,
                                                       self.n, self.is_even) == 0
            else:
                fn = {2: ref.refgpu_velocity_interpolated, 3: ref.refgpu_velocity_interpolated_incompressible,
                      4: ref.refgpu_velocity_with_pressure}[self.vkind]
                assert fn(*(_p(a) for a in v), _p(self.dist), _p(k), _p(q), nbc, self.omega, *nb, self.n,
                          self.is_even) == 0
        if "noslip" in self.bcs:
            self._noslip(ref, self.bcs["noslip"], self.nkind)
        if "geometry" in self.bcs:
            k, q, _, nbc = self.bcs["geometry"]
            if drag is not None:
                assert ref.refgpu_drag_lift_post(_p(self.dist), _p(k), _p(q), nbc, *(_p(a) for a in drag[3:]), *nb,
                                                 self.n, self.is_even) == 0
            self._noslip(ref, self.bcs["geometry"], self.gkind)
        self.is_even = 1 - self.is_even
        if "geometry" in self.bcs and drag is not None:
            k, q, _, nbc = self.bcs["geometry"]
            assert ref.refgpu_drag_lift_pre(_p(self.dist), _p(k), _p(q), nbc, *(_p(a) for a in drag[:3]), *nb,
                                            self.n, self.is_even) == 0
        for k, kn, rho, nbc, direction in self.pressure:
            if self.pkind == 0:
                assert ref.refgpu_pressure_neq(_p(rho), _p(self.dist), _p(k), _p(kn), nbc, *nb, self.n,
                                               self.is_even, direction) == 0
            elif self.pkind == 1:
                assert ref.refgpu_pressure_neq_incompressible(_p(rho), _p(self.dist), _p(k), _p(kn), nbc, *nb,
                                                              self.n, self.is_even, direction) == 0
            else:
                assert ref.refgpu_outflow(_p(rho), _p(self.dist), _p(k), _p(kn), nbc, self.omega, *nb, self.n,
                                          self.is_even, direction, int(self.pkind == 3), self.correction) == 0


def _para(omega, forcing=(0.0, 0.0, 0.0)):
    p = Parameter()
    p.set_viscosity_lb((1.0 / omega - 0.5) / 3.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage, p.arith = N.STORAGE_F64, N.ARITH_EXACT
    p.set_forcing(*forcing)
    return p


def _fields(g, seed, amp_rho=1e-2, amp_u=0.03):
    rng = np.random.default_rng(seed)
    x, y, z = (g.coords[a].astype(np.float64) for a in range(3))
    out = []
    for amp in (amp_rho, amp_u, amp_u, amp_u):
        k = rng.integers(1, 3, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        f = amp * np.cos(2 * np.pi * k[0] * x / g.nx + ph[0]) * np.cos(2 * np.pi * k[1] * y / g.ny + ph[1]) \
            * np.cos(2 * np.pi * k[2] * z / g.nz + ph[2])
        f[0] = 0.0
        out.append(f)
    return out


def _both(ref, grid, bcf, omega, steps, vkind=1, nkind=1, gkind=0, fields=None, forcing=(0.0, 0.0, 0.0)):
    import torch
    sim = Simulation(_para(omega, forcing), grid, bcf)
    rl = RefLevel(grid, sim.para.omega, vkind, nkind, gkind, forces=forcing)
    fields = fields or [None] * 4
    sim.init(*fields)
    rl.init(ref, *fields)
    torch.cuda.synchronize()
    assert np.array_equal(sim.populations(), rl.dist.cpu().numpy())  # InitNavierStokesCompressible_Device
    for _ in range(steps):
        rl.step(ref)
    sim.run(steps)
    torch.cuda.synchronize()
    return sim, rl


def test_periodic_with_forcing_matches_reference_gpu_kernels_bitwise(ref, cuda):
    g = ListGrid(12, 10, 8, periodic=(True, True, True))
    sim, rl = _both(ref, g, BCF(), 1.8, 20, fields=_fields(g, 1), forcing=(1e-5, -2e-6, 3e-6))
    assert np.array_equal(sim.populations(), rl.dist.cpu().numpy())


def test_cavity_bounce_back_matches_reference_gpu_kernels_bitwise(ref, cuda):
    g = ListGrid(12, 12, 12)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim, rl = _both(ref, g, bcf, 1.7, 100)
    assert np.array_equal(sim.populations(), rl.dist.cpu().numpy())


def test_lid_driven_cavity_64_2000_steps_matches_reference_gpu_kernels_bitwise(ref, cuda):
    """The 64^3 lid-driven cavity (lid 0.05, Re = 100, FP64, 2000 steps) through the reference's own
    kernels and through the library: identical populations, hence identical fields and mass."""
    n = 64
    omega = 1.0 / (3.0 * (0.05 * n / 100.0) + 0.5)
    g = ListGrid(n, n, n)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim, rl = _both(ref, g, bcf, omega, 2000)
    assert np.array_equal(sim.populations(), rl.dist.cpu().numpy())


def test_interpolated_bcs_pressure_outlet_and_obstacle_match_reference_gpu_kernels_bitwise(ref, cuda):
    g = ListGrid(24, 12, 12, periodic=(False, True, False))
    g.add_side("MZ", "noslip")
    g.add_side("PZ", "noslip")
    g.add_side("MX", "velocity", velocity=(0.02, 0.0, 0.0))
    g.add_side("PX", "pressure", rho=0.001)
    g.add_box_obstacle((7.3, 3.6, -0.5), (11.6, 7.8, 4.4))
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    bcf.set_pressure_boundary_condition(BCF.PressureBC.PressureNonEquilibriumCompressible)
    bcf.set_geometry_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    sim, rl = _both(ref, g, bcf, 1.8, 80, vkind=2, nkind=2, gkind=2)
    assert np.array_equal(sim.populations(), rl.dist.cpu().numpy())


def test_macroscopic_output_matches_reference_gpu_kernel_bitwise(ref, cuda):
    import torch
    g = ListGrid(12, 10, 8, periodic=(True, True, True))
    sim, rl = _both(ref, g, BCF(), 1.8, 7, fields=_fields(g, 4))
    m = sim.macroscopic()
    out = [torch.zeros(g.number_of_nodes, dtype=torch.float64, device="cuda") for _ in range(5)]
    nb = [_p(x) for x in rl.nb]
    assert ref.refgpu_macros(_p(out[1]), _p(out[2]), _p(out[3]), _p(out[0]), _p(out[4]), _p(rl.geo), *nb, rl.n,
                             _p(rl.dist), rl.is_even) == 0
    torch.cuda.synchronize()
    for i, key in enumerate(("rho", "vx", "vy", "vz", "pressure")):
        assert np.array_equal(m[key], out[i].cpu().numpy()), key


def test_drag_lift_matches_reference_gpu_kernels_bitwise(ref, cuda):
    """DragLiftPost27 / DragLiftPre27 per node, on the state of a running channel with an obstacle."""
    import torch
    g = ListGrid(24, 12, 12, periodic=(False, True, False))
    g.add_side("MZ", "noslip")
    g.add_side("PZ", "noslip")
    g.add_side("MX", "velocity", velocity=(0.02, 0.0, 0.0))
    g.add_side("PX", "pressure", rho=0.0)
    bc = g.add_box_obstacle((7.3, 3.6, -0.5), (11.6, 7.8, 4.4))
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    bcf.set_pressure_boundary_condition(BCF.PressureBC.PressureNonEquilibriumCompressible)
    bcf.set_geometry_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    sim, rl = _both(ref, g, bcf, 1.8, 30, vkind=2, nkind=2, gkind=2)
    ng = bc.k.size
    ref_drag = [torch.zeros(ng, dtype=torch.float64, device="cuda") for _ in range(6)]
    rl.step(ref, drag=ref_drag)                       # step 31 on the reference side, with drag
    mine = [torch.zeros(ng, dtype=torch.float64, device="cuda") for _ in range(6)]
    gb = sim._bcs["geometry"]
    L = sim.level
    # the same step on the library side, by its entry points: collision, BCs, drag post, swap, drag pre
    N.check(N.lib().vfb_k17_run_on_indices(C.byref(L), _p(sim.fluid), int(g.fluid.size), 0, None))
    for kind, fn in (("velocity", "vfb_velocity_interpolated_compressible"),
                     ("noslip", "vfb_noslip_interpolated_compressible")):
        N.check(getattr(N.lib(), fn)(C.byref(L), C.byref(sim._bcs[kind]), None))
    N.check(N.lib().vfb_drag_lift_post_27(C.byref(L), C.byref(gb), *(_p(a) for a in mine[3:]), None))
    N.check(N.lib().vfb_noslip_interpolated_compressible(C.byref(L), C.byref(gb), None))
    L.is_even_timestep = 1 - L.is_even_timestep
    N.check(N.lib().vfb_drag_lift_pre_27(C.byref(L), C.byref(gb), *(_p(a) for a in mine[:3]), None))
    torch.cuda.synchronize()
    for a, b in zip(mine, ref_drag):
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())
    assert np.abs(ref_drag[0].cpu().numpy()).max() > 0
    # calcDragLift: the node-ordered host sum of the reference against the library's device sum
    want = [float(np.sum(ref_drag[c].cpu().numpy() - ref_drag[3 + c].cpu().numpy())) for c in range(3)]
    nbytes = N.lib().vfb_drag_lift_workspace_bytes(ng)
    ws = torch.zeros((nbytes + 7) // 8, dtype=torch.float64, device="cuda")
    force = (C.c_double * 3)()
    N.check(N.lib().vfb_drag_lift_force(*(_p(a) for a in mine), ng, _p(ws), nbytes, force, None))
    seq = np.zeros(3)
    pre = [a.cpu().numpy() for a in ref_drag]
    for i in range(ng):
        for c in range(3):
            seq[c] += pre[c][i] - pre[3 + c][i]
    for c in range(3):
        assert abs(force[c] - seq[c]) <= 1e-13 * np.abs(pre[c] - pre[3 + c]).sum()
        assert abs(want[c] - seq[c]) <= 1e-13 * np.abs(pre[c] - pre[3 + c]).sum()


@pytest.mark.parametrize("fine_to_coarse", [False, True], ids=["coarse_to_fine", "fine_to_coarse"])
def test_scaling_matches_reference_gpu_kernels(ref, cuda, fine_to_coarse):
    import torch
    from test_gpu_refinement import _cells, _level

    gc, coarse = _level(8, 1.65, N.STORAGE_F64, N.ARITH_EXACT, 3, 3)
    gf, fine = _level(12, 1.8, N.STORAGE_F64, N.ARITH_EXACT, 2, 4)
    n_cells = 180
    fine_cells, coarse_cells, off = _cells(gc, gf, n_cells, 5, fine_disjoint=not fine_to_coarse,
                                           coarse_disjoint=fine_to_coarse, offsets=True)
    dc = coarse.dist.clone()
    df = fine.dist.clone()
    cells = InterpolationCells(fine_cells, coarse_cells, off)
    (scale_fine_to_coarse if fine_to_coarse else scale_coarse_to_fine)(coarse, fine, cells)
    fn = ref.refgpu_scale_fc if fine_to_coarse else ref.refgpu_scale_cf
    assert fn(_p(dc), _p(df), *(_p(x) for x in coarse.nb), *(_p(x) for x in fine.nb), gc.number_of_nodes,
              gf.number_of_nodes, coarse.level.is_even_timestep, _p(cells.coarse), _p(cells.fine), n_cells,
              coarse.para.omega, fine.para.omega, *(_p(o) for o in cells.offsets)) == 0
    torch.cuda.synchronize()
    got = (coarse if fine_to_coarse else fine).populations()
    want = (dc if fine_to_coarse else df).cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("vkind,nkind,pkind", [(3, 3, 1), (4, 2, 2), (2, 2, 3), (4, 3, 3)],
                         ids=["incompressible", "with_pressure_outflow", "outflow_correction", "mixed"])
def test_remaining_bc_variants_match_reference_gpu_kernels_bitwise(ref, cuda, vkind, nkind, pkind):
    """VelocityInterpolatedIncompressible / VelocityWithPressureInterpolatedCompressible,
    NoSlipInterpolatedIncompressible, PressureNonEquilibriumIncompressible, OutflowNonReflecting and
    OutflowNonReflectingPressureCorrection through the factory, against the reference's kernels."""
    import torch
    g = ListGrid(20, 10, 10, periodic=(False, True, False))
    g.add_side("MZ", "noslip")
    g.add_side("PZ", "noslip")
    g.add_side("MX", "velocity", velocity=(0.02, 0.0, 0.0))
    g.add_side("PX", "pressure", rho=0.001)
    bcf = BCF()
    bcf.set_velocity_boundary_condition({2: BCF.VelocityBC.VelocityInterpolatedCompressible,
                                         3: BCF.VelocityBC.VelocityInterpolatedIncompressible,
                                         4: BCF.VelocityBC.VelocityWithPressureInterpolatedCompressible}[vkind])
    bcf.set_no_slip_boundary_condition({2: BCF.NoSlipBC.NoSlipInterpolatedCompressible,
                                        3: BCF.NoSlipBC.NoSlipInterpolatedIncompressible}[nkind])
    bcf.set_pressure_boundary_condition({1: BCF.PressureBC.PressureNonEquilibriumIncompressible,
                                         2: BCF.PressureBC.OutflowNonReflective,
                                         3: BCF.PressureBC.OutflowNonReflectivePressureCorrection}[pkind])
    para = _para(1.8)
    para.set_outflow_pressure_correction_factor(0.5)
    sim = Simulation(para, g, bcf)
    rl = RefLevel(g, sim.para.omega, vkind, nkind, pkind=pkind, correction=0.5)
    sim.init()
    rl.init(ref)
    for _ in range(40):
        rl.step(ref)
    sim.run(40)
    torch.cuda.synchronize()
    assert np.array_equal(sim.populations(), rl.dist.cpu().numpy())
    assert np.abs(sim.macroscopic()["vx"]).max() > 1e-3
