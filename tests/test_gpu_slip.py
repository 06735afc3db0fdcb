"""The slip BC on the GPU (vfb_slip_compressible; the driver's slip list; slip as the geometry BC)
against the reference's own SlipCompressible_Device (oracle/_ref/libvfref_gpu64.so and
libvfref_gpu32.so, built without FMA contraction) stepped with the reference's runCollision<K17>,
and against the oracle: exact arithmetic bit for bit in FP64 and FP32."""
import ctypes as C

import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import ListGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu

STEPS = 25


def _fields(g, seed):
    rng = np.random.default_rng(seed)
    x, y, z = (g.coords[a].astype(np.float64) for a in range(3))
    out = []
    for amp, base in ((1e-2, 0.0), (0.02, 0.04), (0.02, 0.0), (0.02, 0.01)):
        ph = rng.uniform(0, 2 * np.pi, 3)
        f = base + amp * np.cos(2 * np.pi * x / g.nx + ph[0]) * np.cos(2 * np.pi * y / g.ny + ph[1]) \
            * np.cos(2 * np.pi * z / g.nz + ph[2])
        f[0] = 0.0
        out.append(f)
    return out


def _grid(geometry=False):
    g = ListGrid(14, 10, 9, periodic=(True, False, True))
    if geometry:
        for side in ("MY", "PY"):
            g.add_side(side, "noslip")
        g.add_box_obstacle((4.4, 3.4, 2.4), (8.6, 6.6, 5.6))
    else:
        g.add_side("MY", "slip")
        g.add_side("PY", "slip")
    return g


def _sim(g, storage, geometry=False):
    p = Parameter()
    p.set_viscosity_lb((1.0 / 1.8 - 0.5) / 3.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage, p.arith = storage, N.ARITH_EXACT
    bcf = BCF()
    if geometry:
        bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
        bcf.set_geometry_boundary_condition(BCF.SlipBC.SlipCompressible)
    else:
        bcf.set_slip_boundary_condition(BCF.SlipBC.SlipCompressible)
    sim = Simulation(p, g, bcf)
    sim.init(*_fields(g, 5))
    return sim


def _p(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("real_bytes", [8, 4], ids=["f64", "f32"])
def test_slip_walls_match_reference_kernels_bitwise(cuda, oracle, real_bytes):
    import torch
    ref = oracle.refgpu(real_bytes)
    if ref is None:
        pytest.fail("oracle/_ref/libvfref_gpu*.so is missing: run `make -C oracle ref` where the reference tree is")
    g = _grid()
    storage = N.STORAGE_F64 if real_bytes == 8 else N.STORAGE_F32
    sim = _sim(g, storage)
    omega = float(sim.levels[0].level.omega)
    dt = torch.float64 if real_bytes == 8 else torch.float32
    real = C.c_double if real_bytes == 8 else C.c_float
    dev = torch.device("cuda", 0)
    n = g.number_of_nodes
    dist = torch.from_numpy(sim.populations()).to(dev).to(dt)        # the same initial state
    nb = [torch.from_numpy(g.neighbor[a].astype(np.int32)).to(dev) for a in range(3)]
    fluid = torch.from_numpy(g.fluid.astype(np.int32)).to(dev)
    k, q, _ = g.merged("slip")
    kd = torch.from_numpy(k.astype(np.int32)).to(dev)
    qd = torch.from_numpy(q.reshape(-1).copy()).to(dev).to(dt)
    forces = torch.zeros(3, dtype=dt, device=dev)
    lim = torch.full((3,), 0.01, dtype=dt, device=dev)
    even = 1
    for _ in range(STEPS):
        assert ref.refgpu_k17(_p(dist), C.c_uint64(n), *(_p(x) for x in nb), _p(fluid), C.c_uint(fluid.numel()),
                              C.c_int(even), real(omega), _p(forces), _p(lim), real(1.0)) == 0
        assert ref.refgpu_slip(_p(dist), _p(kd), _p(qd), C.c_uint(k.size), real(omega), *(_p(x) for x in nb),
                               C.c_uint64(n), C.c_int(even)) == 0
        even = 1 - even
    sim.run(STEPS)
    torch.cuda.synchronize()
    assert np.array_equal(sim.populations(), dist.double().cpu().numpy())
    sim.close()


@pytest.mark.parametrize("geometry", [False, True], ids=["slip-list", "geometry-slip"])
def test_slip_matches_oracle_bitwise(cuda, oracle, geometry):
    g = _grid(geometry)
    sim = _sim(g, N.STORAGE_F64, geometry)
    omega = float(sim.levels[0].level.omega)
    lv = oracle.OracleLevel(g, omega)
    lv.init(*_fields(g, 5))
    assert np.array_equal(sim.populations(), lv.f)
    lib, ptr = oracle.lib(), oracle.ptr
    lists = []
    if geometry:
        k, q, _ = g.merged("noslip")
        lists.append(("noslip", np.ascontiguousarray(k.astype(np.int32)), np.ascontiguousarray(q.reshape(-1))))
    kind = "geometry" if geometry else "slip"
    k, q, _ = g.merged(kind)
    lists.append(("slip", np.ascontiguousarray(k.astype(np.int32)), np.ascontiguousarray(q.reshape(-1))))
    for _ in range(STEPS):
        lib.orc_collision(C.byref(lv.L), ptr(lv.fluid), lv.fluid.size, lv.is_even.value, omega, ptr(lv.lim),
                          ptr(lv.forces), 0, None, None, None, None, 0)
        for name, kk, qq in lists:          # no-slip list, then the geometry list (UpdateGrid27 order)
            if name == "noslip":
                lib.orc_bc_noslip_interpolated(C.byref(lv.L), ptr(kk), ptr(qq), kk.size, lv.is_even.value, omega)
            else:
                lib.orc_bc_slip(C.byref(lv.L), ptr(kk), ptr(qq), kk.size, lv.is_even.value, omega)
        lv.is_even.value = 1 - lv.is_even.value
    sim.run(STEPS)
    assert np.array_equal(sim.populations(), lv.f)
    sim.close()


def test_slip_factory_values(cuda):
    fn = C.c_void_p()
    N.check(N.lib().vfb_bc_factory_slip(N.SLIP_COMPRESSIBLE, C.byref(fn)))
    assert fn.value
    N.check(N.lib().vfb_bc_factory_slip(N.SLIP_NOT_SPECIFIED, C.byref(fn)))
    assert not fn.value
    assert N.lib().vfb_bc_factory_slip(N.SLIP_TURBULENT_VISCOSITY_COMPRESSIBLE, C.byref(fn)) == N.VFB_ERR_UNSUPPORTED


@pytest.mark.parametrize("storage", [N.STORAGE_F64, N.STORAGE_F32], ids=["f64", "f32"])
def test_box_slip_walls_match_the_driver_bitwise(cuda, storage):
    """The structured box's slip list (vfb_box_set_bc with VFB_BOX_BC_SLIP) computes the bits of the
    driver's slip list on the same grid."""
    from virtualfluids_b200 import Box
    g = _grid()
    sim = _sim(g, storage)
    bcf = BCF()
    bcf.set_slip_boundary_condition(BCF.SlipBC.SlipCompressible)
    box = Box.from_grid(g, float(sim.levels[0].level.omega), bcf, storage="f64" if storage == N.STORAGE_F64 else "f32",
                        arith="exact")
    Dx, Dy, Dz = g.dims
    f0 = g.first_node
    fields = _fields(g, 5)
    box.init(*(np.ascontiguousarray(a[f0:f0 + Dx * Dy * Dz]) for a in fields))
    sim.run(STEPS)
    box.step(STEPS)
    got = box.fields()
    want = sim.macroscopic()
    for key in ("rho", "vx", "vy", "vz"):
        a = np.asarray(got[key]).reshape(-1)[g.fluid - f0]
        b = np.asarray(want[key]).reshape(-1)[g.fluid]
        assert np.array_equal(a, b), key
    sim.close()


def test_velocity_geometry_bc_matches_oracle_bitwise(cuda, oracle):
    """setGeometryBoundaryCondition with a VelocityBC value: the geometry list runs the interpolated
    velocity kernel with the list's own wall velocities (here a moving obstacle)."""
    g = ListGrid(14, 10, 9, periodic=(True, False, True))
    for side in ("MY", "PY"):
        g.add_side(side, "noslip")
    g.add_box_obstacle((4.4, 3.4, 2.4), (8.6, 6.6, 5.6))
    for b in g.bcs:                                 # the obstacle moves along x
        if b.kind == "geometry":
            b.velocity = (0.01, 0.0, 0.0)
    p = Parameter()
    p.set_viscosity_lb((1.0 / 1.8 - 0.5) / 3.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage, p.arith = N.STORAGE_F64, N.ARITH_EXACT
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    bcf.set_geometry_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    sim = Simulation(p, g, bcf)
    sim.init(*_fields(g, 5))
    omega = float(sim.levels[0].level.omega)
    lv = oracle.OracleLevel(g, omega)
    lv.init(*_fields(g, 5))
    lib, ptr = oracle.lib(), oracle.ptr
    kn, qn, _ = g.merged("noslip")
    kn, qn = np.ascontiguousarray(kn.astype(np.int32)), np.ascontiguousarray(qn.reshape(-1))
    kg, qg, vg = g.merged("geometry")
    kg, qg = np.ascontiguousarray(kg.astype(np.int32)), np.ascontiguousarray(qg.reshape(-1))
    vg = [np.ascontiguousarray(vg[a], dtype=np.float64) for a in range(3)]
    assert np.all(vg[0] == 0.01)
    for _ in range(STEPS):
        lib.orc_collision(C.byref(lv.L), ptr(lv.fluid), lv.fluid.size, lv.is_even.value, omega, ptr(lv.lim),
                          ptr(lv.forces), 0, None, None, None, None, 0)
        lib.orc_bc_noslip_interpolated(C.byref(lv.L), ptr(kn), ptr(qn), kn.size, lv.is_even.value, omega)
        lib.orc_bc_velocity_interpolated(C.byref(lv.L), ptr(kg), ptr(qg), kg.size, lv.is_even.value, omega,
                                         *(ptr(a) for a in vg))
        lv.is_even.value = 1 - lv.is_even.value
    sim.run(STEPS)
    assert np.array_equal(sim.populations(), lv.f)
    assert np.abs(sim.macroscopic()["vx"]).max() > 1e-4          # the moving obstacle drives the flow
    sim.close()
