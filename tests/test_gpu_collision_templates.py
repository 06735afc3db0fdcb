"""The four non-default CollisionTemplates of vfb_k17_run_on_indices against the reference's own
runCollision kernel and against the oracle.

K17CompressibleNavierStokes<None>::runOnIndices (K17CompressibleNavierStokes.cu:114-139) picks
runCollision<.., writeMacroscopicVariables, applyBodyForce> by template: WriteMacroVars <true, false>,
ApplyBodyForce <false, true>, AllFeatures and SubDomainBorder <true, true>. The body-force variant
adds the node's body force to the global forcing before the half-force scaling and resets it to
zero (RunCollision.cuh:88-98); the macroscopic variant writes drho and u (:133-138). Each template
runs once on the same device state through the library (exact arithmetic) and through the
reference's kernel (oracle/_ref/libvfref_gpu64.so and libvfref_gpu32.so, built without FMA
contraction); populations, macroscopic arrays and body-force arrays must agree bit for bit. In
FP64 the oracle's restatement (orc_collision_template) must agree too.
"""
import ctypes as C

import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import ListGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu

TEMPLATES = {1: (True, False), 2: (False, True), 3: (True, True), 4: (True, True)}


def _p(t):
    return C.c_void_p(t.data_ptr())


def _smooth(g, seed):
    rng = np.random.default_rng(seed)
    x, y, z = (g.coords[a].astype(np.float64) for a in range(3))
    out = []
    for amp in (1e-2, 0.03, 0.03, 0.03):
        k = rng.integers(1, 3, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        f = amp * np.cos(2 * np.pi * k[0] * x / g.nx + ph[0]) * np.cos(2 * np.pi * k[1] * y / g.ny + ph[1]) \
            * np.cos(2 * np.pi * k[2] * z / g.nz + ph[2])
        f[0] = 0.0
        out.append(f)
    return out


@pytest.mark.parametrize("real_bytes", [8, 4], ids=["f64", "f32"])
@pytest.mark.parametrize("tmpl", [1, 2, 3, 4])
def test_collision_template_matches_reference_kernel_and_oracle(oracle, cuda, tmpl, real_bytes):
    import torch
    ref = oracle.refgpu(real_bytes)
    if ref is None:
        pytest.fail("oracle/_ref/libvfref_gpu{64,32}.so is missing: run `make -C oracle ref` where the reference is")
    assert ref.refgpu_real_bytes() == real_bytes
    dt = torch.float64 if real_bytes == 8 else torch.float32
    write_macro, body_force = TEMPLATES[tmpl]

    g = ListGrid(12, 10, 8, periodic=(True, True, True))
    p = Parameter()
    p.set_viscosity_lb((1.0 / 1.8 - 0.5) / 3.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage = N.STORAGE_F64 if real_bytes == 8 else N.STORAGE_F32
    p.arith = N.ARITH_EXACT
    sim = Simulation(p, g, BCF())
    sim.init(*_smooth(g, 11))
    sim.run(3)
    torch.cuda.synchronize()
    n = g.number_of_nodes
    pops0 = sim.populations().copy()

    forces = (2e-6, -1e-6, 5e-7)
    level = 1                                            # forceFactor 2^-1
    rng = np.random.default_rng(100 + tmpl)
    bf0 = [rng.uniform(-1e-5, 1e-5, n) for _ in range(3)]
    sentinel = 7.0

    def arrays():
        macro = [torch.full((n,), sentinel, dtype=dt, device="cuda") for _ in range(4)]
        bf = [torch.from_numpy(b).to("cuda", dt) for b in bf0]
        return macro, bf

    # the library: vfb_k17_run_on_indices with the template
    mine_macro, mine_bf = arrays()
    L = type(sim.level).from_buffer_copy(sim.level)
    L.level = level
    L.forces[0], L.forces[1], L.forces[2] = forces
    L.rho, L.velocity_x, L.velocity_y, L.velocity_z = (t.data_ptr() for t in mine_macro)
    L.body_force_x, L.body_force_y, L.body_force_z = (t.data_ptr() for t in mine_bf)
    is_even = int(L.is_even_timestep)
    N.check(N.lib().vfb_k17_run_on_indices(C.byref(L), _p(sim.fluid), int(g.fluid.size), tmpl, None))
    torch.cuda.synchronize()
    mine_pops = sim.populations()

    # the reference's runCollision on a copy of the same state
    ref_macro, ref_bf = arrays()
    dist = torch.from_numpy(pops0).to("cuda", dt)   # populations() returns the stored values as float64
    nb = [torch.from_numpy(g.neighbor[a].astype(np.int32)).to("cuda") for a in range(3)]
    fluid = torch.from_numpy(g.fluid.astype(np.int32)).to("cuda")
    fdev = torch.tensor(forces, dtype=dt, device="cuda")
    lim = torch.full((3,), 0.01, dtype=dt, device="cuda")
    assert ref.refgpu_k17_template(_p(dist), n, *(_p(x) for x in nb), _p(fluid), int(g.fluid.size), is_even,
                                   float(sim.para.omega), _p(fdev), _p(lim), 0.5,
                                   *(_p(t) for t in ref_macro), *(_p(t) for t in ref_bf), tmpl) == 0
    torch.cuda.synchronize()
    assert np.array_equal(mine_pops, dist.cpu().numpy())
    for a, b in zip(mine_macro + mine_bf, ref_macro + ref_bf):
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())

    fl = g.fluid
    got_bf = [t.cpu().numpy() for t in mine_bf]
    got_macro = [t.cpu().numpy() for t in mine_macro]
    if body_force:
        assert all(np.all(b[fl] == 0.0) for b in got_bf)       # reset after use
        other = np.setdiff1d(np.arange(n), fl)
        assert all(np.array_equal(b[other], b0.astype(b.dtype)[other]) for b, b0 in zip(got_bf, bf0))
    else:
        assert all(np.array_equal(b, b0.astype(b.dtype)) for b, b0 in zip(got_bf, bf0))
    if write_macro:
        assert all(np.all(m[fl] != sentinel) for m in got_macro)
    else:
        assert all(np.all(m == sentinel) for m in got_macro)

    if real_bytes == 8:
        # the oracle's restatement, sequential on the host
        orc = oracle.OracleLevel(g, omega=sim.para.omega)
        orc.f[:] = pops0
        om = [np.full(n, sentinel) for _ in range(4)]
        ob = [b.copy() for b in bf0]
        lim_h, forces_h = np.full(3, 0.01), np.array(forces)   # held while the call reads them
        oracle.lib().orc_collision_template(C.byref(orc.L), oracle.ptr(orc.fluid), int(g.fluid.size), is_even,
                                            float(sim.para.omega), oracle.ptr(lim_h), oracle.ptr(forces_h), level,
                                            int(write_macro), int(body_force), *(oracle.ptr(a) for a in om + ob))
        assert np.array_equal(orc.f, mine_pops)
        for a, b in zip(om + ob, got_macro + got_bf):
            assert np.array_equal(a, b)


def test_collision_template_without_arrays_is_rejected(cuda):
    """The macroscopic and body-force templates need their arrays (the reference dereferences them)."""
    g = ListGrid(6, 6, 6, periodic=(True, True, True))
    p = Parameter()
    p.set_viscosity_lb(0.01)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    sim = Simulation(p, g, BCF())
    sim.init()
    L = type(sim.level).from_buffer_copy(sim.level)
    L.body_force_x = L.body_force_y = L.body_force_z = None
    for tmpl in (2, 3, 4):
        assert N.lib().vfb_k17_run_on_indices(C.byref(L), _p(sim.fluid), int(g.fluid.size), tmpl,
                                              None) == N.VFB_ERR_INVALID_ARGUMENT
    L.rho = None
    assert N.lib().vfb_k17_run_on_indices(C.byref(L), _p(sim.fluid), int(g.fluid.size), 1,
                                          None) == N.VFB_ERR_INVALID_ARGUMENT
    assert N.lib().vfb_k17_run_on_indices(C.byref(L), _p(sim.fluid), int(g.fluid.size), 5,
                                          None) == N.VFB_ERR_INVALID_ARGUMENT
