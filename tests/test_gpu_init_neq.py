"""The non-equilibrium initialisation on the GPU (vfb_init_navier_stokes_compressible_non_equilibrium;
Simulation with Parameter.use_init_neq) against the reference's own kernel,
InitNavierStokesCompressibleNonEquilibrium_Device (InitNavierStokesCompressible_Device.cu:216-501),
from oracle/_ref/libvfref_gpu64.so and libvfref_gpu32.so (built without FMA contraction), and against
the oracle. Bars: exact arithmetic bit for bit in FP64 and FP32, both before and after steps; the
other storage forms within their rounding of the FP64 values."""
import ctypes as C

import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import ListGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu

GRIDS = [((14, 11, 9), (True, True, True)), ((13, 10, 8), (False, True, False))]
W27 = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)


def _smooth(g, seed, amp_rho=1e-2, amp_u=0.03, modes=3):
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
        out.append(f * amp / modes)
    return out


def _p(t):
    return C.c_void_p(t.data_ptr())


def _sim(g, storage, arith, omega, fields):
    p = Parameter()
    p.set_viscosity_lb((1.0 / omega - 0.5) / 3.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage, p.arith = storage, arith
    p.set_use_init_neq(True)
    sim = Simulation(p, g, BCF())
    sim.init(*fields)
    return sim


def _reference(ref, g, fields, omega, double):
    import torch
    dt = torch.float64 if double else torch.float32
    dev = torch.device("cuda", 0)
    n = g.number_of_nodes
    dist = torch.zeros(27 * n, dtype=dt, device=dev)
    nb = [torch.from_numpy(g.neighbor[a].astype(np.int32)).to(dev) for a in range(3)]
    inv = torch.from_numpy(g.neighbor_inverse.astype(np.int32)).to(dev)
    geo = torch.from_numpy(g.geo.astype(np.int32)).to(dev)
    arrs = [torch.from_numpy(np.ascontiguousarray(a)).to(dev).to(dt) for a in fields]
    om = C.c_double(omega) if double else C.c_float(omega)
    for ev in (0, 1):
        assert ref.refgpu_init_neq(*(_p(x) for x in nb), _p(inv), _p(geo), *(_p(a) for a in arrs), C.c_uint(n),
                                   _p(dist), om, C.c_int(ev)) == 0
    torch.cuda.synchronize()
    return dist.double().cpu().numpy()


@pytest.mark.parametrize("real_bytes", [8, 4], ids=["f64", "f32"])
@pytest.mark.parametrize("dims,periodic", GRIDS, ids=["periodic", "walls"])
def test_neq_init_matches_reference_kernel_bitwise(cuda, oracle, real_bytes, dims, periodic):
    ref = oracle.refgpu(real_bytes)
    if ref is None:
        pytest.fail("oracle/_ref/libvfref_gpu*.so is missing: run `make -C oracle ref` where the reference tree is")
    g = ListGrid(*dims, periodic=periodic)
    fields = _smooth(g, 11)
    storage = N.STORAGE_F64 if real_bytes == 8 else N.STORAGE_F32
    sim = _sim(g, storage, N.ARITH_EXACT, 1.75, fields)
    omega = float(sim.levels[0].level.omega)
    got = sim.populations()
    want = _reference(ref, g, fields, omega, real_bytes == 8)
    assert np.array_equal(got, want)
    eq = _sim(g, storage, N.ARITH_EXACT, 1.75, fields)
    eq.para.use_init_neq = False
    eq.init(*fields)
    assert not np.array_equal(got, eq.populations())          # the part was added
    for s in (sim, eq):
        s.close()


@pytest.mark.parametrize("dims,periodic", GRIDS, ids=["periodic", "walls"])
def test_neq_init_and_steps_match_oracle_bitwise(cuda, oracle, dims, periodic):
    g = ListGrid(*dims, periodic=periodic)
    fields = _smooth(g, 12)
    sim = _sim(g, N.STORAGE_F64, N.ARITH_EXACT, 1.8, fields)
    omega = float(sim.levels[0].level.omega)
    lv = oracle.OracleLevel(g, omega)
    lv.init(*fields, neq=True)
    assert np.array_equal(sim.populations(), lv.f)
    if all(periodic):                               # no BC lists: the collision alone
        sim.run(20)
        lv.run(20)
        assert np.array_equal(sim.populations(), lv.f)
    sim.close()


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "e3m12"])
def test_neq_init_other_forms_within_their_rounding(cuda, oracle, storage):
    g = ListGrid(14, 11, 9, periodic=(True, True, True))
    fields = _smooth(g, 13)
    st = {"f32": N.STORAGE_F32, "f16": N.STORAGE_F16, "bf16": N.STORAGE_BF16, "e3m12": N.STORAGE_E3M12}[storage]
    sim = _sim(g, st, N.ARITH_FAST, 1.8, fields)
    lv = oracle.OracleLevel(g, float(sim.levels[0].level.omega))
    lv.init(*fields, neq=True)
    n = g.number_of_nodes
    got = sim.populations()
    if storage != "f32":
        got = got * np.repeat(W27, n)               # (f - w)/w back to f - w (a plane holds d or inv(d))
    fl = np.zeros(27 * n, dtype=bool)
    for p in range(27):
        fl[p * n + g.fluid] = True
    tol = {"f32": 1e-8, "f16": 2e-4, "bf16": 2e-3, "e3m12": 5e-5}[storage]
    err = np.abs(got[fl] - lv.f[fl]).max()
    assert err < tol, err
    sim.close()


def test_neq_init_needs_the_inverse_neighbours(cuda):
    g = ListGrid(6, 5, 4, periodic=(True, True, True))
    sim = _sim(g, N.STORAGE_F64, N.ARITH_EXACT, 1.8, _smooth(g, 1))
    st = N.lib().vfb_init_navier_stokes_compressible_non_equilibrium(C.byref(sim.levels[0].level), None, None)
    assert st == N.VFB_ERR_INVALID_ARGUMENT
    sim.close()
