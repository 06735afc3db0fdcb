"""Parity of the interpolation between refinement levels (scaleCoarseToFineCompressible /
scaleFineToCoarseCompressible) with the oracle, on the GPU, through the C ABI.

Both levels are run for a few steps on the GPU so that their populations carry non-equilibrium
parts, then the same state is handed to the oracle and both interpolate the same cells.
Tolerances, relative to the largest |f - w| of the level that is written: exact arithmetic is
bit-identical to the oracle; FMA arithmetic within 1e-12 (F64); F32 storage within 1e-5; the
16-bit storage forms within what their rounding of the written values allows.
"""
import ctypes as C

import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory, InterpolationCells, ListGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N
from virtualfluids_b200 import scale_coarse_to_fine, scale_fine_to_coarse

pytestmark = pytest.mark.gpu

W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
TOL = {(N.STORAGE_F64, N.ARITH_FAST): 1e-12, (N.STORAGE_F32, N.ARITH_FAST): 1e-5,
       (N.STORAGE_F32, N.ARITH_EXACT): 1e-5, (N.STORAGE_F16, N.ARITH_FAST): 3e-3,
       (N.STORAGE_BF16, N.ARITH_FAST): 3e-2}


def _para(omega, storage, arith):
    p = Parameter()
    p.set_viscosity_lb((1.0 / omega - 0.5) / 3.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage, p.arith = storage, arith
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


def _level(n, omega, storage, arith, steps, seed):
    g = ListGrid(n, n, n, periodic=(True, True, True))
    sim = Simulation(_para(omega, storage, arith), g, BoundaryConditionFactory())
    sim.init(*_fields(g, seed))
    sim.run(steps)
    return g, sim


def _decode(sim):
    """f - w of the stored populations (direction-major planes), as float64."""
    raw = sim.populations().reshape(27, -1)
    if sim.para.storage in (N.STORAGE_F16, N.STORAGE_BF16):
        return (raw * W[:, None]).reshape(-1)
    return raw.reshape(-1)


class _OrcLevel(C.Structure):
    _fields_ = [("n", C.c_uint64), ("f", C.c_void_p), ("nbx", C.c_void_p), ("nby", C.c_void_p), ("nbz", C.c_void_p)]


def _orc_level(g, f):
    nb = [np.ascontiguousarray(g.neighbor[a].astype(np.uint32)) for a in range(3)]
    L = _OrcLevel(g.number_of_nodes, f.ctypes.data, *(a.ctypes.data for a in nb))
    return L, nb


def _cells(gc, gf, n_cells, seed, fine_disjoint, coarse_disjoint, offsets):
    """n_cells interpolation cells: random coarse and fine MMM nodes; fine cells on even
    coordinates (disjoint eight-node blocks) for coarse to fine, distinct coarse targets for fine
    to coarse."""
    rng = np.random.default_rng(seed)
    nf, nc = gf.nx, gc.nx
    if fine_disjoint:
        blocks = np.array([(x, y, z) for z in range(0, nf, 2) for y in range(0, nf, 2) for x in range(0, nf, 2)])
        pick = blocks[rng.choice(len(blocks), n_cells, replace=False)]
    else:
        pick = rng.integers(0, nf, (n_cells, 3))
    fine = gf.node_index(pick[:, 0], pick[:, 1], pick[:, 2])
    if coarse_disjoint:
        flat = rng.choice(nc ** 3, n_cells, replace=False)
        cp = np.stack([flat % nc, (flat // nc) % nc, flat // (nc * nc)], axis=1)
    else:
        cp = rng.integers(0, nc, (n_cells, 3))
    coarse = gc.node_index(cp[:, 0], cp[:, 1], cp[:, 2])
    off = np.zeros((3, n_cells))
    if offsets:
        off[:, 1::3] = rng.choice([-0.5, 0.0, 0.5], (3, len(range(1, n_cells, 3))))
        off[:, 2::3] = rng.uniform(-0.5, 0.5, (3, len(range(2, n_cells, 3))))
    return fine.astype(np.uint32), coarse.astype(np.uint32), off


def _run(oracle, storage, arith, fine_to_coarse, coarse_steps, n_cells=200, offsets=True, seed=3):
    oc, of = 1.65, 1.8
    gc, coarse = _level(8, oc, storage, arith, coarse_steps, seed)
    gf, fine = _level(12, of, storage, arith, 2, seed + 1)
    fine_cells, coarse_cells, off = _cells(gc, gf, n_cells, seed + 2, fine_disjoint=not fine_to_coarse,
                                           coarse_disjoint=fine_to_coarse, offsets=offsets)
    fc_ = np.ascontiguousarray(_decode(coarse))
    ff_ = np.ascontiguousarray(_decode(fine))
    cells = InterpolationCells(fine_cells, coarse_cells, off, storage=storage)
    if fine_to_coarse:
        scale_fine_to_coarse(coarse, fine, cells)
    else:
        scale_coarse_to_fine(coarse, fine, cells)
    Lc, keep_c = _orc_level(gc, fc_)
    Lf, keep_f = _orc_level(gf, ff_)
    offs = [np.ascontiguousarray(off[a]) for a in range(3)]
    fn = oracle.lib().orc_scale_fc if fine_to_coarse else oracle.lib().orc_scale_cf
    fn(C.byref(Lc), C.byref(Lf), oracle.ptr(coarse_cells), oracle.ptr(fine_cells), n_cells,
       *(oracle.ptr(o) for o in offs), coarse.level.is_even_timestep, coarse.para.omega, fine.para.omega)
    if fine_to_coarse:
        return _decode(coarse), fc_, _decode(fine), ff_
    return _decode(fine), ff_, _decode(coarse), fc_


@pytest.mark.parametrize("fine_to_coarse", [False, True], ids=["coarse_to_fine", "fine_to_coarse"])
@pytest.mark.parametrize("coarse_steps", [2, 3], ids=["coarse_even", "coarse_odd"])
def test_scaling_exact_is_bitwise(oracle, cuda, fine_to_coarse, coarse_steps):
    got, want, other_got, other_want = _run(oracle, N.STORAGE_F64, N.ARITH_EXACT, fine_to_coarse, coarse_steps)
    assert np.array_equal(got, want)
    assert np.array_equal(other_got, other_want)  # the source level is untouched


@pytest.mark.parametrize("storage,arith", [(N.STORAGE_F64, N.ARITH_FAST), (N.STORAGE_F32, N.ARITH_EXACT),
                                           (N.STORAGE_F32, N.ARITH_FAST), (N.STORAGE_F16, N.ARITH_FAST),
                                           (N.STORAGE_BF16, N.ARITH_FAST)], ids=["f64", "f32x", "f32", "f16", "bf16"])
@pytest.mark.parametrize("fine_to_coarse", [False, True], ids=["coarse_to_fine", "fine_to_coarse"])
def test_scaling_storage_forms_within_tolerance(oracle, cuda, storage, arith, fine_to_coarse):
    got, want, _, _ = _run(oracle, storage, arith, fine_to_coarse, 3)
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= TOL[(storage, arith)] * scale


def test_scaling_without_cells_writes_nothing(oracle, cuda):
    got, want, _, _ = _run(oracle, N.STORAGE_F64, N.ARITH_FAST, False, 2, n_cells=0)
    assert np.array_equal(got, want)


def test_scaling_ragged_cell_counts(oracle, cuda):
    """Cell counts that leave partial warps and blocks (8 lanes per cell)."""
    for n in (1, 3, 17, 215):
        got, want, _, _ = _run(oracle, N.STORAGE_F64, N.ARITH_EXACT, False, 2, n_cells=n, seed=n)
        assert np.array_equal(got, want), n
        got, want, _, _ = _run(oracle, N.STORAGE_F64, N.ARITH_EXACT, True, 3, n_cells=n, seed=n)
        assert np.array_equal(got, want), n
