"""Domain pools on the GPU: many independent boxes of uneven sizes advanced by one persistent
launch per step (graph replay), with admission against the arena and removal mid-run.

Every domain must compute exactly what the same box computes alone (bit for bit, in every storage
form and arithmetic), whatever else shares the pool, when it joined, which launch shape the
autotuner picked and whether the steps were replayed from a CUDA graph. Rectangular-duct Poiseuille
domains (periodic in x, walls in y and z, body force) must reach the analytic duct profile.
"""
import numpy as np
import pytest

from virtualfluids_b200 import Box, Pool
from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu


def _stream():
    import torch
    return torch.cuda.Stream()


def _fields(shape, seed, amp_rho=1e-2, amp_u=0.03):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    out = []
    for amp in (amp_rho, amp_u, amp_u, amp_u):
        k = rng.integers(1, 3, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        out.append((amp * np.cos(2 * np.pi * k[0] * x / nx + ph[0]) * np.cos(2 * np.pi * k[1] * y / ny + ph[1])
                    * np.cos(2 * np.pi * k[2] * z / nz + ph[2])).reshape(-1))
    return out


def _wall_mask(shape, periodic):
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    wall = np.zeros_like(x, dtype=bool)
    for c, n, p in ((x, nx, periodic[0]), (y, ny, periodic[1]), (z, nz, periodic[2])):
        if not p:
            wall |= (c == 0) | (c == n - 1)
    return (~wall).astype(np.uint8).reshape(-1)


DOMAINS = [((16, 12, 10), (True, True, True), 1.8, (0.0, 0.0, 0.0)),
           ((21, 9, 13), (True, False, False), 1.75, (2e-5, 0.0, 0.0)),
           ((8, 24, 11), (False, True, False), 1.85, (0.0, 1e-5, 0.0)),
           ((33, 17, 5), (True, True, False), 1.7, (0.0, 0.0, 0.0)),
           ((12, 12, 40), (False, False, True), 1.9, (0.0, 0.0, 3e-6))]


def _alone(shape, periodic, omega, forces, storage, arith, seed, steps):
    mask = None if all(periodic) else _wall_mask(shape, periodic)
    b = Box(*shape, omega, periodic=periodic, storage=storage, arith=arith, forces=forces, mask=mask)
    b.init(*_fields(shape, seed))
    b.step(steps)
    f = b.fields()
    return [f[k].reshape(shape[2], shape[1], shape[0]) for k in ("rho", "vx", "vy", "vz")]


@pytest.mark.parametrize("storage,arith", [("f64", "exact"), ("f64", "fast"), ("f32", "fast"), ("f16", "fast"),
                                           ("bf16", "fast"), ("e3m12", "fast")])
def test_pool_domains_match_boxes_alone_bitwise(cuda, storage, arith):
    steps = 37
    s = _stream()
    pool = Pool(1 << 28, storage=storage, arith=arith, max_domains=64)
    ids = []
    for i, (shape, periodic, omega, forces) in enumerate(DOMAINS):
        d = pool.add(shape, omega, periodic=periodic, forces=forces)
        pool.init(d, *_fields(shape, 10 + i), stream=s)
        ids.append(d)
    pool.step(steps, stream=s)
    s.synchronize()
    for i, (shape, periodic, omega, forces) in enumerate(DOMAINS):
        got = pool.fields(ids[i], stream=s)
        want = _alone(shape, periodic, omega, forces, storage, arith, 10 + i, steps)
        fl = _wall_mask(shape, periodic).reshape(shape[2], shape[1], shape[0]) != 0
        for g, w in zip(got, want):
            assert np.array_equal(g[fl], w[fl]), (i, storage, arith)


def test_joining_late_leaving_early_graph_and_shapes_change_nothing(cuda):
    """A domain that joins at an odd step, a neighbour removed mid-run, graph replay on or off and
    every autotuner shape: the remaining domains' bits are those of their runs alone."""
    s = _stream()
    pool = Pool(1 << 28, storage="f32", max_domains=16)
    (sa, pa, oa, fa), (sb, pb, ob, fb), (sc, pc, oc, fc) = DOMAINS[0], DOMAINS[1], DOMAINS[2]
    a = pool.add(sa, oa, periodic=pa, forces=fa)
    pool.init(a, *_fields(sa, 1), stream=s)
    b = pool.add(sb, ob, periodic=pb, forces=fb)
    pool.init(b, *_fields(sb, 2), stream=s)
    pool.step(5, stream=s)                          # pool parity now odd
    c = pool.add(sc, oc, periodic=pc, forces=fc)
    pool.init(c, *_fields(sc, 3), stream=s)         # joins at an odd step
    pool.set_launch(threads=64, nodes_per_thread=2, use_graph=False)
    pool.step(11, stream=s)
    pool.remove(b)
    pool.set_launch(threads=256, nodes_per_thread=1, use_graph=True)
    pool.step(33, stream=s)                         # graph replays (16 + 16) and one direct step
    pool.autotune(trial_steps=2, stream=s)          # 15 shapes x 4 steps = 60 more steps
    pool.step(20, stream=s)
    s.synchronize()
    total_a = 5 + 11 + 33 + 60 + 20
    total_c = 11 + 33 + 60 + 20
    for d, (shape, periodic, omega, forces), seed, steps in ((a, DOMAINS[0], 1, total_a), (c, DOMAINS[2], 3, total_c)):
        got = pool.fields(d, stream=s)
        want = _alone(shape, periodic, omega, forces, "f32", "fast", seed, steps)
        fl = _wall_mask(shape, periodic).reshape(shape[2], shape[1], shape[0]) != 0
        for g, w in zip(got, want):
            assert np.array_equal(g[fl], w[fl])
    assert pool.stats()["active_domains"] == 2


def test_admission_against_the_arena(cuda):
    s = _stream()
    shape = (24, 24, 24)
    probe = Pool(1 << 20, storage="f32", max_domains=4)
    per = probe.domain_bytes(shape, periodic=(True, False, False), has_mask=True)
    probe.close()
    pool = Pool(3 * per + 1024, storage="f32", max_domains=8)
    ids = [pool.try_add(shape, 1.8, periodic=(True, False, False)) for _ in range(4)]
    assert ids[3] is None and all(i is not None for i in ids[:3])
    for i in ids[:3]:
        pool.init(i, stream=s)
    pool.step(4, stream=s)
    pool.remove(ids[1])
    assert pool.try_add(shape, 1.8, periodic=(True, False, False)) is None   # not reusable until the stream drains
    pool.synchronize(stream=s)
    again = pool.try_add(shape, 1.8, periodic=(True, False, False))
    assert again is not None
    st = pool.stats()
    assert st["used_bytes"] == 3 * per and st["active_domains"] == 2


def _duct_series(ny, nz, g, nu, terms=101):
    """Rectangular-duct Poiseuille profile u(y, z) for a body force g along x, no-slip walls
    half-way between the solid layers and the first fluid nodes (series solution of the Poisson
    problem lap u = -g / nu)."""
    a, b = (ny - 2) / 2.0, (nz - 2) / 2.0
    y = np.arange(ny) - (ny - 1) / 2.0
    z = np.arange(nz) - (nz - 1) / 2.0
    Z, Y = np.meshgrid(z, y, indexing="ij")
    u = np.zeros_like(Y)
    for n in range(1, terms + 1, 2):
        k = n * np.pi / (2 * a)
        u += (-1) ** ((n - 1) // 2) / n ** 3 * (1 - np.cosh(k * Z) / np.cosh(k * b)) * np.cos(k * Y)
    return 16 * a * a * g / (nu * np.pi ** 3) * u


def test_duct_poiseuille_domains_reach_the_analytic_profile(cuda):
    """Viscosities at or below 1/42: above it K17 is unstable (a shear wave grows at nu = 0.04 in
    the reference's own arithmetic), which is why Parameter warns there."""
    s = _stream()
    pool = Pool(1 << 28, storage="f32", max_domains=16)
    cases = [(8, 14, 10, 0.01), (6, 18, 12, 0.015), (4, 10, 16, 0.02)]
    ids = []
    for nx, ny, nz, nu in cases:
        omega = 1.0 / (3 * nu + 0.5)
        g = 2e-6
        d = pool.add((nx, ny, nz), omega, periodic=(True, False, False), forces=(g, 0.0, 0.0))
        pool.init(d, stream=s)
        ids.append((d, ny, nz, nu, g))
    pool.step(6000, stream=s)
    s.synchronize()
    for d, ny, nz, nu, g in ids:
        _, ux, _, _ = pool.fields(d, stream=s)
        u = ux.mean(axis=2)[1:-1, 1:-1]               # average over x, fluid nodes only
        ref = _duct_series(ny, nz, g, nu)[1:-1, 1:-1]
        err = np.sqrt(((u - ref) ** 2).sum() / (ref ** 2).sum())
        assert err < 0.02, (ny, nz, nu, err)


def _porous_alone(g, omega, storage, arith, steps, seed):
    b = Box(*g["shape"], omega, periodic=(False, True, True), storage=storage, arith=arith, mask=g["mask"])
    k, q = g["bcs"]["noslip"]
    b.set_bc("noslip", k, q, N.NOSLIP_INTERPOLATED_COMPRESSIBLE)
    pk, pkn, prho, pdir = g["bcs"]["pressure"]
    for d in (N.DIR_M00, N.DIR_P00):
        sel = pdir == d
        b.add_pressure_bc(pk[sel], pkn[sel], prho[sel], d)
    b.init(*_fields(g["shape"], seed, amp_u=0.005))
    b.step(steps)
    f = b.fields()
    nx, ny, nz = g["shape"]
    return [f[key].reshape(nz, ny, nx) for key in ("rho", "vx", "vy", "vz")]


@pytest.mark.parametrize("storage,arith", [("f64", "exact"), ("f32", "fast"), ("f16", "fast")])
def test_pool_boundary_condition_lists_match_boxes_alone_bitwise(cuda, storage, arith):
    """Porous blocks between pressure planes with exact sphere q: the pool's per-domain no-slip and
    pressure lists (one launch each for all domains) compute what a box with the same lists does."""
    from virtualfluids_b200.workloads import porous_block_bcs
    geos = [porous_block_bcs(side, seed, porosity=0.75) for side, seed in ((20, 1), (28, 2), (24, 3))]
    steps, omegas = 41, (1.8, 1.7, 1.9)
    s = _stream()
    pool = Pool(1 << 28, storage=storage, arith=arith, max_domains=8)
    plain = pool.add((12, 10, 8), 1.8)           # a domain without lists shares the steps
    pool.init(plain, *_fields((12, 10, 8), 9), stream=s)
    ids = []
    for i, g in enumerate(geos):
        assert g["bcs"]["noslip"][0].size > 0
        d = pool.add(g["shape"], omegas[i], periodic=(False, True, True), mask=g["mask"], bcs=g["bcs"])
        pool.init(d, *_fields(g["shape"], 20 + i, amp_u=0.005), stream=s)
        ids.append(d)
    pool.step(steps, stream=s)
    s.synchronize()
    assert pool.kernel_launches() >= 3 * steps
    for i, g in enumerate(geos):
        got = pool.fields(ids[i], stream=s)
        want = _porous_alone(g, omegas[i], storage, arith, steps, 20 + i)
        nx, ny, nz = g["shape"]
        fl = g["mask"].reshape(nz, ny, nx) != 0
        for a, b in zip(got, want):
            assert np.array_equal(a[fl], b[fl]), (i, storage)
        assert np.abs(got[1][fl]).max() > 0


def test_pool_rejects_bad_boundary_condition_lists(cuda):
    from virtualfluids_b200.workloads import porous_block_bcs
    g = porous_block_bcs(20, 1, porosity=0.8)
    pool = Pool(1 << 26, storage="f32", max_domains=4)
    k, q = g["bcs"]["noslip"]
    solid = int(np.nonzero(g["mask"] == 0)[0][0])
    for bad in ({"noslip": (np.array([solid]), np.zeros((27, 1)))},
                {"noslip": (np.array([10 ** 7]), np.zeros((27, 1)))},
                {"pressure": (np.array([30]), np.array([10 ** 8]), 0.0, N.DIR_M00)},
                {"pressure": (np.array([30]), np.array([31]), 0.0, 7)}):
        with pytest.raises(N.VfbError) as e:
            pool.add(g["shape"], 1.8, periodic=(False, True, True), mask=g["mask"], bcs=bad)
        assert e.value.status == N.VFB_ERR_INVALID_ARGUMENT
    assert pool.stats()["used_bytes"] == 0


def test_watchdog_flags_only_the_diverged_domain(cuda):
    """A domain initialised with a NaN velocity is reported by the watchdog; the others keep their
    FP64 mass (periodic: conserved to round-off) and run on after it is removed."""
    s = _stream()
    pool = Pool(1 << 27, storage="f64", max_domains=8)
    shapes = [(12, 10, 8), (9, 9, 9), (16, 6, 7)]
    ids = []
    for i, shape in enumerate(shapes):
        d = pool.add(shape, 1.8)
        f = _fields(shape, 30 + i)
        if i == 1:
            f[1] = f[1].copy()
            f[1][5] = np.nan
        pool.init(d, *f, stream=s)
        ids.append(d)
    assert pool.watchdog(stream=s) == [ids[1]]
    m0 = pool.domain_mass(stream=s)
    assert np.isnan(m0[ids[1]]) and np.isfinite(m0[ids[0]]) and np.isfinite(m0[ids[2]])
    pool.remove(ids[1])
    pool.step(50, stream=s)
    assert pool.watchdog(stream=s) == []
    m1 = pool.domain_mass(stream=s)
    for d in (ids[0], ids[2]):
        assert abs(m1[d] - m0[d]) <= 1e-12 * m0[d]
    assert abs(m0[ids[0]] - np.prod(shapes[0])) < 1.0      # sum(1 + drho) ~ node count
