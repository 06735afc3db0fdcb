"""The slab decomposition on the GPU (virtualfluids_b200.slab): slabs of one periodic box advanced
in one process on one GPU, border planes first on a second stream beside the interior planes, with
either transport: the halo exchange as device copies (LocalTransport; the NCCL transport is the
same exchange over torch.distributed, its logic runs in tests/test_dist_slab.py with gloo), or the
fused border planes that store straight into the neighbouring slabs' arrays (LocalPeerTransport,
the kernels of DistPeerTransport with local addresses). After several steps the slabs' populations
equal the undivided box's bit for bit (exact FP64, FMA FP64 and FP32); with the 16-bit forms,
whose stochastic rounding is keyed by the slot's offset in its own array, within the storage
error. The slots of plane 0 that the slab below reads through its ghost plane are compared there:
the fused border stores them only where they are read."""
import numpy as np
import pytest

from virtualfluids_b200 import Box
from virtualfluids_b200.slab import LocalPeerTransport, LocalTransport, Slab, exchange_planes, slab_bounds, step

pytestmark = pytest.mark.gpu
NX, NY, NZ = 32, 24, 32


def _fields(nz=NZ, z0=0, n=NX):
    z = ((np.arange(nz) + z0) + 0.5)[:, None, None] / NZ * 2 * np.pi - np.pi
    y = (np.arange(NY) + 0.5)[None, :, None] / NY * 2 * np.pi - np.pi
    x = (np.arange(NX) + 0.5)[None, None, :] / NX * 2 * np.pi - np.pi
    u0 = 0.04
    rho = 3 * (u0 ** 2 / 16) * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2)
    ux = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    uy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    uz = 0.01 * np.sin(2 * x) * np.cos(y) + 0 * z
    return [np.broadcast_to(a, (nz, NY, NX)).reshape(-1).copy() for a in (rho, ux, uy, uz)]


def _run(world, storage, arith, steps, omega=1.9, transport="copy"):
    import torch
    ref = Box(NX, NY, NZ, omega, storage=storage, arith=arith)
    ref.init(*_fields())
    ref.step(steps)
    want, even = ref.read_populations()
    want = want.reshape(27, NZ, NY, NX)
    slabs = []
    for r in range(world):
        z0, nzl = slab_bounds(NZ, world, r)
        s = Slab(NX, NY, NZ, z0, nzl, omega, storage=storage, arith=arith)
        s.init(*_fields(nzl, z0))
        slabs.append(s)
    tr = LocalTransport(slabs) if transport == "copy" else LocalPeerTransport(slabs)
    comm = torch.cuda.Stream()
    for _ in range(steps):
        step(slabs, tr, comm=comm)
    torch.cuda.synchronize()
    full = []
    for s in slabs:
        assert s.even == even
        full.append(s.f[:, :(s.nzl + 1) * NX * NY].cpu().numpy().reshape(27, s.nzl + 1, NY, NX))
    # the planes whose plane-0 slots the last step sent down (its parity is the opposite of the
    # current one): their values for the next step are in the ghost plane of the slab below
    _, down = exchange_planes(not even)
    got = []
    for r, a in enumerate(full):
        own = a[:, :slabs[r].nzl].copy()
        below = full[(r - 1) % world]
        for P in down:
            own[P, 0] = below[P, -1]
        got.append(own)
    return np.concatenate(got, axis=1), want


@pytest.mark.parametrize("transport", ["copy", "fused"])
@pytest.mark.parametrize("world", [1, 2, 4])
@pytest.mark.parametrize("storage,arith", [("f64", "exact"), ("f64", "fast"), ("f32", "fast")])
def test_slabs_equal_the_undivided_box(cuda, world, storage, arith, transport):
    got, want = _run(world, storage, arith, steps=9, transport=transport)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("world", [1, 2])
def test_fused_slab_fields_equal_the_undivided_box(cuda, world):
    """the macroscopic fields of every slab node, which read only slots the fused stores keep
    correct, after an even and an odd number of steps"""
    import torch
    for steps in (6, 7):
        ref = Box(NX, NY, NZ, 1.9, arith="exact")
        ref.init(*_fields())
        ref.step(steps)
        want = ref.fields()
        slabs = []
        for r in range(world):
            z0, nzl = slab_bounds(NZ, world, r)
            s = Slab(NX, NY, NZ, z0, nzl, 1.9, arith="exact")
            s.init(*_fields(nzl, z0))
            slabs.append(s)
        tr = LocalPeerTransport(slabs)
        for _ in range(steps):
            step(slabs, tr)
        torch.cuda.synchronize()
        got = [s.fields() for s in slabs]
        for k in ("rho", "vx", "vy", "vz"):
            assert np.array_equal(np.concatenate([g[k] for g in got]), want[k]), (steps, k)


@pytest.mark.parametrize("transport", ["copy", "fused"])
def test_sixteen_bit_slabs_within_storage_error(cuda, transport):
    import torch
    got, want = _run(2, "f16", "fast", steps=9, transport=transport)
    g = torch.from_numpy(got.view(np.int16)).view(torch.float16).float().numpy()
    w = torch.from_numpy(want.view(np.int16)).view(torch.float16).float().numpy()
    assert np.abs(g - w).max() <= 5e-3 * np.abs(w).max()
