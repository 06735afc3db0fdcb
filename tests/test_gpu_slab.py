"""The slab decomposition on the GPU (virtualfluids_b200.slab): slabs of one periodic box advanced
in one process on one GPU, border planes first, the halo exchange as device copies on a second
stream overlapped with the interior planes (the NCCL transport is the same exchange over
torch.distributed; its logic runs in tests/test_dist_slab.py with gloo). After several steps the
slabs' populations equal the undivided box's bit for bit (exact FP64, FMA FP64 and FP32); with the
16-bit forms, whose stochastic rounding is keyed by the slot's offset in its own array, within the
storage error."""
import numpy as np
import pytest

from virtualfluids_b200 import Box
from virtualfluids_b200.slab import LocalTransport, Slab, slab_bounds, step

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


def _run(world, storage, arith, steps, omega=1.9):
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
    tr = LocalTransport(slabs)
    comm = torch.cuda.Stream()
    for _ in range(steps):
        step(slabs, tr, comm=comm)
    torch.cuda.synchronize()
    got = []
    for s in slabs:
        assert s.even == even
        a = s.f[:, :s.nzl * NX * NY].cpu().numpy().reshape(27, s.nzl, NY, NX)
        got.append(a)
    return np.concatenate(got, axis=1), want


@pytest.mark.parametrize("world", [1, 2, 4])
@pytest.mark.parametrize("storage,arith", [("f64", "exact"), ("f64", "fast"), ("f32", "fast")])
def test_slabs_equal_the_undivided_box(cuda, world, storage, arith):
    got, want = _run(world, storage, arith, steps=9)
    assert np.array_equal(got, want)


def test_sixteen_bit_slabs_within_storage_error(cuda):
    import torch
    got, want = _run(2, "f16", "fast", steps=9)
    g = torch.from_numpy(got.view(np.int16)).view(torch.float16).float().numpy()
    w = torch.from_numpy(want.view(np.int16)).view(torch.float16).float().numpy()
    assert np.abs(g - w).max() <= 5e-3 * np.abs(w).max()
