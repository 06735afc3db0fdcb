"""The slab decomposition's halo exchange (virtualfluids_b200.slab) on the CPU: ranks of gloo
processes each advance one slab of a periodic box with the oracle's collision, exchange the border
planes through the library's DistTransport (the same point-to-point code the GPUs run over NCCL),
and after several steps every slab equals its planes of the undivided box bit for bit. One slab
(the ghost plane wrapping onto itself) and the plane sets of the exchange are checked in-process.
The host side of the fused transport (DistPeerTransport: every rank's IPC handle gathered, the
ranks above and below chosen) runs on gloo ranks with stand-in handles."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from virtualfluids_b200.gridgen import ImportedLevel
from virtualfluids_b200.slab import (DistTransport, LocalTransport, exchange_handles, exchange_planes, neighbours,
                                     slab_bounds)

NX, NY, NZ = 6, 5, 12
OMEGA = 1.8


def _fields(nz, z0=0):
    z = (np.arange(nz) + z0)[:, None, None]
    y = np.arange(NY)[None, :, None]
    x = np.arange(NX)[None, None, :]
    k = 2 * np.pi
    rho = 1e-3 * np.cos(k * x / NX) * np.sin(k * z / NZ) + 0 * y
    ux = 0.03 * np.sin(k * y / NY) * np.cos(k * z / NZ) + 0 * x
    uy = 0.02 * np.cos(k * x / NX) * np.sin(k * z / NZ) + 0 * y
    uz = 0.025 * np.sin(k * x / NX + 0.3) * np.cos(k * y / NY) + 0 * z
    return [np.broadcast_to(a, (nz, NY, NX)).reshape(-1).copy() for a in (rho, ux, uy, uz)]


def _level(nz, ghost):
    """a box of nz planes (x fastest, node 0 the dummy), periodic in x and y; with a ghost plane on
    top (never collided, its +z neighbour the dummy) or periodic in z"""
    planes = nz + (1 if ghost else 0)
    n = 1 + NX * NY * planes
    x, y, z = np.meshgrid(np.arange(NX), np.arange(NY), np.arange(planes), indexing="xy")
    x, y, z = (a.transpose(2, 0, 1).reshape(-1) for a in (x, y, z))
    k = 1 + x + NX * (y + NY * z)
    nb = np.zeros((3, n), dtype=np.uint32)
    nb[0, k] = 1 + (x + 1) % NX + NX * (y + NY * z)
    nb[1, k] = 1 + x + NX * ((y + 1) % NY + NY * z)
    zp = z + 1 if ghost else (z + 1) % planes
    nb[2, k] = np.where(zp < planes, 1 + x + NX * (y + NY * np.minimum(zp, planes - 1)), 0)
    geo = np.full(n, 16, dtype=np.uint32)
    fluid = k[z < nz].astype(np.uint32)
    geo[fluid] = 19
    coords = np.zeros((3, n))
    return ImportedLevel(number_of_nodes=n, neighbor=nb, geo=geo, fluid=fluid, coords=coords, delta=1.0)


class OracleSlab:
    """a slab advanced by the oracle, with the plane views DistTransport exchanges (host tensors)"""

    def __init__(self, oracle, z0, nzl):
        self.z0, self.nzl = z0, nzl
        self.level = _level(nzl, ghost=True)
        self.o = oracle.OracleLevel(self.level, omega=OMEGA)
        full = [np.concatenate([[0.0], a, np.zeros(NX * NY)]) for a in _fields(nzl, z0)]
        self.o.init(*full)                           # the ghost plane is not fluid: left untouched
        self.t = torch.from_numpy(self.o.f).view(27, -1)

    def plane(self, P, z):
        a = 1 + z * NX * NY
        return self.t[P, a:a + NX * NY]

    def collide(self, oracle, nodes):
        lim, forces = np.full(3, 0.01), np.zeros(3)
        oracle.lib().orc_collision(C.byref(self.o.L), oracle.ptr(nodes), nodes.size, self.o.is_even.value, OMEGA,
                                   oracle.ptr(lim), oracle.ptr(forces), 0, None, None, None, None, 1)

    def step(self, oracle, transport):
        planes = NX * NY
        even = bool(self.o.is_even.value)
        fl = self.level.fluid
        border = np.concatenate([fl[:planes], fl[-planes:]])
        self.collide(oracle, border)
        transport.exchange(even)
        self.collide(oracle, np.ascontiguousarray(fl[planes:-planes]))
        self.o.is_even.value = 1 - self.o.is_even.value

    def own(self):
        """populations of the slab's own planes, (27, nzl * NX * NY)"""
        return self.t[:, 1:1 + self.nzl * NX * NY].numpy().copy()


def _undivided(oracle, steps):
    g = _level(NZ, ghost=False)
    o = oracle.OracleLevel(g, omega=OMEGA)
    o.init(*[np.concatenate([[0.0], a]) for a in _fields(NZ)])
    o.run(steps)
    return o.f.reshape(27, -1)[:, 1:]


def _rank(rank, world, path, steps, out):
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("gloo", init_method=f"file://{path}", rank=rank, world_size=world)
    try:
        from oracle import pyoracle as oracle
        z0, nzl = slab_bounds(NZ, world, rank)
        s = OracleSlab(oracle, z0, nzl)
        tr = DistTransport(s)
        for _ in range(steps):
            s.step(oracle, tr)
        np.save(os.path.join(out, f"slab{rank}.npy"), s.own())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_decomposed_run_equals_the_undivided_box(oracle, world, tmp_path):
    steps = 7
    path = tempfile.mktemp(prefix="vfb_slab_")
    mp.start_processes(_rank, args=(world, path, steps, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    want = _undivided(oracle, steps)
    for r in range(world):
        z0, nzl = slab_bounds(NZ, world, r)
        got = np.load(tmp_path / f"slab{r}.npy")
        assert np.array_equal(got, want[:, z0 * NX * NY:(z0 + nzl) * NX * NY]), r


def test_single_slab_wraps_onto_itself(oracle):
    steps = 5
    s = OracleSlab(oracle, 0, NZ)
    tr = LocalTransport([s])
    for _ in range(steps):
        s.step(oracle, tr)
    assert np.array_equal(s.own(), _undivided(oracle, steps))


def test_exchange_plane_sets():
    for even in (True, False):
        up, down = exchange_planes(even)
        assert len(up) == 9 and len(down) == 9 and not set(up) & set(down)
        # a plane sent up after one parity is sent down after the other (the directions swap planes)
        assert set(exchange_planes(not even)[1]) == set(up)
    with pytest.raises(ValueError):
        slab_bounds(10, 3, 0)


def _handles_rank(rank, world, path, out):
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("gloo", init_method=f"file://{path}", rank=rank, world_size=world)
    try:
        mine = bytes([rank + 1]) * 64                   # a stand-in for a 64-byte CUDA IPC handle
        handles = exchange_handles(mine)
        above, below = neighbours(rank, world)
        np.save(os.path.join(out, f"h{rank}.npy"),
                np.array([handles == [bytes([r + 1]) * 64 for r in range(world)], handles[above][0] - 1,
                          handles[below][0] - 1]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_fused_transport_host_side(world, tmp_path):
    path = tempfile.mktemp(prefix="vfb_handles_")
    mp.start_processes(_handles_rank, args=(world, path, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        ok, above, below = np.load(tmp_path / f"h{r}.npy")
        assert ok and above == (r + 1) % world and below == (r - 1) % world
