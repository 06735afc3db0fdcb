"""The fused slab transport across processes (virtualfluids_b200.slab.DistPeerTransport): two
processes, each with one slab of a periodic box, swap the CUDA IPC handles of their population
arrays, open each other's, and step with border planes that store into the neighbour's array. The
two processes share one GPU here (their kernels never wait on each other; the step barrier is the
host's: a stream synchronisation and a gloo barrier), so the IPC mapping and the peer stores run as
they do across GPUs, without NVLink. Every node's fields equal the undivided box's bit for bit."""
import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
NX, NY, NZ, OMEGA, STEPS = 32, 24, 32, 1.9, 7


def _fields(nz, z0=0):
    z = ((np.arange(nz) + z0) + 0.5)[:, None, None] / NZ * 2 * np.pi - np.pi
    y = (np.arange(NY) + 0.5)[None, :, None] / NY * 2 * np.pi - np.pi
    x = (np.arange(NX) + 0.5)[None, None, :] / NX * 2 * np.pi - np.pi
    u0 = 0.04
    rho = 3 * (u0 ** 2 / 16) * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2)
    ux = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    uy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    uz = 0.01 * np.sin(2 * x) * np.cos(y) + 0 * z
    return [np.broadcast_to(a, (nz, NY, NX)).reshape(-1).copy() for a in (rho, ux, uy, uz)]


def _rank(rank, world, path, out):
    import torch
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"file://{path}", rank=rank, world_size=world)
    try:
        from virtualfluids_b200.slab import DistPeerTransport, Slab, slab_bounds, step
        z0, nzl = slab_bounds(NZ, world, rank)
        s = Slab(NX, NY, NZ, z0, nzl, OMEGA, arith="exact")
        s.init(*_fields(nzl, z0))
        torch.cuda.synchronize()
        tr = DistPeerTransport(s)
        for _ in range(STEPS):
            step([s], tr)
        torch.cuda.synchronize()
        dist.barrier()
        f = s.fields()
        np.save(os.path.join(out, f"fields{rank}.npy"), np.stack([f[k] for k in ("rho", "vx", "vy", "vz")]))
        dist.barrier()                    # nobody unmaps or frees an array another rank still maps
        tr.close()
        dist.barrier()
        s.close()
    finally:
        dist.destroy_process_group()


def test_two_processes_store_into_each_other(tmp_path):
    path = tempfile.mktemp(prefix="vfb_ipc_")
    mp.start_processes(_rank, args=(2, path, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    from virtualfluids_b200 import Box
    ref = Box(NX, NY, NZ, OMEGA, arith="exact")
    ref.init(*_fields(NZ))
    ref.step(STEPS)
    want = ref.fields()
    got = np.concatenate([np.load(tmp_path / f"fields{r}.npy") for r in range(2)], axis=1)
    for i, k in enumerate(("rho", "vx", "vy", "vz")):
        assert np.array_equal(got[i], want[k]), k
