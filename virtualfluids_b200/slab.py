"""One domain split into z slabs over several GPUs (one process per GPU), with the halo exchange of
the esoteric-twist layout.

The reference splits a domain into subdomains with a layer of received nodes each, and after the
collision sends the 27 populations of its send nodes to the neighbour: a kernel collects them into
a buffer, MPI moves it through host memory, a kernel scatters it into the receive nodes
(Communication/ExchangeData27.cpp:52-226, ExchangeData27_Device.cu:51-460); the border nodes
collide first and the exchange overlaps the rest (Calculation/CollisisionStrategy.cpp:100-135).

Here a periodic nx x ny x NZ box is cut into R slabs of nz_local = NZ / R planes. Slab r holds its
planes [r nz_local, (r + 1) nz_local) and one ghost plane above them that stands for plane 0 of
slab r + 1 (mod R). What crosses a slab border follows from who touches each slot: in the
esoteric twist a node reads and writes the slots of its directions either at itself or, for a
direction with a negative component along an axis, at its +1 neighbour along that axis
(KernelUtilities.h:221-378), and on the next step the planes of d and inv(d) swap. So a slot in
plane P of the border plane is touched, in a step of parity e, by the node below the border when
the direction living in P at e has a negative z component, and by the node on the border when it
has a positive one (zero-z directions never cross). After the step:

* up: the ghost plane's slots of the negative-z directions (just written by this slab's top
  layer) go to plane 0 of the slab above, where its bottom layer reads them next step;
* down: plane 0's slots of the positive-z directions (just written by this slab's bottom layer) go
  to the ghost plane of the slab below, where its top layer reads them next step.

Nine direction planes each way, each a contiguous run of nx * ny values in the population array
(planes of 27 directions, x fastest), so the transfers read and write the population array in
place: no pack or unpack kernel, and nothing goes through host memory. With one slab the ghost
plane wraps onto its own plane 0.

A step: the two border planes collide on a second stream and the exchange follows them there
(NCCL point-to-point sends and receives grouped per step over NVLink, or device copies between
slabs of one process), while the interior planes collide on the compute stream; then the parity
toggles.

The fused transports (LocalPeerTransport, DistPeerTransport) have no exchange step: each border
plane's collision stores the slots a neighbour reads straight into the neighbour's population
array (vfb_box_collide_border) -- an array of this process, or another GPU's opened through CUDA IPC,
so that the stores cross NVLink as peer writes -- and a barrier between steps (a one-element NCCL
all-reduce on the exchange stream, after every rank's border planes) orders them against the
neighbour's next step. The stores go into exactly the slots the exchange would have copied, and no
node of the receiving slab touches them in the same step.
Initialisation: the slab's box is periodic in z, so each ghost node writes its slots of the
negative-z directions into plane 0 -- the slots the node below the slab owns, which no node of the
slab reads in the first step and the first exchange overwrites -- and never into the ghost-plane
slots that the slab's top layer writes. Every slot a node reads in the first step is written by a
node of its own slab. The collision never touches the ghost plane (it runs over planes
[0, nz_local) only), so the z periodicity changes nothing else.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .box import Box

# D3Q27 (src/lbm/constants/D3Q27.h:42-72)
_CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1])
_INV = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 26, 25, 24, 23, 22, 21, 20, 19])


def exchange_planes(even):
    """(up, down): the array planes sent up (ghost plane -> plane 0 of the slab above) and down
    (plane 0 -> ghost plane of the slab below) after a step of the given parity."""
    P = np.arange(27)
    d = P if even else _INV[P]
    return P[_CZ[d] < 0], P[_CZ[d] > 0]


def slab_bounds(nz_total, world, rank):
    """first global plane and plane count of a rank's slab (nz_total a multiple of world)"""
    if nz_total % world:
        raise ValueError(f"{nz_total} planes do not split into {world} equal slabs")
    n = nz_total // world
    return rank * n, n


class _Device:
    """a device buffer as a torch tensor (no copy), through __cuda_array_interface__"""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class Slab:
    """One slab of a periodic nx x ny x nz_total box on the current GPU: a structured box of
    nz_local + 1 planes (periodic in x, y and, for the initialisation only, z), the last plane the
    ghost, which is never collided."""

    def __init__(self, nx, ny, nz_total, z0, nz_local, omega, storage="f64", arith="exact"):
        import torch
        if nz_local < 2:
            raise ValueError("a slab needs at least two planes (a bottom and a top border)")
        self.nx, self.ny, self.nz_total, self.z0, self.nzl = int(nx), int(ny), int(nz_total), int(z0), int(nz_local)
        self.box = Box(nx, ny, self.nzl + 1, omega, periodic=(True, True, True), storage=storage, arith=arith)
        dist, pitch, even = C.c_void_p(), C.c_uint64(), C.c_int32()
        N.check(N.lib().vfb_box_populations(self.box._h, C.byref(dist), C.byref(pitch), C.byref(even)))
        dt = {N.STORAGE_F64: (torch.float64, "<f8"), N.STORAGE_F32: (torch.float32, "<f4"),
              N.STORAGE_F16: (torch.float16, "<f2"), N.STORAGE_BF16: (torch.int16, "<i2"),
              N.STORAGE_E3M12: (torch.int16, "<i2")}[self.box.storage]
        # the population array as a (27, pitch) tensor on the device, aliasing the box's memory
        self.f = torch.as_tensor(_Device(dist.value, (27, pitch.value), dt[1]), device="cuda")
        if dt[0] == torch.int16:
            self.f = self.f.view(torch.int16)
        self.plane_nodes = self.nx * self.ny

    @property
    def even(self):
        dist, pitch, even = C.c_void_p(), C.c_uint64(), C.c_int32()
        N.check(N.lib().vfb_box_populations(self.box._h, C.byref(dist), C.byref(pitch), C.byref(even)))
        return bool(even.value)

    def plane(self, P, z):
        """the nx * ny slots of array plane P at slab plane z (z = nz_local: the ghost plane)"""
        a = z * self.plane_nodes
        return self.f[P, a:a + self.plane_nodes]

    def init(self, rho, ux, uy, uz, stream=None):
        """equilibrium of the slab's own planes from host fields of nz_local * ny * nx values (x
        fastest); the ghost plane starts at rest (its values are never read as data)"""
        m = self.nzl * self.plane_nodes
        pad = lambda a: np.concatenate([np.asarray(a, dtype=self.box.real).reshape(-1)[:m],
                                        np.zeros(self.plane_nodes, dtype=self.box.real)])
        self.box.init(*(pad(a) for a in (rho, ux, uy, uz)), stream=stream)

    def collide(self, z_begin, z_end, stream=None):
        N.check(N.lib().vfb_box_collide_planes(self.box._h, int(z_begin), int(z_end), stream))

    @property
    def base(self):
        """device address of the population array (what a neighbour's fused border stores target)"""
        dist, pitch, even = C.c_void_p(), C.c_uint64(), C.c_int32()
        N.check(N.lib().vfb_box_populations(self.box._h, C.byref(dist), C.byref(pitch), C.byref(even)))
        return dist.value

    def collide_border(self, z, up=None, down=None, stream=None):
        """the border plane z with its neighbour stores fused (vfb_box_collide_border): up / down are
        device addresses of the population arrays of the slabs above / below, or None"""
        N.check(N.lib().vfb_box_collide_border(self.box._h, int(z), C.c_void_p(up) if up else None,
                                               C.c_void_p(down) if down else None, stream))

    def ipc_handle(self) -> bytes:
        """the CUDA IPC handle of the population array (for a neighbour in another process)"""
        h = (C.c_char * N.VFB_IPC_HANDLE_BYTES)()
        N.check(N.lib().vfb_box_ipc_handle(self.box._h, h))
        return bytes(h)

    def toggle(self):
        N.check(N.lib().vfb_box_toggle_parity(self.box._h))

    def fields(self):
        """drho, ux, uy, uz of the slab's own planes (host arrays of nz_local * ny * nx values)"""
        f = self.box.fields()
        m = self.nzl * self.plane_nodes
        return {k: v[:m] for k, v in f.items()}

    def close(self):
        self.box.close()


class LocalTransport:
    """The exchange between slabs that live in one process (device-to-device copies on the exchange
    stream): slabs[r] sits below slabs[r + 1], periodically."""

    def __init__(self, slabs):
        self.slabs = list(slabs)

    def exchange(self, even):
        up, down = exchange_planes(even)
        R = len(self.slabs)
        for r, s in enumerate(self.slabs):
            above, below = self.slabs[(r + 1) % R], self.slabs[(r - 1) % R]
            for P in up:
                above.plane(P, 0).copy_(s.plane(P, s.nzl))
            for P in down:
                below.plane(P, below.nzl).copy_(s.plane(P, 0))


class DistTransport:
    """The exchange of one slab per process with its neighbours over torch.distributed
    point-to-point operations: NCCL over NVLink for slabs on GPUs (one group of 18 sends and 18
    receives per step), gloo for host tensors. Rank r's slab lies below rank r + 1's, periodically;
    a single rank exchanges with itself by copies."""

    def __init__(self, slab, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.slab = slab
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0

    def exchange(self, even):
        up, down = exchange_planes(even)
        s = self.slab
        if self.world == 1:
            LocalTransport([s]).exchange(even)
            return
        dist = self.dist
        above, below = (self.rank + 1) % self.world, (self.rank - 1) % self.world
        ops = []
        # the same order on every rank: receives from below and above, then sends up and down
        ops += [dist.P2POp(dist.irecv, s.plane(P, 0), below, self.group) for P in up]
        ops += [dist.P2POp(dist.irecv, s.plane(P, s.nzl), above, self.group) for P in down]
        ops += [dist.P2POp(dist.isend, s.plane(P, s.nzl), above, self.group) for P in up]
        ops += [dist.P2POp(dist.isend, s.plane(P, 0), below, self.group) for P in down]
        for req in dist.batch_isend_irecv(ops):
            req.wait()


def neighbours(rank, world):
    """(above, below): the ranks whose slabs lie above and below rank's, periodically"""
    return (rank + 1) % world, (rank - 1) % world


class LocalPeerTransport:
    """The fused exchange between slabs of one process: slabs[r] sits below slabs[r + 1],
    periodically, and each border plane stores into its neighbour's array directly."""

    fused = True

    def __init__(self, slabs):
        self.slabs = list(slabs)

    def peers(self, r):
        above, below = neighbours(r, len(self.slabs))
        return self.slabs[above].base, self.slabs[below].base

    def barrier(self):
        pass


class DistPeerTransport:
    """The fused exchange of one slab per process over peer memory: the ranks swap the CUDA IPC
    handles of their population arrays once (all_gather_object), each opens the arrays of the
    ranks above and below it, and the border planes store into them directly. barrier() is a
    one-element all-reduce on the current stream (NCCL: stream-ordered after the border planes on
    every rank), so no rank starts its next step before its neighbours' stores of this step have
    landed. One rank stores into its own array. close() releases the mappings."""

    fused = True

    def __init__(self, slab, group=None):
        import torch
        import torch.distributed as dist
        self.dist, self.group, self.slab = dist, group, slab
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self._opened = {}
        if self.world == 1:
            self._up = self._down = slab.base
            return
        handles = exchange_handles(slab.ipc_handle(), group)
        above, below = neighbours(self.rank, self.world)
        for r in {above, below}:
            ptr = C.c_void_p()
            N.check(N.lib().vfb_ipc_open(handles[r], C.byref(ptr)))
            self._opened[r] = ptr.value
        self._up, self._down = self._opened[above], self._opened[below]
        self._flag = torch.zeros(1, dtype=torch.int32, device="cuda")

    def peers(self, r=0):
        return self._up, self._down

    def barrier(self):
        """NCCL: the stream-ordered all-reduce. Another backend (gloo) cannot order device work,
        so the host waits for the current stream and then meets the other ranks."""
        if self.world == 1:
            return
        if self.dist.get_backend(self.group) == "nccl":
            self.dist.all_reduce(self._flag, group=self.group)
        else:
            import torch
            torch.cuda.current_stream().synchronize()
            self.dist.barrier(group=self.group)

    def close(self):
        for ptr in self._opened.values():
            N.lib().vfb_ipc_close(C.c_void_p(ptr))
        self._opened = {}


def exchange_handles(handle: bytes, group=None) -> list:
    """every rank's IPC handle, indexed by rank (all_gather_object)"""
    import torch.distributed as dist
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, handle, group=group)
    return out


def step(slabs, transport, compute=None, comm=None):
    """One time step of slabs that share a transport. The interior planes collide on the compute
    stream while, on the comm stream, the two border planes collide and then the exchange runs: no
    node of one part touches a slot of another within a step, so the parts run concurrently and the
    interior never waits for the border. The compute stream then waits for the exchange, and the
    parity toggles. compute / comm: torch.cuda streams (the current stream and a new one when
    None); the comm stream first waits for the compute stream's earlier work."""
    import torch
    compute = compute or torch.cuda.current_stream()
    comm = comm or torch.cuda.Stream()
    even = slabs[0].even
    comm.wait_stream(compute)
    cs, ms = C.c_void_p(compute.cuda_stream), C.c_void_p(comm.cuda_stream)
    if getattr(transport, "fused", False):
        for r, s in enumerate(slabs):
            up, down = transport.peers(r)
            s.collide_border(s.nzl - 1, up=up, stream=ms)
            s.collide_border(0, down=down, stream=ms)
        with torch.cuda.stream(comm):
            transport.barrier()
    else:
        for s in slabs:
            s.collide(0, 1, ms)
            s.collide(s.nzl - 1, s.nzl, ms)
        with torch.cuda.stream(comm):
            transport.exchange(even)
    for s in slabs:
        s.collide(1, s.nzl - 1, cs)
    compute.wait_stream(comm)
    for s in slabs:
        s.toggle()
