"""Structured boxes: full-box domains advanced by the arithmetic-neighbour kernels.

A thin owner of a ``vfb_box`` handle (include/vfb.h). Inputs and outputs may be host numpy
arrays (copied inside the call, as an end-to-end user would) or device torch tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .simulation import STORAGE


def _dev_ptr(x):
    return C.c_void_p(x.data_ptr())


class Box:
    def __init__(self, nx, ny, nz, omega, periodic=(True, True, True), storage="f64", arith="fast",
                 forces=(0.0, 0.0, 0.0), quadric_limiters=(0.01, 0.01, 0.01), mask=None):
        self.shape = (int(nx), int(ny), int(nz))
        self.storage = STORAGE[storage] if isinstance(storage, str) else int(storage)
        self.real = np.float64 if self.storage == N.STORAGE_F64 else np.float32
        d = N.BoxDesc()
        d.nx, d.ny, d.nz = self.shape
        d.periodic_x, d.periodic_y, d.periodic_z = (int(bool(p)) for p in periodic)
        d.storage = self.storage
        d.arith = N.ARITH_EXACT if arith == "exact" else N.ARITH_FAST
        d.omega = float(omega)
        for i in range(3):
            d.forces[i] = float(forces[i])
            d.quadric_limiters[i] = float(quadric_limiters[i])
        self._mask = None
        if mask is not None:
            self._mask = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).reshape(-1))
            d.mask = self._mask.ctypes.data
        h = C.c_void_p()
        N.check(N.lib().vfb_box_create(C.byref(d), C.byref(h)))
        self._h = h
        self.n = nx * ny * nz

    def close(self):
        if getattr(self, "_h", None):
            N.lib().vfb_box_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        b = C.c_uint64()
        N.check(N.lib().vfb_box_device_bytes(self._h, C.byref(b)))
        return b.value

    def init(self, rho, ux, uy, uz, stream=None):
        """Equilibrium from drho and velocity fields (x fastest); numpy = host, torch = device."""
        if isinstance(rho, np.ndarray):
            arrs = [np.ascontiguousarray(a, dtype=self.real).reshape(-1) for a in (rho, ux, uy, uz)]
            self._host_keep = arrs
            ptrs = [C.c_void_p(a.ctypes.data) for a in arrs]
            N.check(N.lib().vfb_box_init(self._h, *ptrs, 1, stream))
            N.check(N.lib().vfb_synchronize(stream))
        else:
            N.check(N.lib().vfb_box_init(self._h, *(_dev_ptr(a) for a in (rho, ux, uy, uz)), 0, stream))

    def step(self, steps: int, energy=None, stream=None):
        """Advance; energy: None, host float64 array [steps, 2] or device float64 tensor."""
        if getattr(self, "_drag_len", 0):
            self._drag_done += int(steps)
        if energy is None:
            N.check(N.lib().vfb_box_step(self._h, int(steps), None, 0, stream))
        elif isinstance(energy, np.ndarray):
            assert energy.dtype == np.float64 and energy.size >= 2 * steps
            N.check(N.lib().vfb_box_step(self._h, int(steps), C.c_void_p(energy.ctypes.data), 1, stream))
        else:
            N.check(N.lib().vfb_box_step(self._h, int(steps), _dev_ptr(energy), 0, stream))

    def fields(self, out=None, stream=None):
        """drho, ux, uy, uz of the current state. Host numpy by default; device tensors if given."""
        if out is None:
            arrs = [np.empty(self.n, dtype=self.real) for _ in range(4)]
            N.check(N.lib().vfb_box_fields(self._h, *(C.c_void_p(a.ctypes.data) for a in arrs), 1, stream))
            N.check(N.lib().vfb_synchronize(stream))
            return dict(zip(("rho", "vx", "vy", "vz"), arrs))
        N.check(N.lib().vfb_box_fields(self._h, *(_dev_ptr(a) for a in out), 0, stream))
        return out

    def status(self, stream=None) -> int:
        """Synchronise and check the device status word; raises if a kernel gave up waiting."""
        v = C.c_int32()
        N.check(N.lib().vfb_box_status(self._h, C.byref(v), stream))
        return v.value

    def set_kernel_variant(self, variant: str):
        """'auto', 'direct' (plain loads), 'tma' (bulk copies staged in shared memory), 'async'
        (per-thread asynchronous copies of the next node), 'pairs' (two nodes per thread in packed
        FP32x2 arithmetic; FP32-arithmetic forms) or 'pipe' (persistent blocks, the next node's loads
        in flight in registers while the current node is collided)."""
        N.check(N.lib().vfb_box_set_kernel_variant(
            self._h, {"auto": 0, "direct": 1, "tma": 2, "async": 3, "pairs": 4, "pipe": 5}[variant]))

    # -- boundary conditions (vfb_box_set_bc / vfb_box_add_pressure_bc) -------------------------
    def set_bc(self, kind: str, k, q27, variant, velocity=None):
        """kind: 'velocity', 'noslip', 'slip' or 'geometry'; k: box node indices; q27: (27, n) q values;
        velocity: (3, n) wall velocities for 'velocity'; variant: the factory enum value."""
        kk = np.ascontiguousarray(np.asarray(k, dtype=np.int32).reshape(-1))
        n = kk.size
        q = np.ascontiguousarray(np.asarray(q27, dtype=self.real).reshape(27, n))
        vel = [None, None, None]
        if kind == "velocity":
            v = np.asarray(velocity, dtype=self.real).reshape(3, n)
            vel = [np.ascontiguousarray(v[a]) for a in range(3)]
        code = {"velocity": N.BOX_BC_VELOCITY, "noslip": N.BOX_BC_NOSLIP, "geometry": N.BOX_BC_GEOMETRY,
                "slip": N.BOX_BC_SLIP}[kind]
        N.check(N.lib().vfb_box_set_bc(self._h, code, int(variant), kk.ctypes.data, q.ctypes.data, n,
                                       *(a.ctypes.data if a is not None else None for a in vel)))
        if kind == "geometry":
            self._geometry_nodes = n

    def add_pressure_bc(self, k, k_neighbor, rho, direction, variant=N.PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE):
        kk = np.ascontiguousarray(np.asarray(k, dtype=np.int32).reshape(-1))
        kn = np.ascontiguousarray(np.asarray(k_neighbor, dtype=np.int32).reshape(-1))
        r = np.ascontiguousarray(np.broadcast_to(np.asarray(rho, dtype=self.real), kk.shape))
        N.check(N.lib().vfb_box_add_pressure_bc(self._h, int(variant), kk.ctypes.data, kn.ctypes.data, r.ctypes.data,
                                                kk.size, int(direction)))

    def set_velocity_perturbation(self, seed: int, amplitude: float):
        N.check(N.lib().vfb_box_set_velocity_perturbation(self._h, int(seed), float(amplitude)))

    def enable_drag_lift(self, history_steps: int, device="cuda"):
        import torch
        self._drag_hist = torch.zeros(3 * int(history_steps), dtype=torch.float64, device=device)
        self._drag_len = int(history_steps)
        self._drag_done = 0
        N.check(N.lib().vfb_box_set_drag_lift(self._h, C.c_void_p(self._drag_hist.data_ptr()), self._drag_len))

    def drag_lift_history(self):
        """(steps, 3) FP64 forces of the steps since enable_drag_lift (the last history_steps)."""
        N.check(N.lib().vfb_synchronize(None))
        h = self._drag_hist.view(self._drag_len, 3).cpu().numpy()
        done = self._drag_done
        if done <= self._drag_len:
            return h[:done].copy()
        start = done % self._drag_len
        return np.concatenate([h[start:], h[:start]])

    @classmethod
    def from_grid(cls, grid, omega, bc_factory, storage="f64", arith="fast", forces=(0.0, 0.0, 0.0)):
        """The structured-box form of a ListGrid level: the box spans the grid with its stopper shell
        (list node k = box node k + grid.first_node), the mask marks the fluid nodes, and the grid's
        BC lists become box BC lists with the factory's kernels. It computes what the list form
        computes."""
        Dx, Dy, Dz = grid.dims
        f0 = grid.first_node
        mask = (grid.geo[f0:f0 + Dx * Dy * Dz] == N.GEO_FLUID).astype(np.uint8)
        box = cls(Dx, Dy, Dz, omega, periodic=grid.periodic, storage=storage, arith=arith, forces=forces, mask=mask)
        for kind, variant in (("velocity", bc_factory.velocity), ("noslip", bc_factory.noslip),
                              ("slip", bc_factory.slip), ("geometry", bc_factory.geometry)):
            m = grid.merged(kind)
            if m is None:
                continue
            k, q, vel = m
            box.set_bc(kind, k.astype(np.int64) - f0, q, int(variant), velocity=vel if kind == "velocity" else None)
        from .grid import SIDE_DIR
        for b in grid.bcs:
            if b.kind == "pressure":
                box.add_pressure_bc(b.k.astype(np.int64) - f0, b.k_neighbor.astype(np.int64) - f0, b.rho,
                                    SIDE_DIR[b.side], variant=int(bc_factory.pressure))
        return box

    def kernel_launches(self) -> int:
        """Kernels vfb_box_step has launched for this box so far."""
        c = C.c_uint64()
        N.check(N.lib().vfb_box_kernel_launches(self._h, C.byref(c)))
        return c.value

    def set_launch_shape(self, blocks_per_sm: int = 0, smem_kb: int = 0):
        """Launch shape of the asynchronous-copy kernel (resident blocks per SM, shared-memory
        configuration in KB to pad to; 0 = defaults). Results do not depend on it."""
        N.check(N.lib().vfb_box_set_launch_shape(self._h, int(blocks_per_sm), int(smem_kb)))

    def _storage_np(self):
        return {N.STORAGE_F64: np.float64, N.STORAGE_F32: np.float32}.get(self.storage, np.uint16)

    def read_populations(self):
        """The 27 population planes (27 * nx*ny*nz values as stored, 16-bit forms as raw uint16)
        and the parity."""
        out = np.empty(27 * self.n, dtype=self._storage_np())
        ev = C.c_int32()
        N.check(N.lib().vfb_box_read_populations(self._h, out.ctypes.data, 1, C.byref(ev), None))
        return out, bool(ev.value)

    def write_populations(self, planes, is_even=True):
        a = np.ascontiguousarray(planes, dtype=self._storage_np()).reshape(-1)
        if a.size != 27 * self.n:
            raise ValueError(f"{a.size} values, {27 * self.n} expected")
        N.check(N.lib().vfb_box_write_populations(self._h, a.ctypes.data, 1, int(bool(is_even)), None))

    def save_restart(self, path):
        """The box's populations in the layout of the reference's binary restart file (one level),
        `path` + ".bin"; box node order."""
        from .output import save_restart
        save_restart(path, [self.read_populations()[0]])

    def load_restart(self, path, is_even=True):
        from .output import load_restart
        (a,) = load_restart(path, [self._storage_np()])
        self.write_populations(a, is_even)

    def write_vtk(self, path, spacing=1.0, origin=(0.0, 0.0, 0.0)):
        """drho and velocity of every node as a legacy VTK image (STRUCTURED_POINTS)."""
        from .output import write_vtk_image
        f = self.fields()
        write_vtk_image(path, self.shape, {"drho": f["rho"], "velocity": np.stack([f["vx"], f["vy"], f["vz"]])},
                        origin=origin, spacing=spacing)

    def populations(self):
        """(device pointer, plane pitch in elements, is_even) of the population array."""
        p, pitch, ev = C.c_void_p(), C.c_uint64(), C.c_int32()
        N.check(N.lib().vfb_box_populations(self._h, C.byref(p), C.byref(pitch), C.byref(ev)))
        return p.value, pitch.value, ev.value
