"""Domain pools: many independent boxes of uneven sizes advanced together (``vfb_pool_*``).

A pool owns one device arena sized at creation. Domains are carved from it and released again,
so a request loop can admit solves against an HBM budget; every step advances all active domains
with one persistent kernel over a work list of node blocks, replayed from a captured CUDA graph.
Each domain computes exactly what a :class:`~virtualfluids_b200.box.Box` of the same description
computes. No counterpart in the reference, which runs one domain per simulation.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

_STORAGE = {"f64": N.STORAGE_F64, "f32": N.STORAGE_F32, "f16": N.STORAGE_F16, "bf16": N.STORAGE_BF16,
            "e3m12": N.STORAGE_E3M12}


def _stream_ptr(stream):
    if stream is None:
        return None
    if isinstance(stream, C.c_void_p):
        return stream
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


class Pool:
    def __init__(self, arena_bytes: int, storage: str = "f32", arith: str = "fast", max_domains: int = 8192):
        d = N.PoolDesc(_STORAGE[storage], N.ARITH_EXACT if arith == "exact" else N.ARITH_FAST, int(arena_bytes),
                       int(max_domains))
        h = C.c_void_p()
        N.check(N.lib().vfb_pool_create(C.byref(d), C.byref(h)))
        self._h = h
        self.storage = storage
        self.real = np.float64 if storage == "f64" else np.float32
        self.max_domains = int(max_domains)
        self.domains = {}

    def close(self):
        if getattr(self, "_h", None):
            N.lib().vfb_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def desc(shape, omega, periodic=(True, True, True), forces=(0.0, 0.0, 0.0), limiters=(0.01, 0.01, 0.01)):
        d = N.DomainDesc()
        d.nx, d.ny, d.nz = (int(v) for v in shape)
        d.periodic_x, d.periodic_y, d.periodic_z = (int(bool(v)) for v in periodic)
        d.omega = float(omega)
        for i in range(3):
            d.forces[i] = float(forces[i])
            d.quadric_limiters[i] = float(limiters[i])
        return d

    def domain_bytes(self, shape, omega=1.8, periodic=(True, True, True), has_mask=False, bcs=None) -> int:
        """Arena bytes of a domain of this shape with these BC lists (as for add)."""
        b = C.c_uint64()
        st, keep = self._bcs(bcs)
        N.check(N.lib().vfb_pool_domain_bytes_with_bcs(self._h, C.byref(self.desc(shape, omega, periodic)),
                                                       int(has_mask), C.byref(st) if bcs else None, C.byref(b)))
        del keep
        return b.value

    @staticmethod
    def _bcs(bcs):
        """vfb_domain_bcs from {"noslip": (k, q27[27, n]), "pressure": (k, kN, drho, direction)} (host
        arrays); returns the struct and the arrays it points to."""
        out = N.DomainBCs()
        keep = []
        if bcs and "noslip" in bcs:
            k, q = bcs["noslip"]
            k = np.ascontiguousarray(k, dtype=np.int32).reshape(-1)
            q = np.ascontiguousarray(q, dtype=np.float64).reshape(27, k.size)
            keep += [k, q]
            out.noslip_variant = N.NOSLIP_INTERPOLATED_COMPRESSIBLE
            out.noslip_k, out.noslip_q27, out.number_of_noslip_nodes = k.ctypes.data, q.ctypes.data, k.size
        if bcs and "pressure" in bcs:
            k, kn, rho, direction = bcs["pressure"]
            k = np.ascontiguousarray(k, dtype=np.int32).reshape(-1)
            arrs = [k, np.ascontiguousarray(kn, dtype=np.int32).reshape(-1),
                    np.ascontiguousarray(np.broadcast_to(np.asarray(rho, dtype=np.float64), k.shape)),
                    np.ascontiguousarray(np.broadcast_to(np.asarray(direction, dtype=np.int32), k.shape))]
            keep += arrs
            out.pressure_variant = N.PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE
            out.pressure_k, out.pressure_k_neighbor, out.pressure_rho, out.pressure_direction = \
                (a.ctypes.data for a in arrs)
            out.number_of_pressure_nodes = k.size
        return out, keep

    def add(self, shape, omega, periodic=(True, True, True), forces=(0.0, 0.0, 0.0), mask=None, bcs=None) -> int:
        """Carve a domain; raises VfbError(VFB_ERR_OUT_OF_MEMORY) when the arena has no room. bcs:
        optional boundary-condition lists, {"noslip": (k, q27), "pressure": (k, k_neighbor, drho,
        direction)} in box node indices (NoSlipInterpolatedCompressible and
        PressureNonEquilibriumCompressible; drho and direction scalars or per node)."""
        d = self.desc(shape, omega, periodic, forces)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        i = C.c_uint32()
        b, keep = self._bcs(bcs)
        N.check(N.lib().vfb_pool_add_domain_with_bcs(self._h, C.byref(d), m.ctypes.data if m is not None else None,
                                                     C.byref(b) if bcs else None, C.byref(i)))
        del keep
        self.domains[i.value] = tuple(int(v) for v in shape)
        return i.value

    def try_add(self, *args, **kwargs):
        try:
            return self.add(*args, **kwargs)
        except N.VfbError as e:
            if e.status == N.VFB_ERR_OUT_OF_MEMORY:
                return None
            raise

    def remove(self, domain: int):
        N.check(N.lib().vfb_pool_remove_domain(self._h, int(domain)))
        self.domains.pop(domain, None)

    def synchronize(self, stream=None):
        N.check(N.lib().vfb_pool_synchronize(self._h, _stream_ptr(stream)))

    def init(self, domain: int, rho=None, ux=None, uy=None, uz=None, stream=None):
        """Equilibrium from host arrays (numpy) or device tensors (torch); None = zero."""
        shape = self.domains[domain]
        n = shape[0] * shape[1] * shape[2]
        arrs = [rho, ux, uy, uz]
        if any(a is not None and hasattr(a, "data_ptr") for a in arrs):
            import torch
            dt = torch.float64 if self.real == np.float64 else torch.float32
            dev = next(a.device for a in arrs if a is not None and hasattr(a, "data_ptr"))
            keep = [a.to(dt).contiguous() if a is not None else torch.zeros(n, dtype=dt, device=dev) for a in arrs]
            N.check(N.lib().vfb_pool_init_domain(self._h, int(domain), *(C.c_void_p(t.data_ptr()) for t in keep), 0,
                                                 _stream_ptr(stream)))
            return
        keep = [np.ascontiguousarray(a if a is not None else np.zeros(n), dtype=self.real).reshape(-1) for a in arrs]
        N.check(N.lib().vfb_pool_init_domain(self._h, int(domain), *(a.ctypes.data for a in keep), 1,
                                             _stream_ptr(stream)))

    def step(self, steps: int, stream=None):
        N.check(N.lib().vfb_pool_step(self._h, int(steps), _stream_ptr(stream)))

    def fields(self, domain: int, stream=None):
        """drho, ux, uy, uz of one domain as numpy arrays of shape (nz, ny, nx)."""
        shape = self.domains[domain]
        n = shape[0] * shape[1] * shape[2]
        out = [np.zeros(n, dtype=self.real) for _ in range(4)]
        N.check(N.lib().vfb_pool_domain_fields(self._h, int(domain), *(a.ctypes.data for a in out), 1,
                                               _stream_ptr(stream)))
        return [a.reshape(shape[2], shape[1], shape[0]) for a in out]

    def set_launch(self, threads=128, nodes_per_thread=8, blocks_per_sm=-1, use_graph=True):
        """threads per block (64, 128, 256), nodes per thread per work item (1..32), resident blocks per
        SM of the persistent launch (0: as many as fit; -1: one block per work item, no persistent
        loop), CUDA-graph replay. Results do not depend on the shape."""
        N.check(N.lib().vfb_pool_set_launch(self._h, int(threads), int(nodes_per_thread), int(blocks_per_sm),
                                            int(use_graph)))

    def launch(self):
        out = (C.c_int32 * 4)()
        N.check(N.lib().vfb_pool_get_launch(self._h, out))
        return {"threads": out[0], "nodes_per_thread": out[1], "blocks_per_sm": out[2], "use_graph": bool(out[3])}

    def autotune(self, trial_steps=10, stream=None) -> float:
        ms = C.c_double()
        N.check(N.lib().vfb_pool_autotune(self._h, int(trial_steps), _stream_ptr(stream), C.byref(ms)))
        return ms.value

    def stats(self):
        a, n, u, f = C.c_uint32(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        N.check(N.lib().vfb_pool_stats(self._h, C.byref(a), C.byref(n), C.byref(u), C.byref(f)))
        return {"active_domains": a.value, "active_nodes": n.value, "used_bytes": u.value, "free_bytes": f.value}

    def domain_mass(self, stream=None):
        """FP64 mass sum(1 + drho) of every domain id (0 for inactive ids), at the current state."""
        out = np.zeros(len(self._mass_ids()), dtype=np.float64)
        N.check(N.lib().vfb_pool_domain_mass(self._h, out.ctypes.data, _stream_ptr(stream)))
        return out

    def _mass_ids(self):
        return range(self.max_domains)

    def watchdog(self, max_relative_drift=0.5, stream=None):
        """Ids of the domains whose mass is non-finite or drifted beyond max_relative_drift from their
        mass at the first check after initialisation (vfb_pool_watchdog); [] when all are sound."""
        failed = np.zeros(self.max_domains, dtype=np.uint32)
        n = C.c_uint32()
        st = N.lib().vfb_pool_watchdog(self._h, float(max_relative_drift), failed.ctypes.data, failed.size, C.byref(n),
                                        _stream_ptr(stream))
        if st not in (N.VFB_OK, N.VFB_ERR_WATCHDOG):
            N.check(st)
        return [int(i) for i in failed[:n.value]]

    def kernel_launches(self) -> int:
        c = C.c_uint64()
        N.check(N.lib().vfb_pool_kernel_launches(self._h, C.byref(c)))
        return c.value
