"""Serving: a request loop that runs many solves of different sizes and step counts on one GPU.

Continuous batching over a :class:`~virtualfluids_b200.pool.Pool`: every request becomes a domain
in the pool's device arena when it has arrived and its populations and mask fit (the HBM budget
is the arena size); all admitted solves advance together, one persistent launch per step, and a
solve leaves as soon as its own step count is reached, freeing its memory for waiting requests.
Populations and masks stay resident on the device between steps. A solve computes exactly what it
computes alone (the pool's kernels treat every domain independently), so its result does not
depend on what else is being served.

The porous-block workload: a cube of random non-overlapping spheres. Two drives:

* ``"pressure"`` (the default): the block lies between two pressure planes at x (drho = +-dp/2,
  PressureNonEquilibriumCompressible), periodic in y and z; every link cut by a sphere carries the
  exact q of its intersection (NoSlipInterpolatedCompressible). Both lists stay resident in the
  pool's arena with the populations. Darcy permeability k = nu <u_x> L / (dp / 3);
* ``"force"``: periodic on every axis, driven by the body force g equivalent to the pressure drop,
  the spheres as staircase solids (NoSlipDelayBounceBack); k = nu <u_x> / g.

<u_x> is the superficial velocity: the mean over the block's nodes, solid ones counting zero.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .pool import Pool
from .workloads import porous_block, porous_block_bcs


@dataclass
class Request:
    rid: int
    arrival: float              # seconds after the stream starts
    side: int
    steps: int
    seed: int
    porosity: float
    nu: float = 1.0 / 60.0
    g: float = 1e-6                   # body force of the "force" drive
    drho: float = 3e-3                # density drop across the block of the "pressure" drive
    drive: str = "pressure"
    geo: dict | None = field(default=None, repr=False)
    initial: tuple | None = field(default=None, repr=False)   # (drho, ux, uy, uz) host arrays; None = rest

    def geometry(self):
        """The request's domain (built on first use): shape, periodicity, mask, BC lists and the
        slice of the block's nodes along x."""
        if self.geo is None:
            if self.drive == "pressure":
                g = porous_block_bcs(self.side, self.seed, porosity=self.porosity, drho=self.drho)
                g.update(periodic=(False, True, True), forces=(0.0, 0.0, 0.0), block=slice(1, self.side + 1))
            else:
                mask, spheres, phi = porous_block(self.side, self.seed, porosity=self.porosity)
                g = {"shape": (self.side,) * 3, "mask": mask, "bcs": None, "spheres": spheres, "porosity": phi,
                     "periodic": (True, True, True), "forces": (self.g, 0.0, 0.0), "block": slice(0, self.side)}
            self.geo = g
        return self.geo

    @property
    def fluid_nodes(self) -> int:
        g = self.geometry()
        nx, ny, nz = g["shape"]
        return int(g["mask"].reshape(nz, ny, nx)[:, :, g["block"]].astype(bool).sum())

    def permeability(self, ux) -> float:
        """Darcy permeability from the velocity field (nz, ny, nx) of the domain."""
        g = self.geometry()
        mean = float(ux[:, :, g["block"]].astype(np.float64).mean())
        if self.drive == "pressure":
            return self.nu * mean * g["length"] / (g["drho"] / 3.0)
        return self.nu * mean / self.g


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    fluid_nodes: int
    permeability: float
    ux: np.ndarray | None = field(default=None, repr=False)
    status: str = "ok"                # "watchdog": stopped for non-finite populations or mass drift

    @property
    def time_to_solution(self) -> float:
        return self.finished - self.arrival


def poisson_stream(count, rate, seed=20261203, sides=(32, 192), steps=(1000, 20000), porosity=(0.5, 0.9),
                   drive="pressure"):
    """`count` porous-block requests with exponential inter-arrival times of mean 1 / rate seconds.
    A request carries its geometry (built by Request.geometry, before it is submitted)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        out.append(Request(rid=i, arrival=t, side=int(rng.integers(sides[0], sides[1] + 1)),
                           steps=int(rng.integers(steps[0], steps[1] + 1)), seed=int(rng.integers(1 << 31)),
                           porosity=float(rng.uniform(*porosity)), drive=drive))
    return out


def request_work(req: Request):
    """Node updates of a request (the block's nodes x steps)."""
    return req.side ** 3 * req.steps


class Server:
    """Continuous batching of porous-block solves in one domain pool.

    arena_bytes is the HBM budget of populations, masks and BC lists. Between two scheduling points
    (arrivals admitted, finished solves read out and released) the pool runs a chunk of steps sized
    to about chunk_ms of GPU time and never past the next completion, so admissions wait for at
    most one chunk while the GPU stays busy. After every chunk the pool's watchdog (FP64 mass per
    domain) stops any solve whose populations went non-finite or whose mass drifted by more than
    max_mass_drift: that request ends with status "watchdog", the others go on."""

    def __init__(self, arena_bytes, storage="f32", max_domains=1024, chunk_ms=40.0, stream=None, keep_fields=False,
                 max_mass_drift=0.5, pool=None):
        import torch
        self.pool = pool if pool is not None else Pool(arena_bytes, storage=storage, max_domains=max_domains)
        self.max_mass_drift = float(max_mass_drift)
        self.storage = storage
        self.chunk_ms = float(chunk_ms)
        self.stream = stream or torch.cuda.Stream()
        self.keep_fields = keep_fields
        self._zeros = None
        self.ns_per_node_step = 0.1     # running estimate of the pool's time per node update

    def close(self):
        self.pool.close()

    def _rest(self, n):
        import torch
        if self._zeros is None or self._zeros.numel() < n:
            self._zeros = torch.zeros(n, dtype=torch.float64 if self.storage == "f64" else torch.float32,
                                      device="cuda")
        return self._zeros[:n]

    def _try_admit(self, req):
        g = req.geometry()
        d = self.pool.try_add(g["shape"], 1.0 / (3.0 * req.nu + 0.5), periodic=g["periodic"], forces=g["forces"],
                              mask=g["mask"], bcs=g["bcs"])
        if d is None:
            return None
        if req.initial is not None:
            self.pool.init(d, *req.initial, stream=self.stream)
        else:
            z = self._rest(int(np.prod(g["shape"])))
            self.pool.init(d, z, z, z, z, stream=self.stream)
        return d

    def run(self, requests, realtime=True, clock=time.perf_counter):
        """Serve `requests` (arrival times in seconds from the start). With realtime a request is not
        admitted before its arrival time on the wall clock; otherwise arrivals are taken as past.
        Returns the results in request order and the loop's statistics."""
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting = []                   # arrived, not admitted (arrival order, smaller ones may pass)
        active = {}                    # domain -> [request, steps left, admitted time]
        results = {}
        t0 = clock()
        launches0 = self.pool.kernel_launches()
        peak_active = 0
        failed = 0
        while pending or waiting or active:
            now = clock() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                waiting.append(pending.pop(0))
            still = []
            for req in waiting:
                d = self._try_admit(req)
                if d is None:
                    still.append(req)
                else:
                    active[d] = [req, req.steps, clock() - t0]
            waiting = still
            peak_active = max(peak_active, len(active))
            if not active:
                if waiting:
                    # released memory becomes reusable once the stream has drained
                    self.pool.synchronize(self.stream)
                    d = self._try_admit(waiting[0])
                    if d is None:
                        raise N.VfbError(N.VFB_ERR_OUT_OF_MEMORY, "a request does not fit the whole arena")
                    req = waiting.pop(0)
                    active[d] = [req, req.steps, clock() - t0]
                elif pending and realtime:
                    time.sleep(max(0.0, min(0.002, pending[0].arrival - (clock() - t0))))
                    continue
                else:
                    continue
            nodes = sum(int(np.prod(v[0].geometry()["shape"])) for v in active.values())
            by_time = max(1, int(self.chunk_ms * 1e6 / (self.ns_per_node_step * nodes)))
            chunk = min(by_time, min(v[1] for v in active.values()))
            c0 = clock()
            self.pool.step(chunk, stream=self.stream)
            self.stream.synchronize()
            el = clock() - c0
            self.ns_per_node_step = 0.7 * self.ns_per_node_step + 0.3 * (el * 1e9 / (chunk * nodes))
            # the watchdog fails a diverging request, not the loop
            for d in self.pool.watchdog(self.max_mass_drift, stream=self.stream):
                req, _, adm = active.pop(d)
                results[req.rid] = Result(req.rid, req.arrival, adm, clock() - t0, req.steps, req.fluid_nodes,
                                          float("nan"), status="watchdog")
                self.pool.remove(d)
                failed += 1
            for d in [d for d, v in active.items() if v[1] == chunk]:
                req, _, adm = active.pop(d)
                rho, ux, uy, uz = self.pool.fields(d, stream=self.stream)
                results[req.rid] = Result(req.rid, req.arrival, adm, clock() - t0, req.steps, req.fluid_nodes,
                                          req.permeability(ux), ux.copy() if self.keep_fields else None)
                self.pool.remove(d)
            for v in active.values():
                v[1] -= chunk
        self.stream.synchronize()
        wall = clock() - t0
        tts = np.array([results[r.rid].time_to_solution for r in requests])
        fluid_updates = sum(results[r.rid].fluid_nodes * r.steps for r in requests if results[r.rid].status == "ok")
        stats = {"requests": len(requests), "wall_s": wall, "p50_s": float(np.quantile(tts, 0.5)),
                 "p99_s": float(np.quantile(tts, 0.99)), "mlups": fluid_updates / wall / 1e6,
                 "peak_concurrent": peak_active, "gpu_launches": self.pool.kernel_launches() - launches0,
                 "failed": failed}
        return [results[r.rid] for r in requests], stats


def solve_alone(req: Request, storage="f32", stream=None):
    """One request in a pool of its own (the reference result for the mix, and the FP64 run)."""
    import torch
    s = stream or torch.cuda.Stream()
    g = req.geometry()
    probe = Pool(1 << 20, storage=storage, max_domains=1)
    need = probe.domain_bytes(g["shape"], periodic=g["periodic"], has_mask=True, bcs=g["bcs"])
    probe.close()
    pool = Pool(need + (1 << 20), storage=storage, max_domains=1)
    d = pool.add(g["shape"], 1.0 / (3.0 * req.nu + 0.5), periodic=g["periodic"], forces=g["forces"], mask=g["mask"],
                 bcs=g["bcs"])
    pool.init(d, stream=s)
    pool.step(req.steps, stream=s)
    s.synchronize()
    rho, ux, uy, uz = pool.fields(d, stream=s)
    pool.close()
    return req.permeability(ux), ux
