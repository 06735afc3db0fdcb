"""The serving loop's scheduling on the host, against a stand-in pool: admission against the
budget, chunks that stop at the next completion, release of finished solves, and a request the
watchdog reports ends with status "watchdog" while the others complete (no GPU)."""
import numpy as np

from virtualfluids_b200.serving import Request, Server


class FakePool:
    """Holds domains by id and advances a step counter per domain; `poisoned` ids fail the watchdog."""

    def __init__(self, capacity_nodes):
        self.capacity = capacity_nodes
        self.used = 0
        self.domains = {}
        self.poisoned = set()
        self.launches = 0
        self.max_used = 0

    def try_add(self, shape, omega, periodic=None, forces=None, mask=None, bcs=None):
        n = int(np.prod(shape))
        if self.used + n > self.capacity:
            return None
        d = max(self.domains, default=-1) + 1
        self.domains[d] = {"n": n, "steps": 0, "init": None}
        self.used += n
        self.max_used = max(self.max_used, self.used)
        return d

    def init(self, d, rho, ux, uy, uz, stream=None):
        self.domains[d]["init"] = ux
        if np.isnan(np.asarray(ux)).any():
            self.poisoned.add(d)

    def step(self, steps, stream=None):
        for v in self.domains.values():
            v["steps"] += steps
        self.launches += steps

    def watchdog(self, max_relative_drift, stream=None):
        return sorted(d for d in self.poisoned if d in self.domains)

    def fields(self, d, stream=None):
        v = self.domains[d]
        return [np.full((1, 1, 1), float(v["steps"]))] * 4

    def remove(self, d):
        self.used -= self.domains.pop(d)["n"]
        self.poisoned.discard(d)

    def synchronize(self, stream=None):
        pass

    def kernel_launches(self):
        return self.launches

    def close(self):
        pass


class FakeStream:
    def synchronize(self):
        pass


def _req(rid, side, steps, poison=False):
    r = Request(rid=rid, arrival=0.0, side=side, steps=steps, seed=rid, porosity=0.8, drive="force")
    n = side ** 3
    ux = np.zeros(n, dtype=np.float32)
    if poison:
        ux[0] = np.nan
    r.initial = (np.zeros(n, dtype=np.float32), ux, np.zeros(n, dtype=np.float32), np.zeros(n, dtype=np.float32))
    return r


def test_scheduling_budget_completion_and_watchdog():
    reqs = [_req(0, 16, 300), _req(1, 16, 120), _req(2, 20, 200, poison=True), _req(3, 12, 50), _req(4, 16, 80)]
    pool = FakePool(capacity_nodes=2 * 16 ** 3 + 100)     # at most two of the larger solves at once
    srv = Server(0, pool=pool, stream=FakeStream())
    results, stats = srv.run(reqs, realtime=False)
    assert stats["failed"] == 1
    by = {r.rid: r for r in results}
    assert by[2].status == "watchdog" and np.isnan(by[2].permeability)
    for r in reqs:
        if r.rid == 2:
            continue
        assert by[r.rid].status == "ok"
        # a solve is read out exactly when its own step count is reached
        g = r.geometry()
        assert by[r.rid].permeability == r.nu * float(r.steps) / r.g
    assert pool.max_used <= pool.capacity and not pool.domains
