"""Serving on the GPU: continuous batching of porous-block solves in one domain pool.

Requests of different sizes and step counts are admitted as memory frees up, advance together,
and leave when done; both drives are covered (pressure planes with exact sphere q, whose lists live
in the pool's arena, and the periodic body force). Each result must be the same alone and in the
mix (bit for bit: the pool's kernels treat every domain independently), and the FP16-storage
permeability must stay close to the FP64 one.
"""
import numpy as np
import pytest

from virtualfluids_b200.serving import Request, Server, poisson_stream, solve_alone

pytestmark = pytest.mark.gpu


def _small_stream(n=7, seed=5, drive="pressure"):
    reqs = poisson_stream(n, rate=1000.0, seed=seed, sides=(20, 40), steps=(100, 600), drive=drive)
    for r in reqs:
        r.geometry()
    return reqs


@pytest.mark.parametrize("drive", ["pressure", "force"])
def test_each_result_is_the_same_alone_and_in_the_mix(cuda, drive):
    reqs = _small_stream(drive=drive)
    # an arena that holds about three of these solves at a time, so later ones queue for memory
    per = max(r.side + 2 for r in reqs) ** 3 * (27 * 4 + 1 + 40) + 4096
    srv = Server(3 * per, storage="f32", keep_fields=True)
    results, stats = srv.run(reqs, realtime=False)
    srv.close()
    assert stats["peak_concurrent"] >= 2
    assert all(r.finished >= r.admitted >= 0 for r in results)
    for req, res in zip(reqs, results):
        perm, ux = solve_alone(req, storage="f32")
        assert np.array_equal(res.ux, ux), req.rid
        assert res.permeability == perm and perm > 0


def test_requests_arriving_during_others_are_admitted_before_those_finish(cuda):
    reqs = poisson_stream(6, rate=40.0, seed=11, sides=(24, 40), steps=(2000, 3000))
    for r in reqs:
        r.geometry()
    srv = Server(1 << 30, storage="f32")
    results, stats = srv.run(reqs, realtime=True)
    srv.close()
    overlapped = any(later.admitted < earlier.finished
                     for i, earlier in enumerate(results) for later in results[i + 1:])
    assert overlapped
    assert stats["p99_s"] >= stats["p50_s"] > 0 and stats["mlups"] > 0


@pytest.mark.parametrize("drive", ["pressure", "force"])
def test_fp16_storage_permeability_close_to_fp64(cuda, drive):
    req = Request(rid=0, arrival=0.0, side=40, steps=3000, seed=3, porosity=0.8, drive=drive)
    k64, _ = solve_alone(req, storage="f64")
    k16, _ = solve_alone(req, storage="f16")
    k32, _ = solve_alone(req, storage="f32")
    assert k64 > 0
    assert abs(k32 - k64) <= 1e-4 * k64
    assert abs(k16 - k64) <= 1e-2 * k64


def test_a_diverging_request_fails_alone(cuda):
    """A request whose initial state holds a NaN is stopped by the watchdog with status "watchdog";
    every other request completes with the result it has alone."""
    reqs = _small_stream(n=5, seed=9)
    bad = reqs[2]
    g = bad.geometry()
    n = int(np.prod(g["shape"]))
    ux = np.zeros(n, dtype=np.float32)
    fluid = np.nonzero(g["mask"])[0]
    ux[fluid[fluid.size // 2]] = np.nan          # a fluid node: solid nodes are never initialised
    bad.initial = (np.zeros(n, dtype=np.float32), ux, np.zeros(n, dtype=np.float32), np.zeros(n, dtype=np.float32))
    srv = Server(1 << 30, storage="f32", keep_fields=True)
    results, stats = srv.run(reqs, realtime=False)
    srv.close()
    assert stats["failed"] == 1
    for req, res in zip(reqs, results):
        if req is bad:
            assert res.status == "watchdog" and np.isnan(res.permeability)
            continue
        assert res.status == "ok"
        perm, ux_alone = solve_alone(req, storage="f32")
        assert np.array_equal(res.ux, ux_alone), req.rid
