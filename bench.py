"""Benchmark: D3Q27 K17 + esoteric-twist time step, Taylor-Green vortex 256^3 periodic, FP64.

One "step" is one LBM time step over the whole 256^3 box (16.78 M fluid nodes). Metric: MLUPS
(million fluid-node updates per second, whole job). The population array (3.62 GB in FP64) is
far larger than the 126 MB L2, so no L2 flush is needed between steps. The headline form is the
exact FP64 arithmetic (every operation rounded as the reference's host build rounds it, so the
result is the CPU reference's bit for bit); --arith fast times the FMA form instead.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank advances its own independent 256^3 box (replicas: the
single-domain hot path has no data-path collective), timing is max over ranks, value = all
ranks' node updates / that time ("scaling": "weak").

The JSON line also carries:
  roofline     : achieved HBM bytes/s of the collision kernel (432 B algorithmic per node update
                 in FP64: 27 reads + 27 writes of 8 B) over its CUDA-event launch time averaged
                 over 200 launches, against the measured copy bandwidth of MEASURED_PEAKS.json
  e2e          : the same metric through the public API with host buffers (pinned): initial
                 fields host->device, the steps with the per-step FP64 kinetic energy read back to
                 the host, final fields device->host, all inside the timed region
  forms        : the other arithmetic / storage forms (FMA FP64, FP32, FP16, BF16): MLUPS, kernel
                 roofline and velocity error against the exact FP64 run at the same step
  cpu_baseline : the reference's K17 header built with its Release flags (oracle/_ref), driven over
                 the same layout on this box's host cores, on this same 256^3 workload, and on
                 the 64^3 lid-driven cavity at Re 100 (2000 steps)
  parity       : the cavity run on the GPU in each FP64 form against that CPU run (relative L-inf
                 of drho and u)
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_SIDE = 256
U0 = 0.04
RE = 1600.0
BYTES_PER_NODE = {"f64": 432, "f32": 216, "f16": 108, "bf16": 108, "e3m12": 108}
# DRAM bytes (read + write) per node of one launch of the FP64 direct-load collision kernel of each
# arithmetic, from one ncu capture at 128^3 (2,097,152 nodes); traffic grows with the node count,
# so it is scaled to the bench's box
NCU_DRAM_BYTES_PER_NODE_F64 = {"fast": (453.033728e6 + 395.824384e6) / 2097152,
                               "exact": (453.048832e6 + 395.543040e6) / 2097152}
# launches averaged for the roofline figure, whatever --steps is (a sustained, not a burst, figure)
ROOFLINE_LAUNCHES = 200
# most timed steps of the reference arm (CPU, about 0.3 s per 256^3 step on 16 cores)
REFERENCE_MAX_STEPS = 60
METRIC = "MLUPS (TGV 256^3 D3Q27 K17, FP64)"


def tgv_fields(n, u0, dtype=np.float64):
    x = (np.arange(n) + 0.5) / n * 2 * np.pi - np.pi
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    rho = 3.0 * (u0 * u0 / 16.0) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    ux = u0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    uy = -u0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    return [a.reshape(-1).astype(dtype) for a in (rho, ux, uy, np.zeros_like(ux))]


def omega_tgv(n):
    nu = U0 * n / (2 * np.pi * RE)
    return 1.0 / (3.0 * nu + 0.5)


NOMINAL_HBM_GBS = 8000.0     # nominal B200 HBM3e bandwidth, the figure the 70 % FP64 target is quoted on


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() in ("active", "1")})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def max_over_ranks_of(x, pg, device):
    """The largest of every rank's x (each rank's device time; the job's time is the slowest rank)."""
    if not pg:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_mlups(units_per_rank, world, slowest_ms):
    """Replicas: every rank advances its own box, so the job's rate is all ranks' node updates over
    the slowest rank's time."""
    return units_per_rank * world / (slowest_ms / 1e3) / 1e6


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def tgv_config(n, world, arith, kernel):
    """The workload of the headline line (the reference arm reports the same one)."""
    return {"workload": f"Taylor-Green vortex {n}^3 periodic, u0={U0}, Re={int(RE)}, D3Q27 K17 cumulant + "
                        f"esoteric-twist streaming, FP64, per-step FP64 kinetic energy",
            "nodes_per_gpu": n ** 3, "omega": omega_tgv(n), "replicas": world, "arith": arith, "kernel": kernel,
            "l2": f"inputs larger than L2 ({27 * 8 * n ** 3 / 1e9:.2f} GB populations per GPU), no flush"}


def _reference_cpu():
    """The reference's K17 header for the host: the Release-flag build when present, else the
    parity build, else None (the oracle's restatement is then timed)."""
    from oracle import pyoracle
    rel = pyoracle.ref64_release()
    if rel is not None:
        return rel, "reference", "reference K17 header, Release flags -O3 -funroll-all-loops"
    par = pyoracle.ref64()
    if par is not None:
        return par, "reference", "reference K17 header, -O2 -ffp-contract=off"
    return None, "port", "oracle restatement of the K17 header, -O2 -ffp-contract=off"


def cpu_tgv(n, steps=None, seconds=None, threads=None, warmup=1):
    """The reference CPU path on TGV n^3 periodic: the reference's K17 header over the esoteric-twist
    layout, OpenMP over nodes on `threads` host cores, whole time steps. Either `steps` steps, or
    as many as fit in about `seconds`. Returns (MLUPS, steps, seconds, kind, build)."""
    from oracle import pyoracle
    from virtualfluids_b200.grid import ListGrid
    threads = threads or os.cpu_count()
    ref, kind, build = _reference_cpu()
    g = ListGrid(n, n, n, periodic=(True, True, True))
    lv = pyoracle.OracleLevel(g, omega=omega_tgv(n))
    lv.init(*(np.concatenate([[0.0], a]) for a in tgv_fields(n, U0)))
    lim = np.full(3, 0.01)
    zero = np.zeros(3)

    def sweep():
        ev = lv.is_even.value
        if ref is not None:
            ref.ref_collision_sweep_f64(pyoracle.ptr(lv.f), lv.n, *(pyoracle.ptr(a) for a in lv.nb),
                                        pyoracle.ptr(lv.fluid), lv.fluid.size, ev, lv.omega, pyoracle.ptr(lim), threads)
        else:
            pyoracle.lib().orc_collision(C.byref(lv.L), pyoracle.ptr(lv.fluid), lv.fluid.size, ev, lv.omega,
                                         pyoracle.ptr(lim), pyoracle.ptr(zero), 0, None, None, None, None, threads)
        lv.is_even.value = 1 - ev

    for _ in range(warmup):
        sweep()
    done, t0 = 0, time.perf_counter()
    while True:
        sweep()
        done += 1
        el = time.perf_counter() - t0
        if (steps is not None and done >= steps) or (steps is None and el >= seconds and done >= 3):
            break
    return g.fluid.size * done / el / 1e6, done, el, kind, build


def cavity_grid(n):
    """The lid-driven cavity: lid +z moving in +x, the other five sides halfway bounce-back walls."""
    from virtualfluids_b200.grid import ListGrid
    g = ListGrid(n, n, n)
    for side in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(side, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    return g


def cpu_cavity(threads=None, steps=2000):
    """The lid-driven cavity on the CPU: 64^3, Re 100, FP64, 2000 steps; the collision by the reference's
    K17 header, the bounce-back BCs by the oracle's restatement of the GPU BC kernels (the reference
    has no host form of them). Returns the timing and the final fields."""
    from oracle import pyoracle
    threads = threads or os.cpu_count()
    ref, kind, build = _reference_cpu()
    n = 64
    g = cavity_grid(n)
    lv = pyoracle.OracleLevel(g, omega=1.0 / (3.0 * (0.05 * n / 100.0) + 0.5))
    lv.init()
    t0 = time.perf_counter()
    if ref is not None:
        lv.run_reference_collision(ref, steps, threads=threads)
    else:
        lv.run(steps, threads=threads)
    el = time.perf_counter() - t0
    return {"mlups": round(g.fluid.size * steps / el / 1e6, 2), "steps": steps, "seconds": round(el, 2),
            "kind": kind, "build": build}, (g, lv.omega, lv.macroscopic())


def cpu_baseline(n, threads=None, seconds=12.0):
    """cpu_baseline of the headline line: the reference CPU path on this same TGV n^3 workload (as
    many whole steps as fit in about `seconds` on all host cores), plus the 64^3 cavity's 2000 steps."""
    threads = threads or os.cpu_count()
    mlups, steps, el, kind, build = cpu_tgv(n, seconds=seconds, threads=threads)
    cav, cav_fields = cpu_cavity(threads)
    return {"value": round(mlups, 2), "unit": "MLUPS", "cores": threads, "kind": kind,
            "sample": f"{steps} whole steps of the same TGV {n}^3 periodic box ({build}, esoteric-twist layout, "
                      f"OpenMP over nodes), {el:.1f} s",
            "same_config": True, "cavity_64_2000_steps": cav, "_cavity_fields": cav_fields}


def cavity_parity(cpu, dev):
    """The 64^3 cavity (Re 100, 2000 steps) on the GPU through the drop-in step driver (the reference layout), in each FP64
    form, against the CPU run: relative L-inf of drho and of each velocity component over the
    fluid nodes."""
    import virtualfluids_b200 as vfb
    from virtualfluids_b200 import _native as N
    g, omega, want = cpu
    fl = g.geo == N.GEO_FLUID
    out = {"workload": "64^3 lid-driven cavity, lid u = 0.05, Re 100, bounce-back walls and lid, FP64, 2000 steps",
           "against": "cpu_baseline.cavity_64_2000_steps (reference K17 header + oracle BCs on the host)"}
    for arith in ("exact", "fast"):
        p = vfb.Parameter()
        p.set_viscosity_lb((1.0 / omega - 0.5) / 3.0)
        p.configure_main_kernel("K17CompressibleNavierStokes")
        p.storage, p.arith = N.STORAGE_F64, (N.ARITH_EXACT if arith == "exact" else N.ARITH_FAST)
        bcf = vfb.BoundaryConditionFactory()
        bcf.set_no_slip_boundary_condition(bcf.NoSlipBC.NoSlipBounceBack)
        bcf.set_velocity_boundary_condition(bcf.VelocityBC.VelocityBounceBack)
        sim = vfb.Simulation(p, g, bcf, device=dev)
        sim.init()
        sim.set_graph(16)                 # the step loop replayed from a CUDA graph (same bits)
        import torch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.run(2000)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        got = sim.macroscopic()
        sim.close()
        err = {k: float(np.abs(got[k][fl] - want[k][fl]).max() / np.abs(want[k][fl]).max())
               for k in ("rho", "vx", "vy", "vz")}
        out["f64_" + arith] = {"rel_linf": err, "max_rel_linf": max(err.values()),
                               "within_1e-12": bool(max(err.values()) <= 1e-12),
                               "gpu_ms_per_step": round(el / 2000 * 1e3, 4),
                               "gpu_mlups": round(int(fl.sum()) * 2000 / el / 1e6, 1)}
    return out


def reference_gpu_kernel(n, launches=ROOFLINE_LAUNCHES):
    """The reference's own GPU collision, runCollision with the K17 functor (K17CompressibleNavierStokes.cu
    :85-100), compiled from its sources with its own CUDA flags (FMA contraction on), 64 threads per
    block (Parameter.cpp:400), over TGV n^3 in the reference layout on this GPU: the average CUDA-event
    time of `launches` launches (alternating parity), FP64 and FP32. None without a GPU or the builds."""
    import torch
    from oracle import pyoracle
    from virtualfluids_b200.grid import ListGrid
    if not torch.cuda.is_available():
        return None
    g = ListGrid(n, n, n, periodic=(True, True, True))
    ptr = lambda t: C.c_void_p(t.data_ptr())
    nb = [torch.from_numpy(g.neighbor[a].astype(np.int32)).cuda() for a in range(3)]
    fluid = torch.from_numpy(g.fluid.astype(np.int32)).cuda()
    geo = torch.from_numpy(g.geo.astype(np.int32)).cuda()
    fields = [np.concatenate([[0.0], a]) for a in tgv_fields(n, U0)]
    peak, _ = measured_peak()
    omega = omega_tgv(n)
    out = {"kernel": "vf::gpu::runCollision<K17, TurbulenceModel::None> (reference sources, nvcc -O3 "
                     "--extended-lambda, default FMA contraction), 64 threads per block",
           "workload": f"TGV {n}^3 periodic, reference layout (neighborX/Y/Z, fluid-node list)",
           "launches_timed": launches}
    for rb, dt, key in ((8, torch.float64, "f64"), (4, torch.float32, "f32")):
        L = pyoracle.refgpu(rb, release=True)
        if L is None:
            continue
        dist = torch.zeros(27 * g.number_of_nodes, dtype=dt, device="cuda")
        arrs = [torch.from_numpy(a).to("cuda", dt) for a in fields]
        for ev in (0, 1):
            assert L.refgpu_init(*(ptr(x) for x in nb), ptr(geo), *(ptr(a) for a in arrs), g.number_of_nodes,
                                 ptr(dist), ev) == 0
        forces = torch.zeros(3, dtype=dt, device="cuda")
        lim = torch.full((3,), 0.01, dtype=dt, device="cuda")
        ev = 1

        def launch():
            nonlocal ev
            assert L.refgpu_k17(ptr(dist), g.number_of_nodes, *(ptr(x) for x in nb), ptr(fluid), int(g.fluid.size),
                                ev, omega, ptr(forces), ptr(lim), 1.0) == 0
            ev = 1 - ev

        for _ in range(5):
            launch()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(launches):
            launch()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / launches
        gbs = 2 * 27 * rb * g.fluid.size / (ms / 1e3) / 1e9
        out[key] = {"kernel_ms": round(ms, 4), "mlups": round(g.fluid.size / (ms / 1e3) / 1e6, 1),
                    "hbm_gbs_algorithmic": round(gbs, 1), "frac": round(gbs / peak, 4)}
        del dist, arrs
        torch.cuda.empty_cache()
    return out


def run_reference(args):
    """The reference arm: the reference's CPU path (its K17 header, Release flags, over the same
    esoteric-twist layout, all host cores) on the headline's own workload, TGV 256^3 FP64: W whole
    untimed steps, then min(K, REFERENCE_MAX_STEPS) timed steps. Rank 0 only. Beside it, the
    reference's own GPU collision kernel on the same workload (reference_gpu_kernel)."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count()
    steps = max(1, min(args.steps, REFERENCE_MAX_STEPS))
    mlups, done, el, kind, build = cpu_tgv(args.n, steps=steps, threads=threads, warmup=min(args.warmup, 3))
    cb = {"value": round(mlups, 2), "unit": "MLUPS", "cores": threads, "kind": kind,
          "sample": f"{done} timed whole steps (after {min(args.warmup, 3)} untimed) of TGV {args.n}^3 periodic "
                    f"({build}, esoteric-twist layout, OpenMP over nodes), {el:.1f} s"}
    line = {"metric": METRIC, "value": cb["value"], "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(el / done * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": tgv_config(args.n, 1, "exact", "auto"),
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_gpu_reference:
        try:
            gk = reference_gpu_kernel(args.n)
        except (AssertionError, RuntimeError, OSError) as e:   # reported, never fatal for the CPU arm
            gk = {"unavailable": f"{type(e).__name__}: {e}"}
        if gk:
            line["reference_gpu_kernel"] = gk
    print(json.dumps(line), flush=True)


def run_batch(args):
    """Batch of rectangular-duct Poiseuille domains of uneven sizes in one domain pool, advanced by
    one collision launch per step (CUDA-graph replay, autotuned launch shape), FP32 and FP16
    storage. With --check-steps S > 0 every domain also runs S steps in FP64, FP32 and FP16 and its
    x-averaged profile is compared with the analytic start-up series and with the FP64 run."""
    import torch

    from virtualfluids_b200 import Pool
    from virtualfluids_b200.workloads import duct_batch, duct_transient

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    specs = duct_batch(args.domains, seed=20261203 + rank)
    fluid = sum(d["fluid_nodes"] for d in specs)

    def build(storage):
        probe = Pool(1 << 20, storage=storage, max_domains=1)
        need = sum(probe.domain_bytes(d["shape"], d["omega"], periodic=(True, False, False), has_mask=True)
                   for d in specs)
        probe.close()
        pool = Pool(need + (1 << 20), storage=storage, max_domains=len(specs))
        ids = []
        for d in specs:
            i = pool.add(d["shape"], d["omega"], periodic=(True, False, False), forces=(d["g"], 0.0, 0.0))
            pool.init(i, stream=stream)
            ids.append(i)
        return pool, ids

    forms = {}
    for storage in ("f32", "f16"):
        pool, ids = build(storage)
        tuned = pool.autotune(trial_steps=3, stream=stream)
        pool.step(args.warmup, stream=stream)
        stream.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = pool.kernel_launches()
        with ClockSampler(local) as clk:
            ev0.record(stream)
            pool.step(args.steps, stream=stream)
            ev1.record(stream)
            stream.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
        forms[storage] = {"mlups": round(fluid / (ms / 1e3) / 1e6, 1), "ms_per_step": round(ms, 4),
                          "hbm_gbs_algorithmic": round(BYTES_PER_NODE[storage] * fluid / (ms / 1e3) / 1e9, 1),
                          "launch": pool.launch(), "autotune_ms_per_step": round(tuned, 4),
                          "gpu_launches": pool.kernel_launches() - l0, "clocks": clk.summary()}
        pool.close()
        del pool
        torch.cuda.empty_cache()
    check = None
    if args.check_steps > 0:
        prof = {}
        for storage in ("f64", "f32", "f16"):
            pool, ids = build(storage)
            pool.step(args.check_steps, stream=stream)
            stream.synchronize()
            prof[storage] = [pool.fields(i, stream=stream)[1].mean(axis=2)[1:-1, 1:-1].astype(np.float64) for i in ids]
            pool.close()
            del pool
            torch.cuda.empty_cache()
        ana, e32, e16 = [], [], []
        for k, d in enumerate(specs):
            ref = duct_transient(d["shape"][1], d["shape"][2], d["g"], d["nu"], args.check_steps, terms=31)[1:-1, 1:-1]
            u64 = prof["f64"][k]
            nrm = np.sqrt((u64 ** 2).sum())
            ana.append(np.sqrt(((u64 - ref) ** 2).sum()) / np.sqrt((ref ** 2).sum()))
            e32.append(np.sqrt(((prof["f32"][k] - u64) ** 2).sum()) / nrm)
            e16.append(np.sqrt(((prof["f16"][k] - u64) ** 2).sum()) / nrm)
        q = lambda v: {"median": float(np.median(v)), "p99": float(np.quantile(v, 0.99)), "max": float(np.max(v))}
        check = {"steps": args.check_steps, "fp64_vs_analytic_rel_l2": q(ana), "fp32_vs_fp64_rel_l2": q(e32),
                 "fp16_vs_fp64_rel_l2": q(e16)}
    if rank == 0:
        line = {"metric": "MLUPS (4096 rectangular ducts, one domain pool, FP32 storage)",
                "value": forms["f32"]["mlups"], "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": forms["f32"]["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"{args.domains} ducts, sides log-uniform in [16, 96], periodic x, walls y/z, "
                                       "body force for u_max 0.03, Re uniform in [max(10, 42 u_max H), 500]",
                           "domains": args.domains, "fluid_nodes": fluid,
                           "l2": "inputs larger than L2, no flush"},
                "forms": forms, "gpu_launches": forms["f32"]["gpu_launches"]}
        if check:
            line["check"] = check
        print(json.dumps(line), flush=True)


def run_pool_shapes(args):
    """The pool kernel against the box kernel on the same node counts: one pool each for one
    periodic 256^3 domain, 64 periodic 64^3 domains, the shapes of 1024 ducts with every node
    fluid, and the same ducts with their walls; then a Box of 256^3. FP32 and FP16 storage, the
    pool's default launch shape (one block of 128 threads x 8 nodes per work item),
    graph replay, CUDA events on the pool's stream. MLUPS count fluid nodes."""
    import torch

    import virtualfluids_b200 as vfb
    from virtualfluids_b200 import Pool
    from virtualfluids_b200.workloads import duct_batch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()

    def duct_mask(nx, ny, nz):
        m = np.ones((nz, ny, nx), dtype=np.uint8)
        m[0] = m[-1] = 0
        m[:, 0] = m[:, -1] = 0
        return m.reshape(-1)

    def time_pool(shapes, walls, storage):
        periodic = (True, False, False) if walls else (True, True, True)
        probe = Pool(1 << 20, storage=storage, max_domains=1)
        need = sum(probe.domain_bytes(s, 1.8, periodic=periodic, has_mask=walls) for s in shapes)
        probe.close()
        pool = Pool(need + (1 << 20), storage=storage, max_domains=len(shapes))
        for s in shapes:
            i = pool.add(s, 1.8, periodic=periodic, mask=duct_mask(*s) if walls else None)
            pool.init(i, stream=stream)
        pool.set_launch(128, 8, -1, True)           # the default shape of a new pool
        pool.step(args.warmup, stream=stream)
        stream.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        pool.step(args.steps, stream=stream)
        ev1.record(stream)
        stream.synchronize()
        pool.close()
        return ev0.elapsed_time(ev1) / args.steps

    specs = duct_batch(1024)
    ducts = [d["shape"] for d in specs]
    cases = [("one periodic 256^3 domain", [(256, 256, 256)], False, 256 ** 3),
             ("64 periodic 64^3 domains", [(64, 64, 64)] * 64, False, 64 * 64 ** 3),
             ("1024 duct shapes, every node fluid", ducts, False, int(sum(np.prod(s) for s in ducts))),
             ("1024 ducts with walls", ducts, True, int(sum(d["fluid_nodes"] for d in specs)))]
    out = {}
    for storage in ("f32", "f16"):
        res = {}
        for name, shapes, walls, fluid in cases:
            ms = time_pool(shapes, walls, storage)
            res["pool: " + name] = {"ms_per_step": round(ms, 4), "mlups": round(fluid / (ms / 1e3) / 1e6, 1)}
        n = 256
        sp = C.c_void_p(stream.cuda_stream)
        b = vfb.Box(n, n, n, 1.8, storage=storage)
        z = torch.zeros(n ** 3, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        b.init(z, z, z, z, stream=sp)
        b.step(args.warmup, stream=sp)
        stream.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        b.step(args.steps, stream=sp)
        ev1.record(stream)
        stream.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
        res["box 256^3"] = {"ms_per_step": round(ms, 4), "mlups": round(n ** 3 / (ms / 1e3) / 1e6, 1)}
        del b
        torch.cuda.empty_cache()
        out[storage] = res
    if rank == 0:
        line = {"metric": "MLUPS of the pool kernel on one 256^3 domain (FP32 storage)",
                "value": out["f32"]["pool: one periodic 256^3 domain"]["mlups"], "unit": "MLUPS",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": out["f32"]["pool: one periodic 256^3 domain"]["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": "pool kernel vs box kernel on the same shapes, fluid at rest, omega 1.8",
                           "l2": "inputs larger than L2, no flush"},
                "forms": out}
        print(json.dumps(line), flush=True)


def run_tgv_slab(args):
    """The headline's TGV 256^3 box as ONE domain split into z slabs over the ranks (one process per
    GPU): every step collides each slab's two border planes, exchanges the border planes with the
    neighbouring ranks by NCCL point-to-point transfers straight out of and into the population
    arrays on a second stream, collides the interior planes meanwhile, and toggles the parity.
    Total work is fixed as N grows ("scaling": "strong"); with one rank the slab's ghost plane wraps
    onto itself by a device copy."""
    import datetime

    import torch
    import torch.distributed as dist

    from virtualfluids_b200.slab import DistPeerTransport, DistTransport, Slab, slab_bounds, step

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    n = args.n
    z0, nzl = slab_bounds(n, world, rank)
    omega = omega_tgv(n)
    fields = tgv_fields(n, U0)
    planes = n * n
    s = Slab(n, n, n, z0, nzl, omega, storage="f64", arith=args.arith)
    s.init(*(a[z0 * planes:(z0 + nzl) * planes] for a in fields))
    tr = DistPeerTransport(s) if args.slab_transport == "fused" else DistTransport(s)
    compute, comm = torch.cuda.Stream(), torch.cuda.Stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    with torch.cuda.stream(compute):
        for _ in range(args.warmup):
            step([s], tr, compute=compute, comm=comm)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(compute):
            e0.record(compute)
            for _ in range(args.steps):
                step([s], tr, compute=compute, comm=comm)
            e1.record(compute)
        torch.cuda.synchronize()
    t_ms = max_over_ranks_of(e0.elapsed_time(e1), dist if world > 1 else None, torch.device("cuda", local))
    f = s.fields()
    finite = bool(np.all(np.isfinite(f["vx"])))
    if hasattr(tr, "close"):
        tr.close()
    s.close()
    if rank == 0:
        mlups = n ** 3 * args.steps / (t_ms / 1e3) / 1e6
        peak, peak_src = measured_peak()
        gbs = BYTES_PER_NODE["f64"] * n ** 3 * args.steps / (t_ms / 1e3) / 1e9
        line = {"metric": f"MLUPS (TGV {n}^3 as one domain in z slabs over the GPUs, FP64)", "value": round(mlups, 1),
                "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(t_ms / args.steps, 4), "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"Taylor-Green vortex {n}^3 periodic, {world} slab(s) of {nzl} planes, "
                                       "border-first collision on a second stream, halo exchange "
                                       + ("fused into the border planes' stores (peer writes over NVLink, one "
                                          "NCCL all-reduce as the step barrier)" if args.slab_transport == "fused"
                                          else "by NCCL point-to-point transfers of 2 x 9 direction planes"),
                           "arith": args.arith, "transport": args.slab_transport,
                           "halo_bytes_per_step_per_rank": 2 * 9 * planes * 8 * 2,
                           "l2": "inputs larger than L2, no flush"},
                "hbm_gbs_algorithmic": round(gbs / world, 1), "frac_per_gpu": round(gbs / world / peak, 4),
                "peak_source": peak_src, "finite": finite, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_cube(args):
    """Duct flow past a wall-mounted cube (512 x 256 x 256 fluid nodes, FP32 storage) on a
    structured box with the reference layout's BC lists: interpolated no-slip walls, interpolated
    velocity inlet (parabolic, seeded +-1 % per node and step), non-equilibrium pressure outlet,
    interpolated bounce-back on the cube with the FP64 drag/lift every step."""
    import torch

    from virtualfluids_b200 import Box
    from virtualfluids_b200 import BoundaryConditionFactory as BCF
    from virtualfluids_b200.workloads import cube_duct

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    g, omega, meta = cube_duct(*args.cube_dims)
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    bcf.set_pressure_boundary_condition(BCF.PressureBC.PressureNonEquilibriumCompressible)
    bcf.set_geometry_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
    box = Box.from_grid(g, omega, bcf, storage="f32")
    setup_s = time.perf_counter() - t0
    Dx, Dy, Dz = g.dims
    zero = torch.zeros(Dx * Dy * Dz, dtype=torch.float32, device="cuda")
    box.init(zero, zero, zero, zero)
    box.set_velocity_perturbation(20261203, 0.01)
    box.enable_drag_lift(history_steps=args.warmup + args.steps)
    fluid = int(g.fluid.size)
    box.step(args.warmup)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = box.kernel_launches()
    with ClockSampler(local) as clk:
        ev0.record()
        box.step(args.steps)
        ev1.record()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    launches = box.kernel_launches() - l0
    hist = box.drag_lift_history()
    tail = hist[-min(1000, len(hist)):]
    fx = float(tail[:, 0].mean())
    cd = 2.0 * fx / (meta["u_max"] ** 2 * meta["area"])
    if rank == 0:
        line = {"metric": "MLUPS (duct past a wall-mounted cube, 512x256x256, FP32)",
                "value": round(fluid / (ms / 1e3) / 1e6, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "duct past a wall-mounted cube: cube 32^3 on the z = 0 wall at x = 128, parabolic inlet u_max 0.05 "
                                       "+-1 % per node and step (Philox), pressure outlet, Re 3000 on the cube height",
                           "fluid_nodes": fluid, "box": [Dx, Dy, Dz], "omega": omega, "setup_s": round(setup_s, 2),
                           "l2": "inputs larger than L2, no flush"},
                "drag": {"force_x_mean_last_steps": fx, "force_z_mean_last_steps": float(tail[:, 2].mean()),
                         "cd_from_u_max": cd, "steps_averaged": int(len(tail)), "dtype": "f64"},
                "hbm_gbs_algorithmic": round(BYTES_PER_NODE["f32"] * fluid / (ms / 1e3) / 1e9, 1),
                "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)


def run_tgv_forms(args):
    """Storage-form accuracy: the 256^3 Taylor-Green vortex for --form-steps steps in FP64, FP32, FP16
    and BF16 storage (FMA arithmetic), the FP64 kinetic-energy decay every 10 steps, and the L2 /
    L-inf velocity error of each form against the FP64 run at steps 1000, 5000 and 10000 (relative
    to the FP64 field's RMS / maximum speed)."""
    import torch

    import virtualfluids_b200 as vfb

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    fields = tgv_fields(n, U0)
    checkpoints = [c for c in (1000, 5000, 10000) if c <= args.form_steps]
    every = 100
    ref = {}
    out = {}
    names = args.tgv_forms.split(",")
    if not names[0].startswith("f64"):
        raise SystemExit("--tgv-forms: the first form is the FP64 reference (f64 or f64:exact)")
    for name in names:
        st, _, ar = name.partition(":")
        dt = torch.float64 if st == "f64" else torch.float32
        box = vfb.Box(n, n, n, omega_tgv(n), storage=st, arith=ar or "fast")
        box.init(*(torch.from_numpy(a).to(dev, dt) for a in fields))
        done, ek, errs = 0, [], {}
        t0 = time.perf_counter()
        for c in checkpoints:
            while done < c:
                k = min(every, c - done)
                e = np.zeros((k, 2))
                box.step(k, energy=e)
                # the kinetic energy after every 10th step (the FP64 sum of every step is computed)
                ek.extend(float(e[i, 1]) for i in range(k) if (done + i + 1) % 10 == 0)
                done += k
            f = box.fields()
            u = np.stack([f["vx"], f["vy"], f["vz"]]).astype(np.float64)
            if name == names[0]:
                ref[c] = u
            else:
                d = u - ref[c]
                rms = np.sqrt((ref[c] ** 2).sum(axis=0).mean())
                errs[c] = {"l2_rel": float(np.sqrt((d ** 2).sum(axis=0).mean()) / rms),
                           "linf_rel": float(np.sqrt((d ** 2).sum(axis=0)).max() / np.sqrt((ref[c] ** 2).sum(axis=0)).max())}
        out[name] = {"wall_s": round(time.perf_counter() - t0, 2), "kinetic_energy_every_10_steps": ek}
        if errs:
            out[name]["velocity_error_vs_fp64"] = errs
        del box
        torch.cuda.empty_cache()
    if rank == 0:
        line = {"metric": "TGV 256^3 kinetic-energy decay and velocity error of the storage forms against FP64",
                "value": out.get("f16", {}).get("velocity_error_vs_fp64", {}).get(checkpoints[-1], {}).get("l2_rel"),
                "unit": "relative L2 velocity error (FP16 storage, last checkpoint)", "n_gpus": world,
                "steps": args.form_steps, "warmup": 0, "ms_per_step": None, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32/f16/bf16", "data": "synthetic",
                "config": {"workload": f"Taylor-Green vortex {n}^3, u0={U0}, Re={int(RE)}", "checkpoints": checkpoints},
                "forms": out}
        print(json.dumps(line), flush=True)


def run_list_path(args, n, omega, fields, dev):
    """The same TGV through the drop-in path: vfb_simulation_run over the reference's layout (node
    list with the dummy node 0, neighborX/Y/Z, planes of number_of_nodes elements), FP64. Reports
    MLUPS and the collision kernel's algorithmic HBM throughput (CUDA events on the launching
    stream; the driver's step is the collision kernel alone on a periodic box)."""
    import torch

    import virtualfluids_b200 as vfb
    from virtualfluids_b200 import _native as N

    out = {"path": "vfb_simulation_run (K17CompressibleNavierStokes over neighborX/Y/Z with neighbour slot tables)",
           "kernel": "k17_box_kernel<double> over the reference layout where the level is a regular periodic box "
                     "(box_addressing), else k17_list_kernel<double>"}
    peak, peak_kind = measured_peak()
    out["peak_source"] = peak_kind
    # node numbering as the reference's grid builder (first node 1, planes of n^3 + 1 nodes), and
    # aligned (first node 32, planes padded to 32 nodes)
    runs = [(1, "reference_numbering", args.arith), (32, "aligned_numbering", args.arith)]
    if args.arith == "exact":
        runs.append((32, "fma_aligned_numbering", "fast"))     # the FMA form of the same path, beside it
    for align, key, arith in runs:
        g = vfb.ListGrid(n, n, n, periodic=(True, True, True), align=align)
        p = vfb.Parameter()
        p.set_viscosity_lb((1.0 / omega - 0.5) / 3.0)
        p.configure_main_kernel("K17CompressibleNavierStokes")
        p.storage, p.arith = N.STORAGE_F64, N.ARITH_EXACT if arith == "exact" else N.ARITH_FAST
        sim = vfb.Simulation(p, g, vfb.BoundaryConditionFactory())
        box_addr = C.c_int32()
        N.check(N.lib().vfb_simulation_level_box_addressing(sim._sim, 0, C.byref(box_addr)))
        full = [np.zeros(g.number_of_nodes) for _ in range(4)]
        for dst, a in zip(full, fields):
            dst[g.first_node:g.first_node + nodes_of(n)] = a
        sim.init(*full)
        sim.run(args.warmup)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        steps = max(args.steps, 1)
        ev0.record()
        sim.run(steps)           # the legacy stream, as the reference's default
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        nodes = int(g.fluid.size)
        achieved = BYTES_PER_NODE["f64"] * nodes / (ms / 1e3) / 1e9
        sim.close()
        del sim
        torch.cuda.empty_cache()
        out[key] = {"mlups": round(nodes / (ms / 1e3) / 1e6, 1), "ms_per_step": round(ms, 4),
                    "hbm_achieved_gbs": round(achieved, 1), "frac": round(achieved / peak, 4),
                    "box_addressing": bool(box_addr.value)}
    return out


def nodes_of(n):
    return n * n * n


def run_porous(args):
    """The serving pool's step without arrivals: porous blocks (cube sides --porous-sides, porosity
    0.75, exact-q spheres, pressure planes along x) resident in one domain pool and advanced
    together, FP32 and FP16 storage. The same blocks are also timed with the spheres as staircase
    solids and no BC lists (body-force drive), which isolates the cost of the lists. Algorithmic
    bytes per step: collision 2 x 27 values per fluid node + the node mask; no-slip list 27 gathered
    values, 26 q and the node index and guard word per BC node + one value per cut link; pressure
    planes 27 gathered + 18 written values and 16 bytes of row data per node."""
    import torch

    from virtualfluids_b200 import Pool
    from virtualfluids_b200.workloads import porous_block_bcs

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    geos = [porous_block_bcs(s, 20261203 + 7 * rank + i, porosity=0.75) for i, s in enumerate(args.porous_sides)]
    fluid = sum(int(np.count_nonzero(g["mask"])) for g in geos)
    box_nodes = sum(int(np.prod(g["shape"])) for g in geos)
    n_bc = sum(int(g["bcs"]["noslip"][0].size) for g in geos)
    cut = sum(int(((g["bcs"]["noslip"][1][1:] >= 0) & (g["bcs"]["noslip"][1][1:] <= 1)).sum()) for g in geos)
    n_pr = sum(int(g["bcs"]["pressure"][0].size) for g in geos)
    peak, peak_src = measured_peak()
    omega = 1.0 / (3.0 / 60.0 + 0.5)
    out = {}
    for storage in ("f32", "f16"):
        rs = 4 if storage == "f32" else 2
        parts = {"collision": 2 * 27 * rs * fluid + box_nodes,
                 "noslip": n_bc * (27 * rs + 26 * 4 + 8) + cut * rs,
                 "pressure": n_pr * (45 * rs + 16)}
        res = {}
        for lists in (True, False):
            probe = Pool(1 << 20, storage=storage, max_domains=1)
            need = sum(probe.domain_bytes(g["shape"], omega, periodic=(False, True, True), has_mask=True,
                                          bcs=g["bcs"] if lists else None) for g in geos)
            probe.close()
            pool = Pool(need + (1 << 20), storage=storage, max_domains=len(geos))
            for g in geos:
                d = pool.add(g["shape"], omega, periodic=(False, True, True) if lists else (True, True, True),
                             forces=(0.0, 0.0, 0.0) if lists else (1e-6, 0.0, 0.0), mask=g["mask"],
                             bcs=g["bcs"] if lists else None)
                pool.init(d, stream=stream)
            pool.step(args.warmup, stream=stream)
            stream.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = pool.kernel_launches()
            with ClockSampler(local) as clk:
                ev0.record(stream)
                pool.step(args.steps, stream=stream)
                ev1.record(stream)
                stream.synchronize()
            ms = ev0.elapsed_time(ev1) / args.steps
            launches = pool.kernel_launches() - l0
            pool.close()
            del pool
            torch.cuda.empty_cache()
            nbytes = sum(parts.values()) if lists else parts["collision"]
            res["lists" if lists else "staircase"] = {
                "ms_per_step": round(ms, 4), "mlups": round(fluid / (ms / 1e3) / 1e6, 1),
                "algorithmic_bytes_per_step": nbytes, "achieved_gbs": round(nbytes / (ms / 1e3) / 1e9, 1),
                "frac": round(nbytes / (ms / 1e3) / 1e9 / peak, 4), "gpu_launches": launches, "clocks": clk.summary()}
        res["list_share_of_step"] = round(1.0 - res["staircase"]["ms_per_step"] / res["lists"]["ms_per_step"], 3)
        res["bytes_by_part"] = parts
        out[storage] = res
    if rank == 0:
        f32 = out["f32"]["lists"]
        line = {"metric": "MLUPS (porous-block pool step with exact-q no-slip and pressure lists, FP32)",
                "value": f32["mlups"], "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": f32["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": "porous blocks of the serving stream resident in one pool, no arrivals",
                           "sides": list(args.porous_sides), "porosity": 0.75, "fluid_nodes": fluid,
                           "box_nodes": box_nodes, "noslip_nodes": n_bc, "cut_links": cut, "pressure_nodes": n_pr,
                           "omega": omega, "l2": "inputs larger than L2, no flush"},
                "roofline": {"bound": "hbm", "achieved": f32["achieved_gbs"], "peak": peak, "unit": "GB/s",
                             "frac": f32["frac"], "peak_source": peak_src, "scope": "whole pool step"},
                "gpu_launches": f32["gpu_launches"], "forms": out}
        print(json.dumps(line), flush=True)


def run_serving(args):
    """Serving: a Poisson stream of porous-block solves served by continuous batching in one domain
    pool whose arena is the HBM budget. Offered loads are fractions of the measured capacity (node
    updates per second of a full pool / the mean work of a request). Reports p50/p99 time to
    solution and aggregate MLUPS in FP32 and FP16 storage, and the permeability error against each
    request solved alone in FP64."""
    import dataclasses

    import torch

    from virtualfluids_b200 import Pool
    from virtualfluids_b200.serving import Server, poisson_stream, solve_alone

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    base = poisson_stream(args.requests, rate=1.0, seed=20261203 + rank)
    for r in base:
        r.geometry()
    mean_work = float(np.mean([r.fluid_nodes * r.steps for r in base]))
    budget = int(args.hbm_gb * (1 << 30))
    out = {}
    k64 = [solve_alone(r, storage="f64")[0] for r in base]
    for storage in ("f32", "f16"):
        # capacity: a pool filled with the stream's first requests, timed over 50 steps
        s = torch.cuda.Stream()
        cal = Pool(budget, storage=storage, max_domains=len(base))
        nodes = 0
        for r in base:
            g = r.geometry()
            d = cal.try_add(g["shape"], 1.0 / (3 * r.nu + 0.5), periodic=g["periodic"], forces=g["forces"],
                            mask=g["mask"], bcs=g["bcs"])
            if d is None:
                break
            cal.init(d, stream=s)
            nodes += r.fluid_nodes
        cal.step(4, stream=s)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        cal.step(50, stream=s)
        e1.record(s)
        s.synchronize()
        throughput = nodes * 50 / (e0.elapsed_time(e1) / 1e3)
        cal.close()
        capacity = throughput / mean_work
        out[storage] = {"capacity_requests_per_s": round(capacity, 4), "node_updates_per_s": round(throughput, 1)}
        for load in args.loads:
            reqs = [dataclasses.replace(r, arrival=r.arrival / (load * capacity)) for r in base]
            srv = Server(budget, storage=storage, max_domains=len(base))
            with ClockSampler(local) as clk:
                results, st = srv.run(reqs, realtime=True)
            srv.close()
            err = [abs(res.permeability - k) / abs(k) for res, k in zip(results, k64)]
            out[storage][f"load_{load}"] = {
                "offered_requests_per_s": round(load * capacity, 4), "p50_s": round(st["p50_s"], 3),
                "p99_s": round(st["p99_s"], 3), "mlups": round(st["mlups"], 1), "wall_s": round(st["wall_s"], 2),
                "peak_concurrent": st["peak_concurrent"], "gpu_launches": st["gpu_launches"],
                "permeability_rel_err_vs_fp64": {"median": float(np.median(err)), "max": float(np.max(err))},
                "clocks": clk.summary()}
            torch.cuda.empty_cache()
    if rank == 0:
        f32 = out["f32"][f"load_{args.loads[0]}"]
        line = {"metric": f"p50/p99 time to solution and MLUPS, porous-block serving stream ({args.requests} "
                          f"requests, {args.hbm_gb} GB HBM budget, FP32)",
                "value": f32["mlups"], "unit": "MLUPS", "n_gpus": world, "steps": None, "warmup": None,
                "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": "Poisson arrivals; cube side U{32..192}; random non-overlapping spheres r in "
                                       "[3, 8] at porosity U[0.5, 0.9] (jammed packings stop near 0.7) with exact-q "
                                       "interpolated no-slip; pressure drop drho = 3e-3 along x between "
                                       "non-equilibrium pressure planes, periodic y/z; steps U{1000..20000}; "
                                       "nu = 1/60; MLUPS over fluid nodes",
                           "requests": args.requests, "hbm_budget_gb": args.hbm_gb, "loads": args.loads},
                "serving": out}
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_SIDE)
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-gpu-reference", action="store_true",
                    help="--impl reference: skip timing the reference's own GPU kernel beside its CPU path")
    ap.add_argument("--no-list", action="store_true", help="skip the reference-layout (list) measurement")
    ap.add_argument("--arith", default="exact", choices=["fast", "exact"],
                    help="the headline's FP64 arithmetic. exact: every operation rounded as the reference's host "
                         "build (bitwise oracle parity); fast: FMA contraction and a rearranged K17")
    ap.add_argument("--kernel", default="auto", choices=["auto", "direct", "tma", "async", "pipe"])
    ap.add_argument("--workload", default="tgv",
                    choices=["tgv", "batch", "serving", "tgv-forms", "cube", "porous", "tgv-slab", "pool-shapes"],
                    help="tgv: the headline (TGV 256^3 FP64); batch: 4096 ducts in one domain pool; "
                         "serving: a Poisson stream of porous-block solves; tgv-forms: storage-form accuracy; "
                         "cube: duct past a wall-mounted cube; porous: the serving pool's step on fixed blocks; "
                         "tgv-slab: the TGV as one domain in z slabs over the GPUs (NCCL halo exchange); "
                         "pool-shapes: the pool kernel against the box kernel on the same shapes")
    ap.add_argument("--form-steps", type=int, default=10000)
    ap.add_argument("--slab-transport", default="fused", choices=["fused", "nccl"],
                    help="tgv-slab: border planes that store into the neighbours' arrays (fused), or NCCL "
                         "point-to-point transfers after them")
    ap.add_argument("--tgv-forms", default="f64,f32,f16,bf16,e3m12",
                    help="tgv-forms: comma-separated storage[:arith] forms, the first the FP64 reference")
    ap.add_argument("--cube-dims", type=int, nargs=5, default=[512, 256, 256, 32, 128],
                    metavar=("NX", "NY", "NZ", "CUBE", "X0"))
    ap.add_argument("--domains", type=int, default=4096)
    ap.add_argument("--porous-sides", type=int, nargs="+", default=[96, 128, 160, 112])
    ap.add_argument("--check-steps", type=int, default=0)
    ap.add_argument("--requests", type=int, default=32)
    ap.add_argument("--hbm-gb", type=float, default=24.0)
    ap.add_argument("--loads", type=float, nargs="+", default=[0.5, 0.9])
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "batch":
        run_batch(args)
        return
    if args.workload == "serving":
        run_serving(args)
        return
    if args.workload == "tgv-forms":
        run_tgv_forms(args)
        return
    if args.workload == "cube":
        run_cube(args)
        return
    if args.workload == "porous":
        run_porous(args)
        return
    if args.workload == "tgv-slab":
        run_tgv_slab(args)
        return
    if args.workload == "pool-shapes":
        run_pool_shapes(args)
        return

    run_tgv(args)


def run_tgv(args):
    """The headline: TGV 256^3 FP64 through the structured box, with the roofline loop, the end-to-end
    run through the C ABI, the other forms with their errors against FP64, the reference layout,
    and (rank 0, one GPU) the CPU baseline on this same workload plus the cavity's parity."""
    import torch

    import virtualfluids_b200 as vfb
    from virtualfluids_b200 import _native as N

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    n = args.n
    nodes = n ** 3
    omega = omega_tgv(n)
    stream = torch.cuda.Stream(device=dev)
    sp = C.c_void_p(stream.cuda_stream)
    fields = tgv_fields(n, U0)

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return max_over_ranks_of(x, pg, dev)

    def timed_steps(box, steps, energy=None):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ev0.record(stream)
            box.step(steps, energy=energy, stream=sp)
            ev1.record(stream)
        stream.synchronize()
        return ev0.elapsed_time(ev1)

    # ---- device-resident throughput: K steps with the per-step FP64 energy kept on the device ----
    box = vfb.Box(n, n, n, omega, storage="f64", arith=args.arith)
    box.set_kernel_variant(args.kernel)
    box.init(*(torch.from_numpy(a).to(dev) for a in fields), stream=sp)
    energy = torch.zeros(2 * max(args.steps, args.warmup), dtype=torch.float64, device=dev)
    box.step(args.warmup, energy=energy, stream=sp)
    barrier()
    launches0 = box.kernel_launches()
    with ClockSampler(local) as clk:
        t_local = timed_steps(box, args.steps, energy)
    launches = box.kernel_launches() - launches0
    barrier()
    t_ms = max_over_ranks(t_local)
    value = whole_job_mlups(nodes * args.steps, world, t_ms)
    clocks = clk.summary()

    # ---- the collision kernel alone: average of ROOFLINE_LAUNCHES launches, whatever --steps is ----
    k_ms = timed_steps(box, ROOFLINE_LAUNCHES) / ROOFLINE_LAUNCHES
    peak, peak_kind = measured_peak()
    achieved = BYTES_PER_NODE["f64"] * nodes / (k_ms / 1e3) / 1e9
    per_node = NCU_DRAM_BYTES_PER_NODE_F64.get(args.arith) if args.kernel in ("auto", "direct") else None
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "frac_of_nominal_8000": round(achieved / NOMINAL_HBM_GBS, 4),
                "traffic": round(per_node * nodes) if per_node else None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 128^3 launch of the "
                                  "same kernel, scaled by nodes",
                "kernel": f"k17_box_kernel<double> ({args.arith} arithmetic; collision + ET streaming)",
                "kernel_ms": round(k_ms, 4), "launches_timed": ROOFLINE_LAUNCHES,
                "algorithmic_bytes_per_launch": BYTES_PER_NODE["f64"] * nodes}
    e_host = energy[: 2 * args.steps].cpu().numpy()
    box.status()
    del box
    torch.cuda.empty_cache()

    # ---- end to end through the public API with pinned host buffers ----
    host_in = [torch.from_numpy(a).pin_memory() for a in fields]
    host_out = [torch.empty(nodes, dtype=torch.float64).pin_memory() for _ in range(4)]
    host_energy = torch.zeros(2 * max(args.steps, args.warmup), dtype=torch.float64).pin_memory()
    box = vfb.Box(n, n, n, omega, storage="f64", arith=args.arith)
    box.set_kernel_variant(args.kernel)
    lib = N.lib()
    # warm-up of the same path
    N.check(lib.vfb_box_init(box._h, *(C.c_void_p(h.data_ptr()) for h in host_in), 1, sp))
    N.check(lib.vfb_box_step(box._h, args.warmup, C.c_void_p(host_energy.data_ptr()), 1, sp))
    stream.synchronize()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        ev0.record(stream)
        N.check(lib.vfb_box_init(box._h, *(C.c_void_p(h.data_ptr()) for h in host_in), 1, sp))
        N.check(lib.vfb_box_step(box._h, args.steps, C.c_void_p(host_energy.data_ptr()), 1, sp))
        N.check(lib.vfb_box_fields(box._h, *(C.c_void_p(h.data_ptr()) for h in host_out), 1, sp))
        ev1.record(stream)
    stream.synchronize()
    wall_e2e = time.perf_counter() - t0
    barrier()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1))
    e2e_value = whole_job_mlups(nodes * args.steps, world, e2e_ms)
    h2d = 4 * nodes * 8
    d2h = 4 * nodes * 8 + 16 * args.steps
    ek = host_energy.numpy()[1: 2 * args.steps: 2]
    assert np.all(np.isfinite(host_out[1].numpy())) and ek[-1] < ek[0], "e2e run produced no decaying vortex"
    del box
    torch.cuda.empty_cache()

    # ---- the other forms: roofline loop each, and the velocity error against the exact FP64 run
    # at the same step (W warm-up + ROOFLINE_LAUNCHES steps) ----
    forms = {}
    if not args.no_forms:
        cmp_steps = args.warmup + ROOFLINE_LAUNCHES
        ref = vfb.Box(n, n, n, omega, storage="f64", arith="exact")
        ref.init(*(torch.from_numpy(a).to(dev) for a in fields), stream=sp)
        ref.step(cmp_steps, stream=sp)
        want = ref.fields(stream=sp)
        del ref
        torch.cuda.empty_cache()
        other = "f64_fast" if args.arith == "exact" else "f64_exact"
        for name in (other, "f32", "f16", "bf16", "e3m12"):
            st = "f64" if name.startswith("f64") else name
            ar = name[4:] if name.startswith("f64") else "fast"
            dt = np.float64 if st == "f64" else np.float32
            b = vfb.Box(n, n, n, omega, storage=st, arith=ar)
            if args.kernel != "async" or st in ("f64", "f32"):
                b.set_kernel_variant(args.kernel)
            b.init(*(torch.from_numpy(a.astype(dt)).to(dev) for a in fields), stream=sp)
            b.step(args.warmup, stream=sp)
            ms = timed_steps(b, ROOFLINE_LAUNCHES) / ROOFLINE_LAUNCHES
            got = b.fields(stream=sp)
            gbs = BYTES_PER_NODE[st] * nodes / (ms / 1e3) / 1e9
            forms[name] = {"mlups": round(nodes / (ms / 1e3) / 1e6, 1), "kernel_ms": round(ms, 4),
                           "hbm_gbs": round(gbs, 1), "frac": round(gbs / peak, 4),
                           "error_vs_f64_exact": field_errors(got, want, cmp_steps)}
            del b
            torch.cuda.empty_cache()
            if st != "f64" and args.kernel == "auto":
                # the two-node kernel (packed FP32x2 arithmetic): not a box's default, since a pool
                # domain computes the direct kernel's bits; timed beside it on the same state
                b = vfb.Box(n, n, n, omega, storage=st, arith=ar)
                b.set_kernel_variant("pairs")
                b.init(*(torch.from_numpy(a.astype(dt)).to(dev) for a in fields), stream=sp)
                b.step(args.warmup, stream=sp)
                ms2 = timed_steps(b, ROOFLINE_LAUNCHES) / ROOFLINE_LAUNCHES
                got2 = b.fields(stream=sp)
                gbs2 = BYTES_PER_NODE[st] * nodes / (ms2 / 1e3) / 1e9
                forms[name]["pairs_kernel"] = {"mlups": round(nodes / (ms2 / 1e3) / 1e6, 1), "kernel_ms": round(ms2, 4),
                                               "hbm_gbs": round(gbs2, 1), "frac": round(gbs2 / peak, 4),
                                               "error_vs_f64_exact": field_errors(got2, want, cmp_steps)}
                del b
                torch.cuda.empty_cache()
        if "f16" in forms:
            forms["f16"]["speedup_vs_headline_kernel"] = round(k_ms / forms["f16"]["kernel_ms"], 3)
            forms["bf16"]["speedup_vs_headline_kernel"] = round(k_ms / forms["bf16"]["kernel_ms"], 3)
            forms["e3m12"]["speedup_vs_headline_kernel"] = round(k_ms / forms["e3m12"]["kernel_ms"], 3)

    # ---- the reference layout: the drop-in step driver over neighborX/Y/Z lists (device resident) ----
    ref_layout = None
    if not args.no_list:
        ref_layout = run_list_path(args, n, omega, fields, dev)

    cb = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline(n, threads=os.cpu_count())
        parity = cavity_parity(cb.pop("_cavity_fields"), dev)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": tgv_config(n, world, args.arith, args.kernel),
            "roofline": roofline,
            "e2e": {"value": round(e2e_value, 1), "unit": "MLUPS", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps, "wall_s": round(wall_e2e, 3)},
            "gpu_launches": launches,
            "clocks": clocks,
            "forms": forms,
            "kinetic_energy": {"first": float(e_host[1]), "last": float(e_host[-1])},
        }
        if ref_layout:
            line["reference_layout"] = ref_layout
        if cb:
            line["cpu_baseline"] = cb
        if parity:
            line["parity"] = parity
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def field_errors(got, want, steps):
    """Velocity error of a form against the exact FP64 run at the same step: relative L2 (RMS of the
    speed of the difference over the RMS speed) and relative L-inf (largest speed of the difference
    over the largest speed); for the FP64 forms also the relative L-inf of drho."""
    u = np.stack([got["vx"], got["vy"], got["vz"]]).astype(np.float64)
    w = np.stack([want["vx"], want["vy"], want["vz"]])
    d2 = ((u - w) ** 2).sum(axis=0)
    w2 = (w ** 2).sum(axis=0)
    out = {"step": steps, "u_l2_rel": float(np.sqrt(d2.mean() / w2.mean())),
           "u_linf_rel": float(np.sqrt(d2.max() / w2.max()))}
    if got["rho"].dtype == np.float64:
        out["drho_linf_rel"] = float(np.abs(got["rho"] - want["rho"]).max() / np.abs(want["rho"]).max())
    return out

if __name__ == "__main__":
    main()
