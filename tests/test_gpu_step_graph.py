"""The step driver's loop as a CUDA graph (vfb_simulation_set_graph): runs that replay captured
steps give the populations of the direct loop bit for bit -- on a lid-driven cavity with bounce-back
and with interpolated BCs plus a pressure outlet, on two refinement levels, across odd step counts
(a parity that differs from the capture's makes a new capture), and after a BC list is set again
(the setter drops the graph). Also times the 64^3 cavity both ways."""
import time

import numpy as np
import pytest
import torch

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import GridScalingFactory, ListGrid, MultiLevelGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu


def _cavity(n=16, interpolated=False, graph=0):
    g = ListGrid(n, n, n)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    p = Parameter()
    p.set_viscosity_lb(0.05 * n / 100.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.arith = N.ARITH_EXACT
    bcf = BCF()
    if interpolated:
        bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipInterpolatedCompressible)
        bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityInterpolatedCompressible)
    else:
        bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
        bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim = Simulation(p, g, bcf)
    sim.init()
    if graph:
        sim.set_graph(graph)
    return sim


@pytest.mark.parametrize("interpolated", [False, True])
def test_graph_runs_equal_direct_runs(cuda, interpolated):
    ref = _cavity(interpolated=interpolated)
    sim = _cavity(interpolated=interpolated, graph=8)
    for steps in (37, 5, 20, 1, 16):
        ref.run(steps)
        sim.run(steps)
        assert np.array_equal(sim.populations(), ref.populations()), steps
    ref.close()
    sim.close()


def test_two_levels_in_a_graph(cuda):
    def make(graph):
        m = MultiLevelGrid.uniform(ListGrid(16, 16, 16, periodic=(True, True, True)))
        m.refine((4, 4, 4), (12, 12, 12))
        p = Parameter()
        p.set_viscosity_lb(0.005)
        p.configure_main_kernel("K17CompressibleNavierStokes")
        p.arith = N.ARITH_EXACT
        s = GridScalingFactory()
        s.set_scaling_factory(GridScalingFactory.GridScaling.ScaleCompressible)
        sim = Simulation(p, m, BCF(), s)
        for level in range(2):
            pos = m.positions(level)
            u = [np.zeros(pos.shape[1])] + [0.01 * np.sin(2 * np.pi * pos[a] / 16.0 + a) for a in range(3)]
            for a in u:
                a[0] = 0.0
            sim.init(*u, level=level)
        if graph:
            sim.set_graph(graph)
        return sim
    ref, sim = make(0), make(4)
    for steps in (11, 6):
        ref.run(steps)
        sim.run(steps)
        for level in range(2):
            assert np.array_equal(sim.populations(level), ref.populations(level)), (steps, level)
    ref.close()
    sim.close()


def test_cavity_64_timing(cuda):
    out = {}
    for graph in (0, 16):
        sim = _cavity(64, graph=graph)
        sim.run(40)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.run(2000)
        torch.cuda.synchronize()
        out[graph] = (time.perf_counter() - t0) / 2000 * 1e3
        sim.close()
    print(f"64^3 cavity ms per step: direct {out[0]:.4f}, graph {out[16]:.4f}")
    assert out[16] <= out[0] * 1.05
