"""Phase timers of the step driver (vfb_simulation_set_timing / vfb_simulation_phase_times, the
reference's TimeStepTimer phases plus the two interpolation directions): on a two-level refined
cavity every phase that has work gets device time, the phase times add up to no more than the run's
own event time, the timed run computes the same bits as an untimed one, and reset clears them."""
import numpy as np
import pytest
import torch

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import GridScalingFactory, ListGrid, MultiLevelGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu


def _cavity(timing):
    m = MultiLevelGrid.uniform(ListGrid(24, 24, 24, periodic=(True, True, True)))
    m.refine((6, 6, 6), (18, 18, 18))
    p = Parameter()
    p.set_viscosity_lb(0.01)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.arith = N.ARITH_EXACT
    s = GridScalingFactory()
    s.set_scaling_factory(GridScalingFactory.GridScaling.ScaleCompressible)
    sim = Simulation(p, m, BCF(), s)
    rng = np.random.default_rng(3)
    for level in range(2):
        n = m.levels[level].number_of_nodes
        u = [np.zeros(n)] + [0.01 * np.sin(2 * np.pi * m.positions(level)[a] / 24.0 + rng.uniform(0, 6)) for a in range(3)]
        for a in u:
            a[0] = 0.0
        sim.init(*u, level=level)
    if timing:
        sim.set_timing(True)
    return sim


def test_phase_times(cuda):
    ref = _cavity(False)
    ref.run(6)
    want = [ref.populations(l) for l in range(2)]
    ref.close()
    sim = _cavity(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(torch.cuda.default_stream())
    sim.run(6)
    e1.record(torch.cuda.default_stream())
    torch.cuda.synchronize()
    total = e0.elapsed_time(e1)
    times, steps = sim.phase_times()
    print(times, total)
    assert steps == 6
    for phase in ("collision", "preCollisionBC", "scalingFineToCoarse", "scalingCoarseToFine"):
        assert times[phase] > 0.0, phase
    assert sum(times.values()) <= total * 1.05 + 0.05
    got = [sim.populations(l) for l in range(2)]
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    times, steps = sim.phase_times(reset=True)
    assert steps == 6
    times, steps = sim.phase_times()
    assert steps == 0 and all(v == 0.0 for v in times.values())
    sim.close()
