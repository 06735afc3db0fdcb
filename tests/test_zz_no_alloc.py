"""The allocation-free mass / kinetic-energy reduction (vfb_mass_energy_no_alloc).

Some callers of this library cannot hand it device memory: a host application that owns every
allocation on the GPU, a solver loop that runs under a strict no-allocation rule, or code that must
not call cudaMalloc because that call can stall the whole device. For them the reduction keeps its
scratch space (the per-block partial sums) in a fixed array inside the library's own device
memory. These tests call that entry point through the C ABI and check it against the regular
entry point, which takes caller-provided workspace, on two calls in a row. Both run the same
partial-sum kernel and the same fixed-order reduction, so the results must be the same bits.
"""
import ctypes as C

import numpy as np
import pytest

from virtualfluids_b200 import BoundaryConditionFactory as BCF
from virtualfluids_b200 import ListGrid, Parameter, Simulation
from virtualfluids_b200 import _native as N

pytestmark = pytest.mark.gpu


def _cavity_simulation(n=16, storage=N.STORAGE_F64, arith=N.ARITH_FAST):
    g = ListGrid(n, n, n)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    p = Parameter()
    p.set_viscosity_lb(0.05 * n / 100.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.storage = storage
    p.arith = arith
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim = Simulation(p, g, bcf)
    sim.init()
    return sim


def _with_workspace(sim):
    """The regular entry point, scratch supplied by the caller."""
    return sim.mass_energy()


def _no_alloc(sim):
    out = (C.c_double * 2)()
    status = N.lib().vfb_mass_energy_no_alloc(C.byref(sim.level), C.c_void_p(sim.fluid.data_ptr()),
                                              int(sim.grid.fluid.size), out, None)
    N.check(status)
    return out[0], out[1]


@pytest.mark.parametrize("storage, arith", [
    (N.STORAGE_F64, N.ARITH_FAST), (N.STORAGE_F32, N.ARITH_FAST), (N.STORAGE_F16, N.ARITH_FAST),
    (N.STORAGE_BF16, N.ARITH_FAST), (N.STORAGE_E3M12, N.ARITH_FAST), (N.STORAGE_F64, N.ARITH_EXACT),
    (N.STORAGE_F32, N.ARITH_EXACT)])
def test_no_alloc_reduction_matches_workspace_reduction_twice(cuda, storage, arith):
    sim = _cavity_simulation(storage=storage, arith=arith)
    sim.run(30)
    first_ref = _with_workspace(sim)
    first = _no_alloc(sim)
    # second call on a different state: the shared scratch array must not leak the first result
    sim.run(40)
    second_ref = _with_workspace(sim)
    second = _no_alloc(sim)
    for got, ref in ((first, first_ref), (second, second_ref)):
        assert np.array_equal(np.array(got), np.array(ref)), (got, ref)
    assert second[1] != first[1]  # the flow developed between the calls
    assert first[1] > 0.0


def test_no_alloc_rejects_more_nodes_than_its_scratch_holds(cuda):
    sim = _cavity_simulation(n=8)
    out = (C.c_double * 2)()
    too_many = (1 << 24) + 1
    status = N.lib().vfb_mass_energy_no_alloc(C.byref(sim.level), C.c_void_p(sim.fluid.data_ptr()), too_many, out,
                                              None)
    assert status == N.VFB_ERR_INVALID_ARGUMENT
    assert b"VFB_NO_ALLOC_MAX_NODES" in N.lib().vfb_last_error()


def test_no_alloc_rejects_the_levels_vfb_mass_energy_rejects(cuda):
    """A bad level is refused by both entry points with the same status, also for an empty list."""
    sim = _cavity_simulation(n=8)
    out = (C.c_double * 2)()
    bad = type(sim.level).from_buffer_copy(sim.level)
    bad.arith = 7
    for size in (0, int(sim.grid.fluid.size)):
        st = N.lib().vfb_mass_energy_no_alloc(C.byref(bad), C.c_void_p(sim.fluid.data_ptr()), size, out, None)
        assert st == N.VFB_ERR_INVALID_ARGUMENT
    bad = type(sim.level).from_buffer_copy(sim.level)
    bad.omega = 2.5
    st = N.lib().vfb_mass_energy_no_alloc(C.byref(bad), C.c_void_p(sim.fluid.data_ptr()), 0, out, None)
    assert st == N.VFB_ERR_INVALID_ARGUMENT
