"""Run by tests/test_gpu_bounds_check.py in a process of its own with VFB_LIBRARY=checked (a process
loads one build of the library). Prints one JSON line with what it measured."""
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

from oracle import pyoracle  # noqa: E402
from virtualfluids_b200 import BoundaryConditionFactory as BCF  # noqa: E402
from virtualfluids_b200 import ListGrid, Parameter, Simulation  # noqa: E402
from virtualfluids_b200 import _native as N  # noqa: E402


def status():
    bad, n = C.c_uint64(), C.c_uint64()
    st = N.lib().vfb_bounds_check_status(C.byref(bad), C.byref(n))
    return st, bad.value, n.value


def main():
    import torch
    out = {"checked": N.lib().vfb_bounds_checked(), "library": str(N._LIB_PATH.name)}
    g = ListGrid(10, 10, 10)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    p = Parameter()
    p.set_viscosity_lb(0.05 * 10 / 100.0)
    p.configure_main_kernel("K17CompressibleNavierStokes")
    p.arith = N.ARITH_EXACT
    bcf = BCF()
    bcf.set_no_slip_boundary_condition(BCF.NoSlipBC.NoSlipBounceBack)
    bcf.set_velocity_boundary_condition(BCF.VelocityBC.VelocityBounceBack)
    sim = Simulation(p, g, bcf)
    sim.init()
    sim.run(40)
    orc = pyoracle.OracleLevel(g, omega=p.omega)
    orc.init()
    orc.run(40)
    out["bitwise_with_checks"] = bool(np.array_equal(sim.populations(), orc.f))
    out["status_clean"] = status()
    # a fluid-node list with one index beyond the level: the checked kernel records it and maps it
    # to the dummy node 0
    n = g.number_of_nodes
    idx = torch.from_numpy(np.concatenate([g.fluid[:50], [n + 5]]).astype(np.int32)).cuda()
    L = type(sim.level).from_buffer_copy(sim.level)
    N.check(N.lib().vfb_k17_run_on_indices(C.byref(L), C.c_void_p(idx.data_ptr()), int(idx.numel()), 0, None))
    out["status_bad_fluid_index"] = status()
    out["status_after_read"] = status()
    # a no-slip list entry beyond the level
    k = torch.tensor([int(g.fluid[7]), n + 11], dtype=torch.int32, device="cuda")
    q = torch.full((27 * 2,), 0.5, dtype=torch.float64, device="cuda")
    bc = N.BC()
    bc.k, bc.q27, bc.number_of_bc_nodes = k.data_ptr(), q.data_ptr(), 2
    N.check(N.lib().vfb_noslip_bounce_back(C.byref(L), C.byref(bc), None))
    out["status_bad_bc_index"] = status()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
