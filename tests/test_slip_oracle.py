"""The slip BC of the oracle (SlipCompressible_Device, BoundaryConditions/Slip/SlipCompressible.cu:
44-550) on the CPU: a uniform flow parallel to slip walls stays uniform, where no-slip walls slow it
down. The GPU kernel is pinned to the reference's own kernel and to this oracle in
tests/test_gpu_slip.py."""
import ctypes as C

import numpy as np

from virtualfluids_b200 import ListGrid


def _step_with_list(oracle, lv, k, q, slip):
    lib = oracle.lib()
    ptr = oracle.ptr
    lib.orc_collision(C.byref(lv.L), ptr(lv.fluid), lv.fluid.size, lv.is_even.value, lv.omega, ptr(lv.lim),
                      ptr(lv.forces), 0, None, None, None, None, 0)
    if slip:
        lib.orc_bc_slip(C.byref(lv.L), ptr(k), ptr(q), k.size, lv.is_even.value, lv.omega)
    else:
        lib.orc_bc_noslip_interpolated(C.byref(lv.L), ptr(k), ptr(q), k.size, lv.is_even.value, lv.omega)
    lv.is_even.value = 1 - lv.is_even.value


def test_uniform_flow_along_slip_walls_stays_uniform(oracle):
    out = {}
    for slip in (True, False):
        g = ListGrid(8, 6, 5, periodic=(True, False, True))
        g.add_side("MY", "slip" if slip else "noslip")
        g.add_side("PY", "slip" if slip else "noslip")
        k, q, _ = g.merged("slip" if slip else "noslip")
        k = np.ascontiguousarray(k.astype(np.int32))
        q = np.ascontiguousarray(q.reshape(-1))
        n = g.number_of_nodes
        lv = oracle.OracleLevel(g, 1.8)
        lv.init(np.zeros(n), np.full(n, 0.05), np.zeros(n), np.zeros(n))
        for _ in range(30):
            _step_with_list(oracle, lv, k, q, slip)
        out[slip] = lv.macroscopic()["vx"][g.fluid]
    np.testing.assert_allclose(out[True], 0.05, rtol=1e-12)
    assert out[False].min() < 0.049                       # the no-slip walls decelerate the flow
