"""The oracle's post-collision BC lists are order-independent: every BC node reads the collision's
values before any node of the list writes (the semantics the GPU kernels keep with guard tables
and snapshots). Around a sphere with exact q some links are cut from both ends, so a BC node's
write lands in a slot that another node of the list reads; the result must still not depend on
the order of the list. Runs on the host only."""
import ctypes as C

import numpy as np

from virtualfluids_b200.grid import CX, CY, CZ, ListGrid


def _sphere_channel():
    g = ListGrid(26, 14, 14, periodic=(False, True, True))
    g.add_side("MX", "velocity", velocity=(0.03, 0.0, 0.0))
    g.add_side("PX", "pressure", rho=0.0)
    g.add_sphere_obstacle((9.4, 6.7, 6.2), 3.3)
    return g


def _mutual_links(g, k, q):
    """Cut links (node i, direction d) whose far end is another node of the same list."""
    at = {tuple(g.coords[:, int(kk)]): i for i, kk in enumerate(k)}
    dims = np.array(g.dims)
    count = 0
    for i, kk in enumerate(k):
        p = g.coords[:, int(kk)]
        for d in range(1, 27):
            if not (0.0 <= q[d, i] <= 1.0):
                continue
            x = np.array([p[0] + CX[d], p[1] + CY[d], p[2] + CZ[d]])
            x[1:] %= dims[1:]
            if tuple(x) in at:
                count += 1
    return count


def test_geometry_bc_result_does_not_depend_on_list_order(oracle):
    g = _sphere_channel()
    k, q, _ = g.merged("geometry")
    assert _mutual_links(g, k, q) > 0
    steps = 30
    runs = []
    for perm in (np.arange(k.size), np.random.default_rng(5).permutation(k.size)):
        orc = oracle.OracleLevel(g, omega=1.85, velocity_kind=2, noslip_kind=2, geometry_kind=2)
        kp = np.ascontiguousarray(k[perm].astype(np.int32))
        qp = np.ascontiguousarray(q[:, perm].reshape(-1))
        orc._keep += [kp, qp]
        orc.geo_bc = type(orc.geo_bc)(kp.ctypes.data_as(C.c_void_p).value, qp.ctypes.data_as(C.c_void_p).value,
                                      k.size, 2)
        orc.init()
        orc.run(steps)
        runs.append(orc.f.copy())
    assert np.array_equal(runs[0], runs[1])
