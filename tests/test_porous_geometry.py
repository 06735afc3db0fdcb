"""The porous-block geometry of the serving workload (workloads.porous_block_bcs), checked by brute
force on the host against its definition:

* the no-slip list holds exactly the fluid nodes with a link that enters a sphere (or a periodic
  image of one in y and z) at a ray parameter t in [0, 1], in ascending node order, once each;
* each cut link's q is the smallest such t over all spheres and images, and p + q c_d lies on that
  sphere's surface;
* the pressure planes are the fluid layers x = 1 (outward normal M00, neighbour x = 2,
  drho = +drho/2) and x = side (P00, neighbour x = side - 1, -drho/2), every (y, z) once.
"""
import numpy as np
import pytest

from virtualfluids_b200 import _native as N
from virtualfluids_b200.workloads import _CX, _CY, _CZ, porous_block_bcs, sphere_link_q


@pytest.fixture(scope="module", params=[(24, 3, 0.75), (20, 7, 0.6)], ids=["24-phi0.75", "20-phi0.6"])
def block(request):
    side, seed, phi = request.param
    return side, porous_block_bcs(side, seed, porosity=phi)


def _fluid_points(g):
    nx, ny, nz = g["shape"]
    k = np.nonzero(g["mask"])[0]
    return k, np.stack([k % nx, (k // nx) % ny, k // (nx * ny)], axis=1).astype(np.float64)


def _brute_q(g, side, pts):
    """Smallest entry parameter over every sphere and periodic image, per link: (27, n), -1 uncut."""
    best = np.full((27, pts.shape[0]), np.inf)
    for (cx, cy, cz, r) in g["spheres"]:
        for oy in (-side, 0, side):
            for oz in (-side, 0, side):
                q = sphere_link_q(pts, (cx + 1.0, cy + oy, cz + oz), r)
                best = np.where((q >= 0.0) & (q < best), q, best)
    return np.where(np.isinf(best), -1.0, best)


def test_noslip_list_is_every_cut_fluid_node_with_its_smallest_q(block):
    side, g = block
    k_list, q_list = g["bcs"]["noslip"]
    assert q_list.shape == (27, k_list.size) and k_list.size > 0
    assert np.all(np.diff(k_list.astype(np.int64)) > 0)
    assert np.all(g["mask"][k_list] != 0)
    k, pts = _fluid_points(g)
    want = _brute_q(g, side, pts)
    cut = (want >= 0.0).any(axis=0)
    assert np.array_equal(k[cut], k_list)
    assert np.array_equal(want[:, cut], q_list)
    assert np.all(q_list[0] == -1.0)


def test_cut_points_lie_on_a_sphere_surface(block):
    side, g = block
    nx, ny, _ = g["shape"]
    k_list, q_list = g["bcs"]["noslip"]
    p = np.stack([k_list % nx, (k_list // nx) % ny, k_list // (nx * ny)], axis=1).astype(np.float64)
    centres = np.array([(cx + 1.0, cy + oy, cz + oz, r) for (cx, cy, cz, r) in g["spheres"]
                        for oy in (-side, 0, side) for oz in (-side, 0, side)])
    checked = 0
    for d in range(1, 27):
        sel = q_list[d] >= 0.0
        if not sel.any():
            continue
        c = np.array([_CX[d], _CY[d], _CZ[d]], dtype=np.float64)
        hit = p[sel] + q_list[d][sel, None] * c
        dist = np.sqrt(((hit[:, None, :] - centres[None, :, :3]) ** 2).sum(axis=2)) - centres[None, :, 3]
        assert np.abs(dist).min(axis=1).max() < 1e-9
        checked += int(sel.sum())
    assert checked > 100


def test_pressure_planes(block):
    side, g = block
    nx, ny, nz = g["shape"]
    k, kn, rho, direction = g["bcs"]["pressure"]
    assert k.size == 2 * ny * nz
    x, yz = k % nx, k // nx
    inlet = direction == N.DIR_M00
    outlet = direction == N.DIR_P00
    assert np.all(inlet | outlet) and inlet.sum() == outlet.sum() == ny * nz
    assert np.all(x[inlet] == 1) and np.all(x[outlet] == side)
    assert np.array_equal(kn[inlet], k[inlet] + 1) and np.array_equal(kn[outlet], k[outlet] - 1)
    assert np.all(rho[inlet] == 0.5 * g["drho"]) and np.all(rho[outlet] == -0.5 * g["drho"])
    assert np.unique(yz[inlet]).size == ny * nz and np.unique(yz[outlet]).size == ny * nz
    assert np.all(g["mask"][k] != 0)
    # the stopper layers are solid, the planes' neighbours fluid
    X = np.arange(nx * ny * nz) % nx
    assert np.all(g["mask"][(X == 0) | (X == nx - 1)] == 0)
    assert np.all(g["mask"][kn] != 0)
