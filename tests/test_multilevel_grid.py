"""Nested refinement levels on the host: the refined-box builder's interface cells against the
rules of the reference's GridInterface, and the oracle's multi-level driver on physical checks.

* coarse-to-fine cells: the outer cell layer of the refined box; their fine nodes are exactly the
  fine level's two outer node layers, at coarse position + 1/4;
* fine-to-coarse cells: centred on the shell of [lo + 2, hi - 2]^3, their MMM fine node at the
  coarse node - 1/4; the coarse nodes inside that shell are not collided;
* a fluid at rest stays at rest to round-off; a uniform flow along one axis is reproduced exactly
  by the interpolation (the product-form equilibrium of one velocity component is the polynomial
  one of the initialisation); a shear wave decays at the analytic rate on both levels.
"""
import numpy as np
import pytest

from virtualfluids_b200 import ListGrid, MultiLevelGrid, refine_box


def _box(n=16, lo=(4, 4, 4), hi=(12, 12, 12)):
    m = MultiLevelGrid.uniform(ListGrid(n, n, n, periodic=(True, True, True)))
    fine = m.refine(lo, hi)
    return m, fine, m.interfaces[0]


def test_interface_cells_follow_the_grid_interface_rules():
    m, fine, it = _box()
    pc, pf = m.positions(0), m.positions(1)
    assert fine.nx == fine.ny == fine.nz == 16
    assert it.coarse_cf.size == 8 ** 3 - 6 ** 3 and it.coarse_fc.size == 5 ** 3 - 3 ** 3
    assert np.array_equal(pf[:, it.fine_cf], pc[:, it.coarse_cf] + 0.25)
    assert np.array_equal(pf[:, it.fine_fc], pc[:, it.coarse_fc] - 0.25)
    # the eight fine nodes of the coarse-to-fine cells are the fine level's two outer layers
    c = fine.coords[:, it.fine_cf]
    covered = {tuple(c[:, i] + (dx, dy, dz)) for i in range(c.shape[1])
               for dx in (0, 1) for dy in (0, 1) for dz in (0, 1)}
    f = fine.coords[:, fine.fluid]
    outer = {tuple(f[:, i]) for i in range(f.shape[1]) if min(f[:, i].min(), (15 - f[:, i]).min()) <= 1}
    assert covered == outer
    # fine-to-coarse centres sit on the shell of [6, 10]^3; nothing below it is collided
    cc = m.levels[0].coords[:, it.coarse_fc]
    assert ((cc >= 6) & (cc <= 10)).all() and ((cc == 6) | (cc == 10)).any(axis=0).all()
    fl = m.levels[0].coords[:, m.levels[0].fluid]
    assert not ((fl >= 7) & (fl <= 9)).all(axis=0).any()
    assert m.levels[0].fluid.size == 16 ** 3 - 3 ** 3
    assert np.all(np.diff(it.coarse_cf.astype(np.int64)) > 0)     # coarse matrix order, as GridInterface


def test_refined_box_bounds_are_checked():
    g = ListGrid(16, 16, 16, periodic=(True, True, True))
    for lo, hi in (((1, 4, 4), (12, 12, 12)), ((4, 4, 4), (14, 12, 12)), ((4, 4, 4), (7, 12, 12))):
        with pytest.raises(ValueError):
            refine_box(g, lo, hi)
    cavity = ListGrid(16, 16, 16)
    cavity.add_box_obstacle((7, 7, 7), (8, 8, 8))
    with pytest.raises(ValueError):
        refine_box(cavity, (4, 4, 4), (12, 12, 12))


def _oracle_run(oracle, m, nu, steps, fields):
    o = oracle.OracleMultiLevel(m, nu)
    for level in range(len(m.levels)):
        o.init(level, *fields(level))
    o.run(steps)
    return o


@pytest.mark.parametrize("u", [(0.0, 0.0, 0.0), (0.03, 0.0, 0.0), (0.0, 0.0, -0.02)], ids=["rest", "ux", "uz"])
def test_oracle_levels_keep_a_uniform_state(oracle, u):
    m, _, _ = _box()
    o = _oracle_run(oracle, m, 0.01, 3,
                    lambda lv: [np.zeros(m.levels[lv].number_of_nodes)] +
                    [np.full(m.levels[lv].number_of_nodes, c) for c in u])
    for level in range(2):
        mac = o.levels[level].macroscopic()
        f = m.levels[level].fluid
        assert np.abs(mac["rho"][f]).max() < 1e-15
        for key, c in zip(("vx", "vy", "vz"), u):
            assert np.abs(mac[key][f] - c).max() < 1e-15


def test_oracle_refined_shear_wave_decays_at_the_analytic_rate(oracle):
    """16^3 box refined over its centre half, 50 coarse steps: the amplitude on both levels is
    within 1.5 % of U exp(-nu k^2 t) (1.25 % on the uniform box at this resolution)."""
    n, U, nu, steps = 16, 0.02, 0.01, 50
    k = 2 * np.pi / n
    m, _, _ = _box(n, (4, 4, 4), (12, 12, 12))
    o = _oracle_run(oracle, m, nu, steps,
                    lambda lv: [None, U * np.sin(k * (m.positions(lv)[2] + 0.5)), None, None])
    want = U * np.exp(-nu * k * k * steps)
    for level in range(2):
        f = m.levels[level].fluid
        s = np.sin(k * (m.positions(level)[2][f] + 0.5))
        ux = o.levels[level].macroscopic()["vx"][f]
        amp = (ux * s).sum() / (s * s).sum()
        assert abs(amp / want - 1.0) < 1.5e-2
        assert np.abs(ux - amp * s).max() < 1e-2 * U


def test_sphere_obstacle_cuts_every_link_into_it_exactly():
    """ListGrid.add_sphere_obstacle: every link from a fluid node to a node inside the sphere has
    q in [0, 1], and p + q c lies on the sphere (to round-off)."""
    from virtualfluids_b200.grid import CX, CY, CZ
    g = ListGrid(20, 16, 16)
    c, r = np.array([9.3, 7.6, 8.1]), 3.7
    bc = g.add_sphere_obstacle(c, r)
    row = {int(k): i for i, k in enumerate(bc.k)}
    pos = g.coords.astype(np.float64)
    checked = 0
    for k in g.fluid:
        for d in range(1, 27):
            cd = np.array([CX[d], CY[d], CZ[d]], dtype=np.float64)
            if ((pos[:, k] + cd - c) ** 2).sum() > r * r:
                continue
            i = row[int(k)]
            q = bc.q[d, i]
            assert 0.0 <= q <= 1.0
            assert abs(np.linalg.norm(pos[:, k] + q * cd - c) - r) < 1e-12
            checked += 1
    assert checked > 500
