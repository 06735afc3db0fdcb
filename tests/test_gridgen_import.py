"""Grids built by the reference's own grid generator (oracle/_ref/libvfref_gridgen.so: its
MultipleGridBuilder compiled from src/gpu/GridGenerator) imported with virtualfluids_b200.gridgen:

* a cavity (five no-slip sides, a moving lid) imports to exactly the level grid.ListGrid builds
  (node numbering, neighbour lists, fluid list, BC nodes and q), which pins the library's own
  builder to the reference's;
* a sphere obstacle's geometry BC (nodes and exact q) equals grid.ListGrid.add_sphere_obstacle's,
  node for node by position;
* a refined cavity whose fine box touches a wall brings interpolation cells with non-zero offsets
  (ICellNeigh), every imported level writes each slot once per step, and the oracle runs it;
* a channel with a velocity inlet, a pressure outlet and a cuboid obstacle imports its per-side
  pressure list with the side's direction;
* bad indices are rejected at import.
"""
import numpy as np
import pytest

from virtualfluids_b200 import ListGrid
from virtualfluids_b200 import _native as N
from virtualfluids_b200.checks import check_grid
from virtualfluids_b200.gridgen import import_levels

BOX = (-0.5, -0.5, -0.5, 0.5, 0.5, 0.5)


@pytest.fixture(scope="module")
def ref(oracle):
    if oracle.refgg() is None:
        pytest.skip("the reference grid generator is not built here (make -C oracle ref)")
    return oracle


def _cavity_levels(ref, delta, refinements=()):
    return ref.reference_grid(BOX, delta, refinements=refinements, noslip=("PX", "MX", "PY", "MY", "MZ"),
                              velocity=[("PZ", 0.05, 0.0, 0.0)])


def test_reference_cavity_is_the_listgrid_cavity(ref):
    G = import_levels(*_cavity_levels(ref, 1 / 16))
    g = G.levels[0]
    ours = ListGrid(16, 16, 16)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        ours.add_side(s, "noslip")
    ours.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    assert g.number_of_nodes == ours.number_of_nodes
    for a in range(3):
        assert np.array_equal(g.neighbor[a], ours.neighbor[a])
    assert np.array_equal(g.fluid, ours.fluid)
    assert np.array_equal(g.geo, ours.geo)           # GEO_FLUID, and GEO_VOID for every other node
    # the builder's no-slip sides are zero-velocity entries of its velocity list (LevelGridBuilder.cpp:266-285)
    k, q, v = g.merged("velocity")
    parts = [ours.merged("noslip"), ours.merged("velocity")]
    ko = np.concatenate([p[0] for p in parts])
    qo = np.concatenate([p[1] for p in parts], axis=1)
    vo = np.concatenate([p[2] for p in parts], axis=1)
    assert np.array_equal(k, ko) and np.array_equal(q, qo) and np.array_equal(v, vo)
    assert check_grid(g)["ok"]


def test_reference_sphere_geometry_matches_listgrid_sphere(ref):
    dx = 1 / 16
    centre, radius = (0.1, -0.05, 0.0), 0.2
    G = import_levels(*ref.reference_grid(BOX, dx, geometries=[("sphere", *centre, radius)],
                                          periodic=(True, True, True), geometry_noslip=True),
                      periodic=(True, True, True))
    g = G.levels[0]
    ours = ListGrid(16, 16, 16, periodic=(True, True, True))
    shift = BOX[0] / dx + 0.5                       # world / dx of fluid-box coordinate 0
    ours.add_sphere_obstacle(tuple(c / dx - shift for c in centre), radius / dx)
    key = lambda c, i: tuple(np.round(c[:, i]).astype(int))
    mine = {key(ours.coords.astype(float), i): i for i in ours.fluid}
    theirs = {key(g.coords - shift, i): i for i in g.fluid}
    assert mine.keys() == theirs.keys()              # the same solid nodes are removed
    k, q, _ = g.merged("geometry")
    ko, qo, _ = ours.merged("geometry")
    pos_of = {int(i): key(g.coords - shift, i) for i in k}
    ours_by_pos = {key(ours.coords.astype(float), int(i)): c for c, i in enumerate(ko)}
    assert set(pos_of.values()) == set(ours_by_pos)
    for c, i in enumerate(k):
        qa, qb = q[:, c], qo[:, ours_by_pos[pos_of[int(i)]]]
        assert np.array_equal(qa >= 0, qb >= 0)
        np.testing.assert_allclose(np.where(qa >= 0, qa, 0), np.where(qb >= 0, qb, 0), rtol=0, atol=1e-12)
    assert check_grid(g)["ok"]


def test_refined_cavity_with_the_fine_box_on_a_wall(ref, oracle):
    lev, ifs = _cavity_levels(ref, 1 / 12, refinements=[((-0.5, -0.25, -0.25, 0.0, 0.25, 0.25), 1)])
    G = import_levels(lev, ifs)
    assert len(G.levels) == 2 and G.spacing == [1.0, 0.5]
    it = G.interfaces[0]
    assert it.coarse_cf.size > 0 and it.coarse_fc.size > 0
    assert np.count_nonzero(it.offsets_cf) > 0      # cells at the wall expand about a shifted point
    assert set(np.unique(it.offsets_cf)) <= {-1.0, 0.0, 1.0}
    for g in G.levels:
        assert check_grid(g)["ok"]
    o = oracle.OracleMultiLevel(G, 0.05 * 12 / 100)
    o.run(10)
    for l in range(2):
        m = o.levels[l].macroscopic()
        assert np.all(np.isfinite(m["vx"])) and np.abs(m["vx"]).max() > 0


def test_channel_with_pressure_outlet_and_cuboid(ref):
    lev, ifs = ref.reference_grid((0.0, 0.0, 0.0, 2.0, 0.5, 0.5), 1 / 16, geometries=[("cuboid", 0.5, 0.1, -0.1, 0.7, 0.3, 0.2)],
                                  periodic=(False, True, False), noslip=("MZ", "PZ"),
                                  velocity=[("MX", 0.02, 0.0, 0.0)], pressure=[("PX", 0.0)], geometry_noslip=True)
    G = import_levels(lev, ifs, periodic=(False, True, False))
    g = G.levels[0]
    kinds = sorted(b.kind for b in g.bcs)
    assert kinds == ["geometry", "pressure", "velocity"]
    pr = [b for b in g.bcs if b.kind == "pressure"][0]
    assert pr.side == "PX" and pr.k.size > 0 and np.all(pr.rho == 0.0)
    # the pressure node's inward neighbour is one spacing in -x
    d = g.coords[:, pr.k] - g.coords[:, pr.k_neighbor]
    assert np.allclose(d[0], 1.0) and np.allclose(d[1:], 0.0)
    assert check_grid(g)["ok"]


def test_import_rejects_out_of_range_indices(ref):
    lev, ifs = _cavity_levels(ref, 1 / 8)
    lev[0]["neighbor"][0] = lev[0]["neighbor"][0].copy()
    lev[0]["neighbor"][0][5] = lev[0]["number_of_nodes"] + 3
    with pytest.raises(ValueError):
        import_levels(lev, ifs)
    lev, ifs = _cavity_levels(ref, 1 / 8)
    lev[0]["velocity"]["k"][0] = -1
    with pytest.raises(ValueError):
        import_levels(lev, ifs)
