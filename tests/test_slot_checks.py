"""Host checker of the esoteric-twist write pattern (virtualfluids_b200.checks): every grid the
builders make writes each slot once per step (collision, BC lists, pressure lists, both parities),
and corrupted neighbour lists or duplicated BC entries are reported."""
import numpy as np
import pytest

from virtualfluids_b200 import ListGrid, MultiLevelGrid
from virtualfluids_b200.checks import assert_slots_written_once, check_grid, check_level


def _cavity(n=8):
    g = ListGrid(n, n + 1, n - 1)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    return g


def _channel():
    g = ListGrid(24, 12, 12, periodic=(False, True, False))
    g.add_side("MZ", "noslip")
    g.add_side("PZ", "noslip")
    g.add_side("MX", "velocity", velocity=(0.02, 0.0, 0.0))
    g.add_side("PX", "pressure", rho=0.0)
    g.add_box_obstacle((7.3, 3.6, -0.5), (11.6, 7.8, 4.4))
    return g


@pytest.mark.parametrize("make", [_cavity, _channel, lambda: ListGrid(7, 6, 5, periodic=(True, True, True)),
                                  lambda: ListGrid(16, 16, 16, periodic=(True, True, True), align=32)],
                         ids=["cavity", "channel_obstacle_pressure", "periodic", "periodic_aligned"])
def test_builder_grids_write_every_slot_once(make):
    g = make()
    r = assert_slots_written_once(g)
    assert r["ok"]
    assert r["collision_even"]["duplicates"] == 0 and r["collision_odd"]["duplicates"] == 0


def test_refined_levels_write_every_slot_once():
    m = MultiLevelGrid.uniform(ListGrid(12, 12, 12, periodic=(True, True, True)))
    m.refine((3, 3, 3), (9, 9, 9))
    for g in m.levels:
        assert check_grid(g)["ok"]


def test_corrupted_neighbour_list_is_reported():
    g = ListGrid(6, 5, 4, periodic=(True, True, True))
    nb = [a.copy() for a in g.neighbor]
    a, b = int(g.fluid[3]), int(g.fluid[10])
    nb[0][a] = nb[0][b]                               # two nodes now reach the same +x node
    r = check_level(nb, g.fluid, g.number_of_nodes)
    assert not r["ok"]
    assert r["collision_even"]["duplicates"] > 0 and r["collision_odd"]["duplicates"] > 0
    plane, node = r["collision_even"]["slots"][0]
    assert node == nb[0][b] or node in (nb[1][nb[0][b]], nb[2][nb[0][b]], nb[2][nb[1][nb[0][b]]])


def test_duplicated_bc_entry_and_overlapping_lists_are_reported():
    g = _cavity()
    k, q, _ = g.merged("noslip")
    k2 = np.concatenate([k, k[:1]])
    q2 = np.concatenate([q.reshape(27, -1), q.reshape(27, -1)[:, :1]], axis=1)
    r = check_level(g.neighbor, g.fluid, g.number_of_nodes, [("noslip", k2, q2)])
    assert not r["ok"] and r["noslip_even"]["duplicates"] > 0
    # the same node in two lists with a common cut link: the later list would overwrite the earlier
    kv, qv, _ = g.merged("velocity")
    r = check_level(g.neighbor, g.fluid, g.number_of_nodes, [("velocity", kv, qv), ("noslip", kv[:2], qv.reshape(27, -1)[:, :2])])
    assert r["velocity_even"]["duplicates"] == 0 and r["noslip_even"]["duplicates"] == 0
    assert r["post_collision_lists_even"]["duplicates"] > 0 and not r["ok"]
    with pytest.raises(ValueError):
        g.bcs.append(g.bcs[0])                        # a side added twice
        assert_slots_written_once(g)
