"""Host-side checks of the esoteric-twist write pattern of a level (no GPU needed).

In esoteric-twist streaming (src/gpu/core/Utilities/KernelUtilities.h:66-378) a node reads each
population from a slot -- an array plane and a node index reached through the +1 neighbours of
neighborX/Y/Z -- and writes its post-collision population back into the slot it read from. The
update is race free only if every slot of a step is written by exactly one node: two fluid nodes
that reach the same slot overwrite each other's populations. The boundary-condition kernels write
the populations of the next step into the slots of the next parity, and the pressure kernels the
current step's, so a slot written twice by two entries of the lists (or by two lists) makes the
result depend on the launch order.

These checks compute every written slot on the host with numpy and report the slots written more
than once. The dummy node 0, the sink every missing neighbour points to, is exempt: its slots are
written by many nodes and never read as data. They are meant for grids built or imported by hand
and for caller-supplied BC lists, before they reach the kernels.
"""
from __future__ import annotations

import numpy as np

# D3Q27 numbering (src/lbm/constants/D3Q27.h:42-72)
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1])
INV = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 26, 25, 24, 23, 22, 21, 20, 19])
# shift class of a direction: bit 0 = +1 in x, bit 1 = +1 in y, bit 2 = +1 in z (negative components)
SHIFT = (CX < 0).astype(int) | ((CY < 0).astype(int) << 1) | ((CZ < 0).astype(int) << 2)


def slot_nodes(neighbor, nodes):
    """(8, n) the eight slot nodes of `nodes` by shift class: k, kx, ky, kxy, kz, kxz, kyz, kxyz
    (ListIndices, KernelUtilities.h:221-250)."""
    nbx, nby, nbz = (np.asarray(a, dtype=np.int64) for a in neighbor)
    k = np.asarray(nodes, dtype=np.int64)
    kx, ky, kz = nbx[k], nby[k], nbz[k]
    kxy = nby[kx]
    return np.stack([k, kx, ky, kxy, kz, nbz[kx], nbz[ky], nbz[kxy]])


def plane(d, even):
    """array plane holding direction d on an even / odd step (getPointersToDistributions)"""
    return np.where(even, d, INV[d])


def collision_slots(neighbor, fluid, n_nodes, even):
    """flat slot index plane * n_nodes + node of every (fluid node, direction) the collision writes
    (setPostCollisionDistribution writes into the slots getPreCollisionDistribution read): (27, n)"""
    sn = slot_nodes(neighbor, fluid)
    d = np.arange(27)
    return plane(d, even)[:, None] * np.int64(n_nodes) + sn[SHIFT[d]]


def bc_slots(neighbor, k, q27, n_nodes, even):
    """slots the post-collision BC kernels write for one list: for every link d with q in [0, 1],
    the population of inv(d) of the next step at the node (NoSlipBounceBack.cu:44-179 and the
    interpolated / velocity variants)"""
    k = np.asarray(k, dtype=np.int64)
    q = np.asarray(q27, dtype=np.float64).reshape(27, -1)
    sn = slot_nodes(neighbor, k)
    di, ii = np.nonzero((q >= 0.0) & (q <= 1.0))
    keep = di > 0
    di, ii = di[keep], ii[keep]
    e = INV[di]
    return plane(e, not even) * np.int64(n_nodes) + sn[SHIFT[e], ii]


def pressure_slots(neighbor, k, direction, n_nodes, even):
    """slots PressureNonEquilibriumCompressible_Device writes at its nodes: the 18 populations whose
    component along the outlet axis is not the outlet's own sign (PressureNonEquilibriumCompressible
    .cu:179-310)"""
    k = np.asarray(k, dtype=np.int64)
    axis = 0 if CX[direction] else (1 if CY[direction] else 2)
    comp = (CX, CY, CZ)[axis]
    sgn = comp[direction]
    d = np.nonzero(comp != sgn)[0]
    sn = slot_nodes(neighbor, k)
    return (plane(d, even)[:, None] * np.int64(n_nodes) + sn[SHIFT[d]]).reshape(-1)


def _duplicates(slots, n_nodes):
    s = np.asarray(slots, dtype=np.int64).reshape(-1)
    s = s[s % np.int64(n_nodes) != 0]                 # the dummy node 0 takes any number of writes
    u, c = np.unique(s, return_counts=True)
    dup = u[c > 1]
    return [(int(x // n_nodes), int(x % n_nodes)) for x in dup[:20]], int(dup.size)


def check_level(neighbor, fluid, n_nodes, bc_lists=(), pressure_lists=()):
    """The slots written twice in one step of a level, for both parities.

    bc_lists: (name, k, q27[27 * n]) of the post-collision lists (velocity, no-slip, geometry) in the
    order they run; pressure_lists: (name, k, direction). Returns a report dict; its "ok" is True
    when no slot except the dummy node's is written twice: by the collision, within one BC list,
    across the post-collision lists, or across the pressure lists. Each entry lists up to 20 of the
    offending (plane, node) slots and their count."""
    report = {"ok": True}
    for even in (True, False):
        tag = "even" if even else "odd"
        slots, count = _duplicates(collision_slots(neighbor, fluid, n_nodes, even), n_nodes)
        report[f"collision_{tag}"] = {"duplicates": count, "slots": slots}
        every = []
        for name, k, q in bc_lists:
            s = bc_slots(neighbor, k, q, n_nodes, even)
            every.append(s)
            slots, count = _duplicates(s, n_nodes)
            report[f"{name}_{tag}"] = {"duplicates": count, "slots": slots}
        if every:
            slots, count = _duplicates(np.concatenate(every), n_nodes)
            report[f"post_collision_lists_{tag}"] = {"duplicates": count, "slots": slots}
        if pressure_lists:
            s = np.concatenate([pressure_slots(neighbor, k, direction, n_nodes, even)
                                for _, k, direction in pressure_lists])
            slots, count = _duplicates(s, n_nodes)
            report[f"pressure_lists_{tag}"] = {"duplicates": count, "slots": slots}
    report["ok"] = all(v["duplicates"] == 0 for key, v in report.items() if key != "ok")
    return report


def check_grid(grid):
    """check_level for a ListGrid with its merged BC lists (velocity, no-slip, geometry) and its
    pressure sides."""
    from .grid import SIDE_DIR
    lists = []
    for kind in ("velocity", "noslip", "geometry"):
        m = grid.merged(kind)
        if m is not None:
            lists.append((kind, m[0], m[1]))
    pressure = [(f"pressure_{b.side}", b.k, SIDE_DIR[b.side]) for b in grid.bcs if b.kind == "pressure"]
    return check_level(grid.neighbor, grid.fluid, grid.number_of_nodes, lists, pressure)


def assert_slots_written_once(grid):
    """Raises ValueError naming the first conflicts when check_grid finds any."""
    r = check_grid(grid)
    if not r["ok"]:
        bad = {k: v for k, v in r.items() if k != "ok" and v["duplicates"]}
        raise ValueError(f"esoteric-twist slots written more than once in a step: {bad}")
    return r
