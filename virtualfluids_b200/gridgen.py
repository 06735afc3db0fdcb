"""Levels built by the reference's own grid generator, imported.

The reference builds its grids with GridGenerator (MultipleGridBuilder: coarse box, refinement
boxes, STL or primitive geometries, side boundary conditions; src/gpu/GridGenerator) and hands
them to the solver through the GridBuilder getters that GridReaderGenerator/GridGenerator.cpp
:91-1020 calls level by level:

* getNodeValues: coordinates, neighborX/Y/Z (node 0 the dummy every missing neighbour points to),
  neighborInverse and typeOfGridNode of getNumberOfNodes(level) + 1 nodes;
* getFluidNodeIndices: the fluid nodes the collision runs over;
* getVelocityValues / getVelocityQs: the velocity BC list (every no-slip side of the builder is a
  zero-velocity entry of it, LevelGridBuilder.cpp:266-285);
* getPressureValues / getPressureQs / getPressureBoundaryConditionDirection: one pressure list per
  side, with the node one step inwards and the side's direction;
* getGeometryIndices / getGeometryQs / getGeometryValues: the geometry BC list;
* getGridInterfaceIndices / getOffsetCF / getOffsetFC: the interpolation cells between each level
  and the next finer one, with the offsets of cells that touch a wall.

:func:`import_levels` takes those arrays (a dict per level and per level pair) and returns an
:class:`ImportedGrid` that Simulation runs as it runs the grids of virtualfluids_b200.grid:
levels with the same attributes as ListGrid (neighbor, geo, fluid, number_of_nodes, coords, bcs,
merged) and the interfaces of MultiLevelGrid. Positions are in units of the coarsest spacing.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .grid import Interface, ListGrid, SideBC

# D3Q27 direction of a pressure side -> the side name the BC drivers use (Side.h:111-115)
_DIR_SIDE = {N.DIR_M00: "MX", N.DIR_P00: "PX", N.DIR_0M0: "MY", N.DIR_0P0: "PY", N.DIR_00M: "MZ", N.DIR_00P: "PZ"}


@dataclass
class ImportedLevel:
    """One level from the reference's grid builder, with ListGrid's attributes."""
    number_of_nodes: int
    neighbor: np.ndarray                 # uint32 [3, n]
    geo: np.ndarray                      # uint32 [n]
    fluid: np.ndarray                    # uint32 fluid node indices
    coords: np.ndarray                   # float64 [3, n] positions in units of the coarsest spacing
    delta: float                         # node spacing in the builder's length unit
    bcs: list = field(default_factory=list)
    neighbor_inverse: np.ndarray | None = None
    periodic: tuple = (False, False, False)
    align: int = 1
    first_node: int = 1

    merged = ListGrid.merged


@dataclass
class ImportedGrid:
    """Levels and interfaces in the form Simulation takes (MultiLevelGrid's attributes)."""
    levels: list
    interfaces: list
    spacing: list                        # spacing of each level in units of the coarsest spacing

    @property
    def origin(self):
        return [np.zeros(3) for _ in self.levels]

    def positions(self, level):
        return self.levels[level].coords


def _flat_q(q27, n):
    q = np.asarray(q27, dtype=np.float64).reshape(27, n)
    return np.ascontiguousarray(q)


def _level(d, delta0, periodic):
    n = int(d["number_of_nodes"])
    nb = np.stack([np.asarray(d["neighbor"][a], dtype=np.uint32).reshape(n) for a in range(3)])
    geo = np.asarray(d["geo"], dtype=np.uint32).reshape(n)
    fluid = np.asarray(d["fluid"], dtype=np.uint32).reshape(-1)
    if nb.max(initial=0) >= n or (fluid.size and fluid.max() >= n):
        raise ValueError("a neighbour or fluid-node index lies beyond the level's node count")
    if fluid.size and np.any(geo[fluid] != N.GEO_FLUID):
        raise ValueError("the fluid-node list names nodes whose type is not GEO_FLUID")
    coords = np.stack([np.asarray(d["coords"][a], dtype=np.float64).reshape(n) for a in range(3)]) / delta0
    bcs = []
    vel = d.get("velocity")
    if vel is not None and len(vel["k"]):
        k = np.asarray(vel["k"], dtype=np.int32)
        v = np.stack([np.asarray(vel[c], dtype=np.float64) for c in ("vx", "vy", "vz")])
        bcs.append(SideBC(side="builder_velocity", kind="velocity", k=k, q=_flat_q(vel["q27"], k.size), velocity=v))
    for p in d.get("pressure", []):
        k = np.asarray(p["k"], dtype=np.int32)
        if not k.size:
            continue
        bcs.append(SideBC(side=_DIR_SIDE[int(p["direction"])], kind="pressure", k=k, q=_flat_q(p["q27"], k.size),
                          rho=np.asarray(p["rho"], dtype=np.float64),
                          k_neighbor=np.asarray(p["k_neighbor"], dtype=np.int32)))
    geom = d.get("geometry")
    if geom is not None and len(geom["k"]):
        k = np.asarray(geom["k"], dtype=np.int32)
        v = np.stack([np.asarray(geom.get(c, np.zeros(k.size)), dtype=np.float64) for c in ("vx", "vy", "vz")])
        bcs.append(SideBC(side="builder_geometry", kind="geometry", k=k, q=_flat_q(geom["q27"], k.size), velocity=v))
    for b in bcs:
        if b.k.size and (b.k.min() < 0 or b.k.max() >= n):
            raise ValueError(f"{b.kind} BC node index beyond the level's node count")
    inv = d.get("neighbor_inverse")
    return ImportedLevel(number_of_nodes=n, neighbor=nb, geo=geo, fluid=fluid, coords=coords, delta=float(d["delta"]),
                         bcs=bcs, neighbor_inverse=None if inv is None else np.asarray(inv, dtype=np.uint32),
                         periodic=tuple(bool(x) for x in periodic))


def import_levels(levels, interfaces=(), periodic=(False, False, False)):
    """An ImportedGrid from the arrays of the reference's GridBuilder getters.

    levels: per level a dict with number_of_nodes (getNumberOfNodes + 1), delta, coords (3 arrays),
    neighbor (3 arrays), geo, fluid, and optionally neighbor_inverse, velocity {k, vx, vy, vz,
    q27 [27 * n]}, pressure [{k, k_neighbor, rho, direction, q27}], geometry {k, q27, vx, vy, vz}.
    interfaces: per pair of levels (l, l + 1) a dict with cf_coarse, cf_fine, fc_coarse, fc_fine and
    offsets_cf, offsets_fc ((3, n) each), as getGridInterfaceIndices / getOffsetCF / getOffsetFC
    give them. Indices are checked against each level's node count."""
    if not levels:
        raise ValueError("no levels")
    delta0 = float(levels[0]["delta"])
    lv = [_level(d, delta0, periodic) for d in levels]
    ifs = []
    for l, d in enumerate(interfaces):
        c, f = lv[l], lv[l + 1]
        arr = {k: np.asarray(d[k], dtype=np.uint32).reshape(-1) for k in ("cf_coarse", "cf_fine", "fc_coarse", "fc_fine")}
        for key, level in (("cf_coarse", c), ("fc_coarse", c), ("cf_fine", f), ("fc_fine", f)):
            if arr[key].size and arr[key].max() >= level.number_of_nodes:
                raise ValueError(f"interface {l}: {key} index beyond the level's node count")
        off_cf = np.asarray(d["offsets_cf"], dtype=np.float64).reshape(3, arr["cf_coarse"].size)
        off_fc = np.asarray(d["offsets_fc"], dtype=np.float64).reshape(3, arr["fc_coarse"].size)
        ifs.append(Interface(coarse_cf=arr["cf_coarse"], fine_cf=arr["cf_fine"], coarse_fc=arr["fc_coarse"],
                             fine_fc=arr["fc_fine"], offsets_cf=off_cf, offsets_fc=off_fc))
    return ImportedGrid(levels=lv, interfaces=ifs, spacing=[l.delta / delta0 for l in lv])
