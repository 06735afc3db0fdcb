"""Host-side construction of levels in the reference GPU layout.

A box of fluid nodes is laid out as the reference's GridGenerator lays out a uniform grid
(src/gpu/GridGenerator/grid/GridImp.cpp):

* sparse node list in x-fastest order, shifted by one so that node 0 is the dummy sink that
  every missing neighbour points to (GridImp.cpp:974, getNodeValues :2146-2185); with align > 1
  the grid starts at node `align` instead and the node count is padded to a multiple of it (the
  unused nodes are solid and point nowhere), so every direction plane and every x-row of a box
  whose row length is a multiple of `align` starts on an aligned boundary;
* a one-node layer of stopper nodes around the fluid on every non-periodic side; stoppers are
  in the node list but never collided (geo GEO_VOID, as getNodeValues marks every non-fluid node);
* neighborX/Y/Z[k] = the node at +1 in x/y/z, wrapped on periodic axes (setNeighborIndices
  :1012-1032, getNeighborIndex :1071-1080); stoppers get their in-grid +1 neighbours only
  (setStopperNeighborCoords :1034-1057);
* boundary-condition nodes are the fluid nodes of the outermost fluid layer of a side, with
  q = 1/2 on every link that points along the side normal into a stopper, and q = -1 elsewhere
  (Side::setQs, Side.cpp:149-167); a diagonal link already owned by a side set earlier is not
  repeated (Side::resetDiagonalsInCaseOfOtherBC, Side.cpp:185-210);
* pressure BC nodes carry the index of the node one step inwards (Side::setPressureNeighborIndices,
  Side.cpp:89-110) and the side's D3Q27 direction (LevelGridBuilder.cpp:721-724).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _native as N

# D3Q27 components in reference numbering (src/lbm/constants/D3Q27.h:42-72)
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1])
INV = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 26, 25, 24, 23, 22, 21, 20, 19])
W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)

# side name -> (axis, sign); D3Q27 direction of the side (Side.h:111-115)
SIDES = {"MX": (0, -1), "PX": (0, 1), "MY": (1, -1), "PY": (1, 1), "MZ": (2, -1), "PZ": (2, 1)}
SIDE_DIR = {"MX": N.DIR_M00, "PX": N.DIR_P00, "MY": N.DIR_0M0, "PY": N.DIR_0P0, "MZ": N.DIR_00M, "PZ": N.DIR_00P}


@dataclass
class SideBC:
    side: str
    kind: str                       # "noslip", "velocity", "slip", "pressure", "geometry"
    k: np.ndarray                   # int32 node indices
    q: np.ndarray                   # float64 [27, n]
    velocity: tuple | np.ndarray = (0.0, 0.0, 0.0)   # constant, or (3, n) per node
    rho: float = 0.0
    k_neighbor: np.ndarray | None = None


def inverse_neighbors(neighbor: np.ndarray) -> np.ndarray:
    """neighborInverse from the +1 neighbour lists (uint32 [3, n]) of any grid: the node m whose +x,
    then +y, then +z neighbour is k becomes inv[k]. Chains that end at the dummy node 0 are dropped,
    and nodes that no chain reaches keep 0."""
    nbx, nby, nbz = (np.asarray(neighbor[a], dtype=np.int64) for a in range(3))
    n = nbx.size
    m = np.arange(1, n, dtype=np.int64)
    a = nbx[m]
    b = np.where(a != 0, nby[a], 0)
    target = np.where(b != 0, nbz[b], 0)
    ok = target != 0
    inv = np.zeros(n, dtype=np.uint32)
    inv[target[ok]] = m[ok].astype(np.uint32)
    return inv


@dataclass
class ListGrid:
    """One level of a fluid box nx*ny*nz in the reference layout (see module docstring)."""
    nx: int
    ny: int
    nz: int
    periodic: tuple = (False, False, False)
    number_of_nodes: int = 0
    neighbor: np.ndarray | None = None      # uint32 [3, n]
    geo: np.ndarray | None = None           # uint32 [n]
    fluid: np.ndarray | None = None         # uint32 fluid node indices
    coords: np.ndarray | None = None        # int64 [3, n] fluid-box coordinates (shell at -1 / n)
    bcs: list = field(default_factory=list)
    align: int = 1                          # > 1: grid nodes start at index `align`, planes padded to it

    def __post_init__(self):
        self.shell = tuple(0 if p else 1 for p in self.periodic)
        self.dims = (self.nx + 2 * self.shell[0], self.ny + 2 * self.shell[1], self.nz + 2 * self.shell[2])
        Dx, Dy, Dz = self.dims
        n_grid = Dx * Dy * Dz
        # node 0 is the dummy; with align > 1 the unused nodes 1 .. align - 1 put the grid's first
        # node, and the padded node count every direction plane, on a multiple of `align` nodes
        a0 = int(self.align)
        self.first_node = a0 if a0 > 1 else 1
        self.number_of_nodes = (self.first_node + n_grid + a0 - 1) // a0 * a0 if a0 > 1 else n_grid + 1
        g0, g1 = self.first_node, self.first_node + n_grid
        i = np.arange(n_grid, dtype=np.int64)
        gx, gy, gz = i % Dx, (i // Dx) % Dy, i // (Dx * Dy)
        # coordinates in fluid-box units: fluid nodes 0..n-1, shell at -1 and n
        coords = np.full((3, self.number_of_nodes), -(10 ** 9), dtype=np.int64)
        coords[0, g0:g1] = gx - self.shell[0]
        coords[1, g0:g1] = gy - self.shell[1]
        coords[2, g0:g1] = gz - self.shell[2]
        self.coords = coords
        fluid_mask = np.zeros(self.number_of_nodes, dtype=bool)
        c = coords[:, g0:g1]
        fluid_mask[g0:g1] = ((c[0] >= 0) & (c[0] < self.nx) & (c[1] >= 0) & (c[1] < self.ny)
                             & (c[2] >= 0) & (c[2] < self.nz))
        self.geo = np.where(fluid_mask, N.GEO_FLUID, N.GEO_VOID).astype(np.uint32)
        self.fluid = np.nonzero(fluid_mask)[0].astype(np.uint32)
        nb = np.zeros((3, self.number_of_nodes), dtype=np.uint32)
        g = [gx, gy, gz]
        for a in range(3):
            nxt = g[a] + 1
            if self.periodic[a]:
                nxt = np.where(nxt >= self.dims[a], 0, nxt)
                ok = np.ones_like(nxt, dtype=bool)
            else:
                ok = nxt < self.dims[a]
            comp = list(g)
            comp[a] = np.where(ok, nxt, 0)
            idx = comp[0] + Dx * (comp[1] + Dy * comp[2]) + g0
            nb[a, g0:g1] = np.where(ok, idx, 0).astype(np.uint32)
        self.neighbor = nb
        self._bc_sides_set = []

    @property
    def neighbor_inverse(self) -> np.ndarray:
        """neighborInverse (uint32 [n]): per node the node at -1 in x, y and z, wrapping on periodic
        axes; 0 (the dummy node) where there is none. Made on first use."""
        inv = getattr(self, "_neighbor_inverse", None)
        if inv is None:
            Dx, Dy, Dz = self.dims
            n_grid = Dx * Dy * Dz
            g0 = self.first_node
            i = np.arange(n_grid, dtype=np.int64)
            g = [i % Dx, (i // Dx) % Dy, i // (Dx * Dy)]
            ok = np.ones(n_grid, dtype=bool)
            prev = []
            for a in range(3):
                p = g[a] - 1
                if self.periodic[a]:
                    p = np.where(p < 0, self.dims[a] - 1, p)
                else:
                    ok &= p >= 0
                prev.append(p)
            idx = prev[0] + Dx * (prev[1] + Dy * prev[2]) + g0
            inv = np.zeros(self.number_of_nodes, dtype=np.uint32)
            inv[g0:g0 + n_grid] = np.where(ok, idx, 0).astype(np.uint32)
            self._neighbor_inverse = inv
        return inv

    # -- indexing ----------------------------------------------------------------------------
    def node_index(self, x, y, z):
        """Node index of fluid-box coordinates (shell allowed on non-periodic axes)."""
        Dx, Dy, _ = self.dims
        gx = np.asarray(x) + self.shell[0]
        gy = np.asarray(y) + self.shell[1]
        gz = np.asarray(z) + self.shell[2]
        return (gx + Dx * (gy + Dy * gz) + self.first_node).astype(np.int64)

    def is_stopper(self, x, y, z):
        inside = ((x >= 0) & (x < self.nx) & (y >= 0) & (y < self.ny) & (z >= 0) & (z < self.nz))
        return ~inside

    # -- boundary conditions (Side::addIndices / setQs) ---------------------------------------
    def _side_nodes(self, side):
        axis, sign = SIDES[side]
        if self.periodic[axis]:
            raise ValueError(f"side {side} lies on a periodic axis")
        ext = (self.nx, self.ny, self.nz)
        layer = ext[axis] - 1 if sign > 0 else 0
        sel = self.fluid[self.coords[axis, self.fluid] == layer]
        return sel.astype(np.int64)

    def _neighbour_coords(self, x, y, z, d):
        nx_, ny_, nz_ = x + CX[d], y + CY[d], z + CZ[d]
        # Side::correctNeighborForPeriodicBoundaries: wrap on periodic axes
        if self.periodic[0]:
            nx_ = nx_ % self.nx
        if self.periodic[1]:
            ny_ = ny_ % self.ny
        if self.periodic[2]:
            nz_ = nz_ % self.nz
        return nx_, ny_, nz_

    def add_side(self, side, kind, velocity=(0.0, 0.0, 0.0), rho=0.0):
        """Set a BC on a side, in the order the reference's app sets them. velocity may be a
        function of the side nodes' fluid-box coordinates (x, y, z) returning (ux, uy, uz) arrays."""
        axis, sign = SIDES[side]
        nodes = self._side_nodes(side)
        x, y, z = self.coords[0, nodes], self.coords[1, nodes], self.coords[2, nodes]
        if callable(velocity):
            velocity = np.array([np.broadcast_to(np.asarray(c, dtype=np.float64), x.shape) for c in velocity(x, y, z)])
        q = np.full((27, nodes.size), -1.0)
        normal = np.zeros(3, dtype=int)
        normal[axis] = sign
        for d in range(1, 27):
            c = np.array([CX[d], CY[d], CZ[d]])
            if c @ normal <= 0:
                continue
            stop = self.is_stopper(*self._neighbour_coords(x, y, z, d))
            qd = np.where(stop, 0.5, -1.0)
            # resetDiagonalsInCaseOfOtherBC: links along the normal of a side set before, on nodes
            # that lie on that side too, stay with the earlier side
            for other in self._bc_sides_set:
                oa, os_ = SIDES[other]
                onormal = np.zeros(3, dtype=int)
                onormal[oa] = os_
                if c @ onormal <= 0:
                    continue
                ocoords = [x.copy(), y.copy(), z.copy()]
                ocoords[oa] = ocoords[oa] + os_
                on_other = self.is_stopper(*ocoords)
                qd = np.where((qd == 0.5) & on_other, -1.0, qd)
            q[d] = qd
        vel = velocity if isinstance(velocity, np.ndarray) else tuple(velocity)
        bc = SideBC(side=side, kind=kind, k=nodes.astype(np.int32), q=q, velocity=vel, rho=rho)
        if kind == "pressure":
            inward = [x.copy(), y.copy(), z.copy()]
            inward[axis] = inward[axis] - sign
            bc.k_neighbor = self.node_index(*inward).astype(np.int32)
        self.bcs.append(bc)
        self._bc_sides_set.append(side)
        return bc

    # -- obstacles (GridImp::calculateQs, GridImp.cpp:1561) ---------------------------------
    def add_box_obstacle(self, lo, hi, kind="geometry"):
        """An axis-aligned solid box [lo, hi] (fluid-box coordinates; faces may lie between nodes).

        Nodes inside become solid and leave the fluid list. Every fluid node with a link d whose
        end node lies inside gets q_d = the ray parameter t in (0, 1] at which p + t c_d enters the
        box (exact ray-box intersection); such nodes form a BC list of the given kind, by default
        the geometry BC (Parameter's geometryBC)."""
        lo = np.asarray(lo, dtype=np.float64)
        hi = np.asarray(hi, dtype=np.float64)
        c = self.coords.astype(np.float64)
        inside = np.ones(self.number_of_nodes, dtype=bool)
        for a in range(3):
            inside &= (c[a] >= lo[a]) & (c[a] <= hi[a])
        inside[0] = False
        was_fluid = self.geo == N.GEO_FLUID
        solid = inside & was_fluid
        self.geo = np.where(solid, N.GEO_VOID, self.geo).astype(np.uint32)
        self.fluid = np.nonzero(self.geo == N.GEO_FLUID)[0].astype(np.uint32)
        for b in self.bcs:
            keep = ~solid[b.k]
            b.k, b.q = b.k[keep], b.q[:, keep]
            if b.k_neighbor is not None:
                b.k_neighbor = b.k_neighbor[keep]
        near = np.ones(self.fluid.size, dtype=bool)
        for a in range(3):
            ca = self.coords[a, self.fluid]
            near &= (ca >= np.floor(lo[a]) - 1) & (ca <= np.ceil(hi[a]) + 1)
        if any(self.periodic):
            near[:] = True          # wrapped neighbours can reach the box from the far side
        nodes = self.fluid[near].astype(np.int64)
        x, y, z = (self.coords[a, nodes] for a in range(3))
        q = np.full((27, nodes.size), -1.0)
        for d in range(1, 27):
            ex, ey, ez = self._neighbour_coords(x, y, z, d)
            hit = (ex >= lo[0]) & (ex <= hi[0]) & (ey >= lo[1]) & (ey <= hi[1]) & (ez >= lo[2]) & (ez <= hi[2])
            if not hit.any():
                continue
            t = np.zeros(nodes.size)
            for a, (p, cd) in enumerate(((x, CX[d]), (y, CY[d]), (z, CZ[d]))):
                if cd == 0:
                    continue
                face = lo[a] if cd > 0 else hi[a]
                ta = (face - p) / cd
                t = np.maximum(t, np.where((p < lo[a]) | (p > hi[a]), ta, 0.0))
            q[d] = np.where(hit, np.clip(t, 0.0, 1.0), -1.0)
        cut = (q >= 0).any(axis=0)
        bc = SideBC(side="obstacle", kind=kind, k=nodes[cut].astype(np.int32), q=q[:, cut])
        self.bcs.append(bc)
        return bc

    def add_sphere_obstacle(self, centre, radius, kind="geometry"):
        """A solid sphere (fluid-box coordinates). Nodes with |p - centre| <= radius become solid and
        leave the fluid list; every fluid node with a link that enters the sphere within one link
        length gets that link's q (Sphere::getIntersection, geometries/Sphere/Sphere.cpp:124-169, the
        smallest non-negative root kept when 0 <= q <= 1, GridImp::calculateQs, GridImp.cpp:1561-1600).
        Those nodes form a BC list of the given kind. Periodic images of the sphere are not added."""
        from .workloads import sphere_link_q
        c = np.asarray(centre, dtype=np.float64)
        r = float(radius)
        pos = self.coords.astype(np.float64)
        d2 = ((pos - c[:, None]) ** 2).sum(axis=0)
        inside = d2 <= r * r
        inside[0] = False
        solid = inside & (self.geo == N.GEO_FLUID)
        self.geo = np.where(solid, N.GEO_VOID, self.geo).astype(np.uint32)
        self.fluid = np.nonzero(self.geo == N.GEO_FLUID)[0].astype(np.uint32)
        for b in self.bcs:
            keep = ~solid[b.k]
            b.k, b.q = b.k[keep], b.q[:, keep]
            if b.k_neighbor is not None:
                b.k_neighbor = b.k_neighbor[keep]
        near = self.fluid[d2[self.fluid] <= (r + 1.8) ** 2].astype(np.int64)
        q = sphere_link_q(pos[:, near].T, c, r)
        cut = (q >= 0).any(axis=0)
        bc = SideBC(side="obstacle", kind=kind, k=near[cut].astype(np.int32), q=q[:, cut])
        self.bcs.append(bc)
        return bc

    def merged(self, kind):
        """All BCs of one kind concatenated, as allocArrays_BoundaryValues fills one struct per kind."""
        parts = [b for b in self.bcs if b.kind == kind]
        if not parts:
            return None
        k = np.concatenate([b.k for b in parts])
        q = np.concatenate([b.q for b in parts], axis=1)
        vel = np.concatenate([np.asarray(b.velocity, dtype=np.float64) if isinstance(b.velocity, np.ndarray)
                              else np.tile(np.array(b.velocity, dtype=np.float64)[:, None], (1, b.k.size))
                              for b in parts], axis=1)
        return k, q, vel


# -- refinement (GridGenerator/grid/GridInterface.cpp) ------------------------------------------
@dataclass
class Interface:
    """The interpolation cells between a coarse level and the fine level nested in it, as the
    reference's GridInterface finds them and LevelGridBuilder hands them to the coarse level's
    fineToCoarse / coarseToFine (ICells) and neighborFineToCoarse / neighborCoarseToFine (ICellNeigh).

    coarse to fine: coarse_cf is the MMM corner of each coarse cell, fine_cf the MMM one of the
    eight fine nodes inside it; fine to coarse: coarse_fc is the coarse node at the centre of each
    fine cell, fine_fc that cell's MMM fine node. Offsets are (3, n), zero for cells whose corners
    are all fluid (findOffsetCF / findOffsetFC give direction 000 there)."""
    coarse_cf: np.ndarray
    fine_cf: np.ndarray
    coarse_fc: np.ndarray
    fine_fc: np.ndarray
    offsets_cf: np.ndarray
    offsets_fc: np.ndarray


@dataclass
class MultiLevelGrid:
    """Nested levels: levels[0] is the coarsest; levels[l + 1] covers a box of levels[l] at half
    the spacing; interfaces[l] couples levels l and l + 1. origin[l] and spacing[l] place fluid node
    (0, 0, 0) of level l and its node distance in units of the coarsest spacing."""
    levels: list
    interfaces: list
    origin: list
    spacing: list

    @classmethod
    def uniform(cls, grid: ListGrid):
        return cls([grid], [], [np.zeros(3)], [1.0])

    def refine(self, lo, hi):
        """Add a finer level over the cells [lo, hi) (per axis, fluid-box coordinates of the
        currently finest level) and return it."""
        fine, iface = refine_box(self.levels[-1], lo, hi)
        h = self.spacing[-1]
        self.origin.append(self.origin[-1] + (np.asarray(lo, dtype=np.float64) + 0.25) * h)
        self.spacing.append(h / 2.0)
        self.levels.append(fine)
        self.interfaces.append(iface)
        return fine

    def positions(self, level):
        """(3, number_of_nodes) node positions of a level in units of the coarsest spacing."""
        g = self.levels[level]
        return self.origin[level][:, None] + g.coords.astype(np.float64) * self.spacing[level]


def refine_box(coarse: ListGrid, lo, hi):
    """A fine level over the coarse cells [lo, hi) of `coarse` and the interpolation cells between
    them, by the rules of GridInterface (GridInterface.cpp:59-205) for a refined box whose
    interface lies in the fluid:

    * fine nodes sit at coarse positions + 1/4 + i/2 (getCoarseToFineIndexOnFineGrid,
      getFineToCoarseIndexOnFineGrid :237-257), a 2(hi - lo) cube per axis with a stopper shell;
    * coarse-to-fine cells (findInterfaceCF :59-90) are the coarse cells of the box whose
      27-neighbourhood leaves it: its outer cell layer. Their corners are the CFC nodes
      [lo, hi]^3 minus [lo + 2, hi - 2]^3, and their fine nodes the fine level's two outer layers;
    * fine-to-coarse cells (findInterfaceFC :125-157) are centred on the coarse nodes next to a
      CFC node that are not CFC themselves: the shell of [lo + 2, hi - 2]^3;
    * coarse nodes under the fine level that are neither (findOverlapStopper :159-205: the
      stopper shell and the nodes removed below it) leave the coarse level's fluid-node list.

    lo and hi must keep the interface two nodes away from the coarse level's edges and leave at
    least four cells: 2 <= lo, lo + 4 <= hi <= n - 3 on every axis."""
    lo = np.asarray(lo, dtype=np.int64)
    hi = np.asarray(hi, dtype=np.int64)
    ext = np.array([coarse.nx, coarse.ny, coarse.nz])
    if lo.shape != (3,) or hi.shape != (3,):
        raise ValueError("lo and hi are three cell coordinates")
    if (lo < 2).any() or (hi > ext - 3).any() or (hi - lo < 4).any():
        raise ValueError("the refined box needs 2 <= lo, lo + 4 <= hi <= n - 3 on every axis")
    c = coarse.coords
    fluid = coarse.geo == N.GEO_FLUID
    box = [(c[a] >= lo[a]) & (c[a] <= hi[a]) for a in range(3)]
    inner2 = [(c[a] >= lo[a] + 2) & (c[a] <= hi[a] - 2) for a in range(3)]
    inner3 = [(c[a] >= lo[a] + 3) & (c[a] <= hi[a] - 3) for a in range(3)]
    in_box = box[0] & box[1] & box[2]
    in2 = inner2[0] & inner2[1] & inner2[2]
    in3 = inner3[0] & inner3[1] & inner3[2]
    if not fluid[in_box].all():
        raise ValueError("the refined box must lie in the fluid")
    fine = ListGrid(int(2 * (hi[0] - lo[0])), int(2 * (hi[1] - lo[1])), int(2 * (hi[2] - lo[2])),
                    periodic=(False, False, False))
    # coarse-to-fine: cells (MMM corner c) in [lo, hi - 1]^3 on the outer layer
    cells = [(c[a] >= lo[a]) & (c[a] <= hi[a] - 1) for a in range(3)]
    cell_in = cells[0] & cells[1] & cells[2]
    shell = np.zeros_like(cell_in)
    for a in range(3):
        shell |= (c[a] == lo[a]) | (c[a] == hi[a] - 1)
    cf_coarse = np.nonzero(cell_in & shell)[0]
    cf_fine = fine.node_index(*(2 * (c[a, cf_coarse] - lo[a]) for a in range(3)))
    # fine-to-coarse: the shell of [lo + 2, hi - 2]^3
    shell2 = np.zeros_like(in2)
    for a in range(3):
        shell2 |= (c[a] == lo[a] + 2) | (c[a] == hi[a] - 2)
    fc_coarse = np.nonzero(in2 & shell2)[0]
    fc_fine = fine.node_index(*(2 * (c[a, fc_coarse] - lo[a]) - 1 for a in range(3)))
    # the coarse nodes below the fine-to-coarse shell are not collided any more
    keep = np.ones(coarse.number_of_nodes, dtype=bool)
    keep[in3] = False
    coarse.fluid = coarse.fluid[keep[coarse.fluid]]
    iface = Interface(coarse_cf=cf_coarse.astype(np.uint32), fine_cf=cf_fine.astype(np.uint32),
                      coarse_fc=fc_coarse.astype(np.uint32), fine_fc=fc_fine.astype(np.uint32),
                      offsets_cf=np.zeros((3, cf_coarse.size)), offsets_fc=np.zeros((3, fc_coarse.size)))
    return fine, iface
