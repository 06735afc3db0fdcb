"""Synthetic workloads with the shapes of the benchmark configurations, and their analytic checks.

* :func:`tgv_fields` — Taylor-Green vortex initial fields on a periodic box (the reference's TGV
  app, apps/gpu/TaylorGreenVortex, on [-pi, pi]^3);
* :func:`duct_batch` — rectangular-duct Poiseuille domains of uneven sizes for the batched sweep,
  with :func:`duct_series` (steady) and :func:`duct_transient` (start-up from rest) profiles;
* :func:`porous_block` — a cube of random non-overlapping spheres at a target porosity, with the
  exact sphere q of every cut link, for the serving stream.

All generators are seeded; the analytic profiles follow from the mathematics of the problems
(eigenfunction series of the Poisson and heat equations on a rectangle).
"""
from __future__ import annotations

import math

import numpy as np

# K17 is unstable above this viscosity (a shear wave grows at nu = 0.04); Parameter warns above it
K17_NU_MAX = 1.0 / 42.0


def tgv_fields(n, u0, dtype=np.float64):
    """drho, ux, uy, uz (x fastest) of the Taylor-Green vortex on an n^3 periodic box."""
    x = (np.arange(n) + 0.5) / n * 2 * np.pi - np.pi
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    rho = 3.0 * (u0 * u0 / 16.0) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    ux = u0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    uy = -u0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    return [a.reshape(-1).astype(dtype) for a in (rho, ux, uy, np.zeros_like(ux))]


def _duct_axes(ny, nz):
    """Half-widths and node coordinates of a duct whose first and last layers in y and z are solid
    walls; the no-slip planes lie half-way between the walls and the first fluid nodes."""
    a, b = (ny - 2) / 2.0, (nz - 2) / 2.0
    y = np.arange(ny) - (ny - 1) / 2.0
    z = np.arange(nz) - (nz - 1) / 2.0
    Z, Y = np.meshgrid(z, y, indexing="ij")
    return a, b, Y, Z


def duct_series(ny, nz, g, nu, terms=101):
    """Steady u(z, y) of a duct driven by the body force g along x (Poisson problem
    nu lap u = -g, u = 0 on the walls), as the single cosine/cosh series."""
    a, b, Y, Z = _duct_axes(ny, nz)
    return _series(a, b, Y, Z, g, nu, terms)


def _series(a, b, Y, Z, g, nu, terms):
    u = np.zeros_like(np.asarray(Y, dtype=np.float64))
    az = np.abs(Z)
    for n in range(1, terms + 1, 2):
        k = n * np.pi / (2 * a)
        # cosh(k z) / cosh(k b) without overflow
        ratio = np.exp(k * (az - b)) * (1 + np.exp(-2 * k * az)) / (1 + np.exp(-2 * k * b))
        u = u + (-1) ** ((n - 1) // 2) / n ** 3 * (1 - ratio) * np.cos(k * Y)
    return 16 * a * a * g / (nu * np.pi ** 3) * u


def duct_transient(ny, nz, g, nu, t, terms=61):
    """u(z, y, t) after the start-up from rest under the body force g: the double series
    sum g_mn / (nu l_mn) (1 - exp(-nu l_mn t)) cos(m pi y / 2a) cos(n pi z / 2b) over odd m, n, with
    g_mn = 16 g (-1)^((m + n) / 2 - 1) / (m n pi^2) and l_mn = (m pi / 2a)^2 + (n pi / 2b)^2."""
    a, b, Y, Z = _duct_axes(ny, nz)
    u = np.zeros_like(Y)
    for m in range(1, terms + 1, 2):
        km = m * np.pi / (2 * a)
        cy = np.cos(km * Y)
        for n in range(1, terms + 1, 2):
            kn = n * np.pi / (2 * b)
            lam = km * km + kn * kn
            gmn = 16.0 * g * (-1) ** ((m + n) // 2 - 1) / (m * n * np.pi ** 2)
            u += gmn / (nu * lam) * (1.0 - np.exp(-nu * lam * t)) * cy * np.cos(kn * Z)
    return u


def duct_peak_per_force(ny, nz, nu):
    """Steady centre-line velocity (at the duct axis) per unit body force."""
    return float(_series((ny - 2) / 2.0, (nz - 2) / 2.0, 0.0, 0.0, 1.0, nu, 101))


def duct_batch(count, seed=20261203, sides=(16, 96), re_range=(10.0, 500.0), u_max=0.03):
    """Rectangular ducts for the batched sweep: each side log-uniform in `sides`, periodic in x with
    walls in y and z, Re = u_max H / nu uniform with H the smaller cross-section side, the body force
    set so the steady centre-line velocity is u_max. Re is drawn from [max(Re_lo, 42 u_max H), Re_hi]
    so that nu stays within K17's stable range (nu <= 1/42)."""
    rng = np.random.default_rng(seed)
    lo, hi = math.log(sides[0]), math.log(sides[1])
    out = []
    for _ in range(count):
        nx, ny, nz = (int(round(math.exp(v))) for v in rng.uniform(lo, hi, 3))
        H = min(ny, nz) - 2
        re_lo = max(re_range[0], u_max * H / K17_NU_MAX)
        re = float(rng.uniform(re_lo, max(re_lo, re_range[1])))
        nu = u_max * H / re
        g = u_max / duct_peak_per_force(ny, nz, nu)
        out.append({"shape": (nx, ny, nz), "nu": nu, "omega": 1.0 / (3.0 * nu + 0.5), "g": g, "re": re,
                    "fluid_nodes": nx * (ny - 2) * (nz - 2)})
    return out


def porous_block(side, seed, porosity=None, radius=(3.0, 8.0), max_tries=40000, x_margin=0):
    """A side^3 block of random non-overlapping spheres added one at a time (random sequential
    addition) until the solid fraction reaches 1 - porosity (porosity uniform in [0.5, 0.9] when
    not given). Returns the node mask (x fastest, nonzero = fluid), the spheres (cx, cy, cz, r) and
    the porosity reached. Sphere centres keep a margin of r from the block faces. Random sequential
    addition of non-overlapping spheres jams near a solid fraction of about 0.3-0.35, so low target
    porosities end at the jammed packing (the porosity reached is returned); the addition stops
    after 8 batches of 256 candidates without a single accepted sphere, or after max_tries candidates.
    x_margin keeps the spheres that many nodes further from the x faces (room for pressure planes)."""
    rng = np.random.default_rng(seed)
    if porosity is None:
        porosity = float(rng.uniform(0.5, 0.9))
    solid = np.zeros((side, side, side), dtype=bool)
    target = (1.0 - porosity) * side ** 3
    cell = 2.0 * radius[1]                      # spheres that can touch have centres in adjacent cells
    nc = int(np.ceil(side / cell)) + 1
    cells = {}
    centres, radii = [], []
    n_solid = 0
    tries = 0
    batch = 256
    idle = 0
    while n_solid < target and tries < max_tries and idle < 8:
        r = rng.uniform(radius[0], radius[1], batch)
        lo_c = np.stack([r + x_margin, r, r], axis=1)
        hi_c = np.stack([side - 1 - r - x_margin, side - 1 - r, side - 1 - r], axis=1)
        c = rng.uniform(0.0, 1.0, (batch, 3)) * (hi_c - lo_c) + lo_c
        tries += batch
        accepted = 0
        for ci, ri in zip(c, r):
            if n_solid >= target:
                break
            key = tuple(int(v // cell) for v in ci)
            near = []
            for dz in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        near.extend(cells.get((key[0] + dx, key[1] + dy, key[2] + dz), ()))
            if near:
                cc = np.asarray([centres[j] for j in near])
                rr = np.asarray([radii[j] for j in near])
                if (((cc - ci) ** 2).sum(axis=1) < (rr + ri) ** 2).any():
                    continue
            lo = np.maximum(np.floor(ci - ri).astype(int), 0)
            hi = np.minimum(np.ceil(ci + ri).astype(int) + 1, side)
            zz, yy, xx = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]), np.arange(lo[0], hi[0]),
                                     indexing="ij")
            inside = (xx - ci[0]) ** 2 + (yy - ci[1]) ** 2 + (zz - ci[2]) ** 2 <= ri * ri
            region = solid[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
            n_solid += int((inside & ~region).sum())
            region |= inside
            cells.setdefault(key, []).append(len(centres))
            centres.append(ci)
            radii.append(ri)
            accepted += 1
        idle = idle + 1 if accepted == 0 else 0
    mask = (~solid).astype(np.uint8).reshape(-1)
    spheres = [(float(c[0]), float(c[1]), float(c[2]), float(r)) for c, r in zip(centres, radii)]
    return mask, spheres, float(mask.mean())


def cube_duct(nx=512, ny=256, nz=256, cube=32, x0=128, u_max=0.05, re=3000.0):
    """Duct flow past a wall-mounted cube. Fluid box nx x ny x nz (stopper shell around
    it); no-slip walls on the y and z faces (interpolated bounce-back, q = 1/2); the inlet at x = 0
    carries u_x = u_max 16 eta (1 - eta) zeta (1 - zeta) (eta, zeta the cross-section coordinates
    between the wall planes); the outlet at x = nx - 1 holds drho = 0 (non-equilibrium pressure BC,
    direction P00); the cube of side `cube` sits on the z = 0 wall, x in [x0, x0 + cube), centred
    in y, with its faces half-way between nodes (exact-geometry q = 1/2) and is the geometry BC of
    the drag. Re = u_max cube / nu. Returns (grid, omega, meta)."""
    from .grid import ListGrid
    g = ListGrid(nx, ny, nz, periodic=(False, False, False))
    for side in ("MY", "PY", "MZ", "PZ"):
        g.add_side(side, "noslip")

    def inlet(x, y, z):
        eta = (y + 0.5) / ny
        zeta = (z + 0.5) / nz
        return (u_max * 16.0 * eta * (1 - eta) * zeta * (1 - zeta), np.zeros_like(eta), np.zeros_like(eta))

    g.add_side("MX", "velocity", velocity=inlet)
    g.add_side("PX", "pressure", rho=0.0)
    y0 = (ny - cube) / 2.0
    g.add_box_obstacle((x0 - 0.5, y0 - 0.5, -0.5), (x0 + cube - 0.5, y0 + cube - 0.5, cube - 0.5))
    nu = u_max * cube / re
    return g, 1.0 / (3.0 * nu + 0.5), {"nu": nu, "u_max": u_max, "cube": cube, "area": float(cube * cube)}


# D3Q27 directions in reference numbering (src/lbm/constants/D3Q27.h:42-72)
_CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
_CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1])
_CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1])


def sphere_link_q(points, centre, radius):
    """q of the 26 links of each point (n, 3) against one sphere: the ray parameter t of
    p + t c_d at which the link enters the sphere, as Sphere::getIntersection computes it
    (geometries/Sphere/Sphere.cpp:124-169: the smaller non-negative root of |p + t c - centre|^2 =
    r^2), kept where 0 <= t <= 1 (GridImp::calculateQs, GridImp.cpp:1561-1600); -1 elsewhere.
    Returns (27, n)."""
    rp = np.asarray(points, dtype=np.float64) - np.asarray(centre, dtype=np.float64)
    q = np.full((27, rp.shape[0]), -1.0)
    rr = (rp * rp).sum(axis=1) - float(radius) * float(radius)
    big = np.float64(np.finfo(np.float32).max)
    for d in range(1, 27):
        c = np.array([_CX[d], _CY[d], _CZ[d]], dtype=np.float64)
        dsq = float(c @ c)
        pc = 2.0 * (rp @ c) / dsq
        qc = rr / dsq
        disc = 0.25 * pc * pc - qc
        ok = disc >= 0.0
        sq = np.sqrt(np.where(ok, disc, 0.0))
        r1 = -0.5 * pc + sq
        r2 = -0.5 * pc - sq
        both_negative = (r1 < 0.0) & (r2 < 0.0)
        r1 = np.where(r1 < 0.0, big, r1)
        r2 = np.where(r2 < 0.0, big, r2)
        t = np.minimum(r1, r2)
        hit = ok & ~both_negative & (t <= 1.0) & (t >= 0.0)
        q[d] = np.where(hit, t, -1.0)
    return q


def porous_block_bcs(side, seed, porosity=None, drho=3e-3, radius=(3.0, 8.0)):
    """The porous-block serving workload as boundary-condition lists of a structured box: a side^3 porous block (spheres
    as :func:`porous_block`, kept three nodes off the x faces) between two pressure planes.

    The box is (side + 2) x side x side, periodic in y and z; its first and last x layers are solid
    stoppers. The fluid layers x = 1 and x = side carry PressureNonEquilibriumCompressible at
    drho = +drho/2 (outward normal M00, neighbour x = 2) and -drho/2 (P00, neighbour x = side - 1),
    as a pressure side of the reference's grid builder sets them (Side.cpp:89-110). Every fluid node
    with a link cut by a sphere is a NoSlipInterpolatedCompressible node with the exact q of each cut
    link (the smallest over the spheres, GridImp.cpp:1561-1600), periodic images included.

    Returns dict(shape, mask, bcs, spheres, porosity, length, drho): mask is the box's node mask
    (nonzero = fluid, the stopper layers solid), bcs the lists for Pool.add / Box, length the
    distance between the pressure planes (side - 1)."""
    from . import _native as N
    inner, spheres, phi = porous_block(side, seed, porosity=porosity, radius=radius, x_margin=3)
    nx, ny, nz = side + 2, side, side
    solid = np.ones((nz, ny, nx), dtype=bool)
    solid[:, :, 1:side + 1] = inner.reshape(side, side, side) == 0
    solid[:, :, 0] = True
    solid[:, :, -1] = True
    mask = (~solid).astype(np.uint8).reshape(-1)
    keys_all, q_all = [], []
    for (cx, cy, cz, r) in spheres:
        for oy in (-side, 0, side):
            for oz in (-side, 0, side):
                c = np.array([cx + 1.0, cy + oy, cz + oz])
                lo = np.floor(c - r - 2).astype(int)
                hi = np.ceil(c + r + 2).astype(int)
                if hi[1] < 0 or lo[1] >= ny or hi[2] < 0 or lo[2] >= nz:
                    continue
                xs = np.arange(max(lo[0], 1), min(hi[0], nx - 2) + 1)
                ys = np.arange(max(lo[1], 0), min(hi[1], ny - 1) + 1)
                zs = np.arange(max(lo[2], 0), min(hi[2], nz - 1) + 1)
                Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
                X, Y, Z = X.reshape(-1), Y.reshape(-1), Z.reshape(-1)
                d2 = (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2
                near = ~solid[Z, Y, X] & (d2 <= (r + 1.8) ** 2)
                if not near.any():
                    continue
                pts = np.stack([X[near], Y[near], Z[near]], axis=1).astype(np.float64)
                q = sphere_link_q(pts, c, r)
                cut = (q >= 0.0).any(axis=0)
                keys_all.append((X[near] + nx * (Y[near] + ny * Z[near]))[cut])
                q_all.append(q[:, cut])
    # per node and direction the smallest q over the spheres (uncut links stay -1)
    if keys_all:
        keys = np.concatenate(keys_all)
        qs = np.concatenate(q_all, axis=1)
        order = np.argsort(keys, kind="stable")
        keys, qs = keys[order], np.where(qs[:, order] < 0.0, np.inf, qs[:, order])
        k_ns, start = np.unique(keys, return_index=True)
        q_ns = np.minimum.reduceat(qs, start, axis=1)
        q_ns = np.where(np.isinf(q_ns), -1.0, q_ns)
        k_ns = k_ns.astype(np.int32)
    else:
        k_ns, q_ns = np.zeros(0, dtype=np.int32), np.zeros((27, 0))
    yy, zz = np.meshgrid(np.arange(ny), np.arange(nz), indexing="xy")
    yy, zz = yy.reshape(-1), zz.reshape(-1)
    k_in = 1 + nx * (yy + ny * zz)
    k_out = side + nx * (yy + ny * zz)
    pressure = (np.concatenate([k_in, k_out]).astype(np.int32),
                np.concatenate([k_in + 1, k_out - 1]).astype(np.int32),
                np.concatenate([np.full(k_in.size, 0.5 * drho), np.full(k_out.size, -0.5 * drho)]),
                np.concatenate([np.full(k_in.size, N.DIR_M00), np.full(k_out.size, N.DIR_P00)]).astype(np.int32))
    return {"shape": (nx, ny, nz), "mask": mask, "bcs": {"noslip": (k_ns, q_ns), "pressure": pressure},
            "spheres": spheres, "porosity": phi, "length": float(side - 1), "drho": float(drho)}
