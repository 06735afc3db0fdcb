"""ORACLE — test infrastructure, not product code.

ctypes binding of the plain-C oracle (liboracle.so, built by oracle/Makefile), of the
reference-header pins (_ref/libvfref64.so, _ref/libvfref32.so) and of the reference's own CUDA
kernels (_ref/libvfref_gpu64.so, run on the GPU). Only the tests, the smoke check
and the benchmark's CPU-baseline / reference legs use this module, and only as a checker or as
the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF64 = HERE / "_ref" / "libvfref64.so"
REF32 = HERE / "_ref" / "libvfref32.so"
REF64_RELEASE = HERE / "_ref" / "libvfref64_release.so"
REFGPU = HERE / "_ref" / "libvfref_gpu64.so"
REFGPU32 = HERE / "_ref" / "libvfref_gpu32.so"

_P = C.c_void_p
_lib = None


def build(reference: str | None = None) -> None:
    """Build liboracle.so, and the reference pins when the reference tree is present."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    ref = reference or os.environ.get("VFB_REFERENCE_DIR", "/root/reference")
    if Path(ref).is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={ref}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        d, i, u = C.c_double, C.c_int, C.c_uint32
        L.orc_k17_f64.argtypes = [_P, d, _P, d, d, d, _P]
        L.orc_k17_f32.argtypes = [_P, C.c_float, _P, C.c_float, C.c_float, C.c_float, _P]
        L.orc_k17_rates_f64.argtypes = [d, _P]
        L.orc_density_f64.argtypes = [_P]
        L.orc_density_f64.restype = d
        L.orc_macro_compressible_f64.argtypes = [_P, _P, _P, _P, _P, _P]
        L.orc_chimera_f64.argtypes = [i, _P, d, d, d, d]
        L.orc_collision.argtypes = [_P, _P, u, i, d, _P, _P, i, _P, _P, _P, _P, i]
        L.orc_collision_template.argtypes = [_P, _P, u, i, d, _P, _P, i, i, i] + [_P] * 7
        L.orc_bc_noslip_bounce_back.argtypes = [_P, _P, _P, u, i]
        L.orc_bc_noslip_interpolated.argtypes = [_P, _P, _P, u, i, d]
        L.orc_bc_velocity_bounce_back.argtypes = [_P, _P, _P, u, i, _P, _P, _P]
        L.orc_bc_velocity_interpolated.argtypes = [_P, _P, _P, u, i, d, _P, _P, _P]
        L.orc_bc_pressure_neq.argtypes = [_P, _P, _P, _P, u, i, i]
        L.orc_init.argtypes = [_P, _P, _P, _P, _P, _P, i]
        L.orc_init_neq.argtypes = [_P, _P, _P, _P, _P, _P, _P, d, i]
        L.orc_read_pre.argtypes = [_P, u, i, _P]
        L.orc_bc_slip.argtypes = [_P, _P, _P, u, i, d]
        L.orc_macros.argtypes = [_P, _P, i, _P, _P, _P, _P, _P]
        L.orc_mass_energy.argtypes = [_P, _P, u, i, _P]
        L.orc_interp_node_moments.argtypes = [_P, d, _P]
        L.orc_interp_coefficients.argtypes = [_P, d, d, d, _P]
        L.orc_interp_point.argtypes = [_P, d, d, d, d, d, i, _P]
        L.orc_scale_cf.argtypes = [_P, _P, _P, _P, u, _P, _P, _P, i, d, d]
        L.orc_scale_fc.argtypes = [_P, _P, _P, _P, u, _P, _P, _P, i, d, d]
        _lib = L
    return _lib


def ref64():
    if not REF64.exists():
        return None
    L = C.CDLL(str(REF64))
    d = C.c_double
    L.ref_k17_f64.argtypes = [_P, d, _P, d, d, d, _P]
    L.ref_chimera_f64.argtypes = [C.c_int, _P, d, d, d, d]
    L.ref_density_f64.argtypes = [_P]
    L.ref_density_f64.restype = d
    L.ref_macro_compressible_f64.argtypes = [_P, _P]
    L.ref_incompressible_velocity_f64.argtypes = [_P, _P]
    L.ref_collision_sweep_f64.argtypes = [_P, C.c_uint64, _P, _P, _P, _P, C.c_uint32, C.c_int, d, _P, C.c_int]
    L.ref_interp_coefficients_f64.argtypes = [_P, d, d, d, d, _P]
    L.ref_interp_cf_f64.argtypes = [_P, d, d, d, d, d, d, d, d, _P]
    L.ref_interp_fc_f64.argtypes = [_P, d, d, d, d, d, _P]
    return L


def ref32():
    if not REF32.exists():
        return None
    L = C.CDLL(str(REF32))
    f = C.c_float
    L.ref_k17_f32.argtypes = [_P, f, _P, f, f, f, _P]
    return L


def ref64_release():
    """The FP64 reference-header shim built with the reference's Release flags (-O3
    -funroll-all-loops), the timed CPU baseline; None if it has not been built."""
    if not REF64_RELEASE.exists():
        return None
    L = C.CDLL(str(REF64_RELEASE))
    d = C.c_double
    L.ref_k17_f64.argtypes = [_P, d, _P, d, d, d, _P]
    L.ref_collision_sweep_f64.argtypes = [_P, C.c_uint64, _P, _P, _P, _P, C.c_uint32, C.c_int, d, _P, C.c_int]
    return L


def refgpu(real_bytes: int = 8, release: bool = False):
    """The reference's own CUDA kernels built from the reference tree, or None: FP64
    (real_bytes = 8) or FP32 (real_bytes = 4, real = float); without FMA contraction (the parity
    pins) or, with release=True, with the reference's own build flags (FMA contraction on)."""
    path = REFGPU if real_bytes == 8 else REFGPU32
    if release:
        path = HERE / "_ref" / f"libvfref_gpu{8 * real_bytes}_release.so"
    if not path.exists():
        return None
    L = C.CDLL(str(path))
    u, i, u64 = C.c_uint32, C.c_int, C.c_uint64
    d = C.c_double if real_bytes == 8 else C.c_float
    L.refgpu_k17.argtypes = [_P, u64, _P, _P, _P, _P, u, i, d, _P, _P, d]
    L.refgpu_k17_template.argtypes = [_P, u64, _P, _P, _P, _P, u, i, d, _P, _P, d] + [_P] * 7 + [i]
    L.refgpu_noslip_bounce_back.argtypes = [_P, _P, _P, u, _P, _P, _P, u64, i]
    L.refgpu_noslip_interpolated.argtypes = [_P, _P, _P, u, d, _P, _P, _P, u64, i]
    L.refgpu_velocity_bounce_back.argtypes = [_P, _P, _P, _P, _P, _P, u, _P, _P, _P, u64, i]
    L.refgpu_velocity_interpolated.argtypes = [_P, _P, _P, _P, _P, _P, u, d, _P, _P, _P, u64, i]
    L.refgpu_pressure_neq.argtypes = [_P, _P, _P, _P, i, _P, _P, _P, u64, i, i]
    L.refgpu_init.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P, u, _P, i]
    L.refgpu_noslip_interpolated_incompressible.argtypes = [_P, _P, _P, u, d, _P, _P, _P, u64, i]
    L.refgpu_velocity_interpolated_incompressible.argtypes = [_P, _P, _P, _P, _P, _P, u, d, _P, _P, _P, u64, i]
    L.refgpu_velocity_with_pressure.argtypes = [_P, _P, _P, _P, _P, _P, u, d, _P, _P, _P, u64, i]
    L.refgpu_pressure_neq_incompressible.argtypes = [_P, _P, _P, _P, i, _P, _P, _P, u64, i, i]
    L.refgpu_outflow.argtypes = [_P, _P, _P, _P, i, d, _P, _P, _P, u64, i, i, i, d]
    L.refgpu_macros.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P, _P, u64, _P, i]
    L.refgpu_scale_cf.argtypes = [_P] * 8 + [u64, u64, i, _P, _P, u, d, d, _P, _P, _P]
    L.refgpu_scale_fc.argtypes = [_P] * 8 + [u64, u64, i, _P, _P, u, d, d, _P, _P, _P]
    L.refgpu_drag_lift_post.argtypes = [_P, _P, _P, i, _P, _P, _P, _P, _P, _P, u64, i]
    L.refgpu_drag_lift_pre.argtypes = [_P, _P, _P, i, _P, _P, _P, _P, _P, _P, u64, i]
    return L


def ptr(a: np.ndarray):
    """A void pointer to the array's data that keeps the array alive while the pointer lives (so
    a temporary array passed straight into a call is not freed before the call reads it)."""
    return a.ctypes.data_as(C.c_void_p) if a is not None else C.c_void_p(0)


class _Level(C.Structure):
    _fields_ = [("n", C.c_uint64), ("f", _P), ("nbx", _P), ("nby", _P), ("nbz", _P)]


class _NoSlip(C.Structure):
    _fields_ = [("k", _P), ("q", _P), ("n", C.c_uint32), ("kind", C.c_int)]


class _Velocity(C.Structure):
    _fields_ = [("k", _P), ("q", _P), ("n", C.c_uint32), ("ux", _P), ("uy", _P), ("uz", _P), ("kind", C.c_int)]


class _Pressure(C.Structure):
    _fields_ = [("k", _P), ("kN", _P), ("rho", _P), ("n", C.c_uint32), ("direction", C.c_int)]


class OracleLevel:
    """A level in the reference layout, advanced on the host by the oracle."""

    def __init__(self, grid, omega, lim=(0.01, 0.01, 0.01), forces=(0.0, 0.0, 0.0), velocity_kind=1, noslip_kind=1,
                 geometry_kind=0, drag_lift=False, level=0):
        self.grid = grid
        self.level = int(level)
        self.n = grid.number_of_nodes
        self.f = np.zeros(27 * self.n, dtype=np.float64)
        self.nb = [np.ascontiguousarray(grid.neighbor[a].astype(np.uint32)) for a in range(3)]
        self.geo = np.ascontiguousarray(grid.geo.astype(np.uint32))
        self.fluid = np.ascontiguousarray(grid.fluid.astype(np.uint32))
        self.omega = float(omega)
        self.lim = np.array(lim, dtype=np.float64)
        self.forces = np.array(forces, dtype=np.float64)
        self.is_even = C.c_int(1)
        self.L = _Level(self.n, self.f.ctypes.data, self.nb[0].ctypes.data, self.nb[1].ctypes.data, self.nb[2].ctypes.data)
        self._keep = []
        self.vel = None
        self.ns = None
        m = grid.merged("velocity")
        if m is not None:
            k, q, v = m
            arrs = [np.ascontiguousarray(k.astype(np.int32)), np.ascontiguousarray(q.reshape(-1))] + \
                   [np.ascontiguousarray(v[a].astype(np.float64)) for a in range(3)]
            self._keep += arrs
            self.vel = _Velocity(arrs[0].ctypes.data, arrs[1].ctypes.data, k.size, arrs[2].ctypes.data,
                                 arrs[3].ctypes.data, arrs[4].ctypes.data, velocity_kind)
        m = grid.merged("noslip")
        if m is not None:
            k, q, _ = m
            arrs = [np.ascontiguousarray(k.astype(np.int32)), np.ascontiguousarray(q.reshape(-1))]
            self._keep += arrs
            self.ns = _NoSlip(arrs[0].ctypes.data, arrs[1].ctypes.data, k.size, noslip_kind)
        self.geo_bc = None
        m = grid.merged("geometry")
        if m is not None:
            k, q, _ = m
            arrs = [np.ascontiguousarray(k.astype(np.int32)), np.ascontiguousarray(q.reshape(-1))]
            self._keep += arrs
            self.geo_bc = _NoSlip(arrs[0].ctypes.data, arrs[1].ctypes.data, k.size, geometry_kind)
        self.drag_lift = drag_lift and self.geo_bc is not None
        self.drag_history = []
        from virtualfluids_b200.grid import SIDE_DIR
        pr = []
        for b in grid.bcs:
            if b.kind != "pressure":
                continue
            arrs = [np.ascontiguousarray(b.k.astype(np.int32)), np.ascontiguousarray(b.k_neighbor.astype(np.int32)),
                    np.ascontiguousarray(np.broadcast_to(np.asarray(b.rho, dtype=np.float64), (b.k.size,)))]
            self._keep += arrs
            pr.append(_Pressure(arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data, b.k.size, SIDE_DIR[b.side]))
        self.pr = (_Pressure * max(len(pr), 1))(*pr) if pr else None
        self.n_pr = len(pr)

    def init(self, rho=None, ux=None, uy=None, uz=None, neq=False):
        """PreProcessorImp::init: the odd, then the even parity; neq: the non-equilibrium init
        (Parameter::setUseInitNeq), which reads the grid's neighborInverse."""
        z = np.zeros(self.n)
        arrs = [np.ascontiguousarray(a if a is not None else z, dtype=np.float64) for a in (rho, ux, uy, uz)]
        if neq:
            inv = np.ascontiguousarray(self.grid.neighbor_inverse, dtype=np.uint32)
            for ev in (0, 1):
                lib().orc_init_neq(C.byref(self.L), ptr(self.geo), ptr(inv), *(ptr(a) for a in arrs), self.omega, ev)
        else:
            lib().orc_init(C.byref(self.L), ptr(self.geo), *(ptr(a) for a in arrs), 0)
            lib().orc_init(C.byref(self.L), ptr(self.geo), *(ptr(a) for a in arrs), 1)
        self.is_even.value = 1

    def run(self, steps, threads=0):
        lib().orc_run_level.argtypes = [_P, C.c_int, _P, C.c_uint32, C.POINTER(C.c_int), C.c_double, _P, _P, _P, _P,
                                        _P, _P, _P, C.c_int, C.c_int, C.c_int]
        hist = np.zeros((int(steps), 3)) if self.drag_lift else None
        rc = lib().orc_run_level(C.byref(self.L), self.level, ptr(self.fluid), self.fluid.size, C.byref(self.is_even),
                                 self.omega, ptr(self.lim), ptr(self.forces), C.byref(self.vel) if self.vel else None,
                                 C.byref(self.ns) if self.ns else None, C.byref(self.geo_bc) if self.geo_bc else None,
                                 ptr(hist) if hist is not None else None, self.pr, self.n_pr, int(steps), int(threads))
        if rc != 0:
            raise MemoryError("oracle step driver could not allocate its drag workspace")
        if hist is not None:
            self.drag_history.extend(hist)

    def run_reference_collision(self, ref, steps, threads=0):
        """The same time steps with the collision sweep of the reference's own K17 header (`ref`,
        ref64() or ref64_release(): ref_collision_sweep_f64 over the esoteric-twist layout) and the
        boundary conditions of the oracle, in UpdateGrid27 order (collision, velocity BC, no-slip
        BC, parity toggle). Levels with forcing, a geometry BC or pressure BCs are not supported."""
        if self.geo_bc is not None or self.n_pr or np.any(self.forces != 0.0) or self.level != 0:
            raise ValueError("run_reference_collision covers unforced single levels with velocity and no-slip BCs")
        L = lib()
        lim = np.ascontiguousarray(self.lim)
        for _ in range(int(steps)):
            ev = self.is_even.value
            ref.ref_collision_sweep_f64(ptr(self.f), self.n, *(ptr(a) for a in self.nb), ptr(self.fluid),
                                        self.fluid.size, ev, self.omega, ptr(lim), int(threads))
            v = self.vel
            if v is not None and v.n:
                if v.kind == 1:
                    L.orc_bc_velocity_bounce_back(C.byref(self.L), v.k, v.q, v.n, ev, v.ux, v.uy, v.uz)
                elif v.kind == 2:
                    L.orc_bc_velocity_interpolated(C.byref(self.L), v.k, v.q, v.n, ev, self.omega, v.ux, v.uy, v.uz)
                else:
                    raise ValueError("velocity BC kind not covered")
            b = self.ns
            if b is not None and b.n:
                if b.kind == 1:
                    L.orc_bc_noslip_bounce_back(C.byref(self.L), b.k, b.q, b.n, ev)
                elif b.kind == 2:
                    L.orc_bc_noslip_interpolated(C.byref(self.L), b.k, b.q, b.n, ev, self.omega)
                else:
                    raise ValueError("no-slip BC kind not covered")
            self.is_even.value = 1 - ev

    def pre(self, k):
        """The 27 pre-collision populations f - w of node k at the current parity (getPreCollisionDistribution)."""
        out = np.zeros(27)
        lib().orc_read_pre(C.byref(self.L), int(k), self.is_even.value, ptr(out))
        return out

    def macroscopic(self):
        out = [np.zeros(self.n) for _ in range(5)]
        lib().orc_macros(C.byref(self.L), ptr(self.geo), self.is_even.value, *(ptr(a) for a in out))
        return dict(zip(("rho", "vx", "vy", "vz", "pressure"), out))

    def mass_energy(self):
        out = np.zeros(2)
        lib().orc_mass_energy(C.byref(self.L), ptr(self.fluid), self.fluid.size, self.is_even.value, ptr(out))
        return float(out[0]), float(out[1])


class OracleMultiLevel:
    """Nested refinement levels advanced on the host: UpdateGrid27::updateGrid's recursion
    (UpdateGrid27.cpp:54-95; a level with a finer one lets it take two steps first) followed by
    Refinement_noExchange (RefinementStrategy.cpp:169-178: fine to coarse, then coarse to fine).
    omega of level l is 1 / (3 nu 2^l + 1/2) (Parameter.cpp:404-406); forces scale by 2^-l."""

    def __init__(self, mgrid, nu, lim=(0.01, 0.01, 0.01), forces=(0.0, 0.0, 0.0), velocity_kind=1, noslip_kind=1):
        self.levels = [OracleLevel(g, 1.0 / (3.0 * (nu * 2.0 ** l) + 0.5), lim, forces, velocity_kind, noslip_kind,
                                   level=l) for l, g in enumerate(mgrid.levels)]
        self.cells = []
        for it in mgrid.interfaces:
            arrs = [np.ascontiguousarray(a.astype(np.uint32)) for a in (it.coarse_fc, it.fine_fc, it.coarse_cf, it.fine_cf)]
            offs = [np.ascontiguousarray(o[a], dtype=np.float64) for o in (it.offsets_fc, it.offsets_cf) for a in range(3)]
            self.cells.append((arrs, offs))

    def init(self, level, rho=None, ux=None, uy=None, uz=None):
        self.levels[level].init(rho, ux, uy, uz)

    def run(self, steps):
        for _ in range(int(steps)):
            self._update(0)

    def _update(self, l):
        finer = l + 1 < len(self.levels)
        if finer:
            self._update(l + 1)
            self._update(l + 1)
        self.levels[l].run(1)
        if finer:
            c, f = self.levels[l], self.levels[l + 1]
            (cfc, ffc, ccf, fcf), offs = self.cells[l]
            lib().orc_scale_fc(C.byref(c.L), C.byref(f.L), ptr(cfc), ptr(ffc), cfc.size, *(ptr(o) for o in offs[:3]),
                               c.is_even.value, c.omega, f.omega)
            lib().orc_scale_cf(C.byref(c.L), C.byref(f.L), ptr(ccf), ptr(fcf), ccf.size, *(ptr(o) for o in offs[3:]),
                               c.is_even.value, c.omega, f.omega)


def k17(f, omega, lim=(0.01, 0.01, 0.01), force=(0.0, 0.0, 0.0), dtype=np.float64):
    """One-node K17 of the oracle: returns (post-collision f, macro[4])."""
    if dtype == np.float64:
        a = np.ascontiguousarray(f, dtype=np.float64).copy()
        m = np.zeros(4)
        lib().orc_k17_f64(ptr(a), omega, ptr(np.array(lim, dtype=np.float64)), *force, ptr(m))
    else:
        a = np.ascontiguousarray(f, dtype=np.float32).copy()
        m = np.zeros(4, dtype=np.float32)
        lib().orc_k17_f32(ptr(a), np.float32(omega), ptr(np.array(lim, dtype=np.float32)), *(np.float32(x) for x in force),
                          ptr(m))
    return a, m


# corners of an interpolation cell in the oracle's order c = ix + 2 iy + 4 iz, and their position in
# the reference's visiting order MMM, MMP, PMP, PMM, MPM, MPP, PPP, PPM
REF_CORNER_ORDER = [0, 4, 5, 1, 2, 6, 7, 3]


def interp_coefficients(f8, omega, offset=(0.0, 0.0, 0.0)):
    """Oracle coefficients of one cell (42, the member order of InterpolationCoefficients)."""
    L = lib()
    mom = np.zeros((8, 9))
    for c in range(8):
        L.orc_interp_node_moments(ptr(np.ascontiguousarray(f8[c], dtype=np.float64)), omega, ptr(mom[c]))
    coef = np.zeros(42)
    L.orc_interp_coefficients(ptr(mom), *(float(x) for x in offset), ptr(coef))
    return coef


def interp_cf_cell(f8, omega_coarse, omega_fine, offset=(0.0, 0.0, 0.0)):
    """Oracle coarse-to-fine for one cell: f8[c] (oracle corner order) -> 8 fine nodes' populations."""
    L = lib()
    coef = interp_coefficients(f8, omega_coarse, offset)
    out = np.zeros((8, 27))
    for c in range(8):
        pos = [0.25 if (c >> a) & 1 else -0.25 for a in range(3)]
        L.orc_interp_point(ptr(coef), omega_fine, 0.5, *pos, 0, ptr(out[c]))
    return out


def interp_fc_cell(f8, omega_fine, omega_coarse, offset=(0.0, 0.0, 0.0)):
    """Oracle fine-to-coarse for one cell: f8[c] (oracle corner order) -> the coarse node's populations."""
    L = lib()
    coef = interp_coefficients(f8, omega_fine, offset)
    out = np.zeros(27)
    L.orc_interp_point(ptr(coef), omega_coarse, 2.0, 0.0, 0.0, 0.0, 1, ptr(out))
    return out


# ---------------------------------------------------------------------------------------------
# the reference's own grid generator (_ref/libvfref_gridgen.so)
# ---------------------------------------------------------------------------------------------
REFGG = HERE / "_ref" / "libvfref_gridgen.so"
SIDE_INDEX = {"MX": 0, "PX": 1, "MY": 2, "PY": 3, "MZ": 4, "PZ": 5, "GEOMETRY": 6}


def refgg():
    """The reference's GridGenerator behind ref_gridgen_shim.cpp, or None where it is not built."""
    if not REFGG.exists():
        return None
    L = C.CDLL(str(REFGG))
    d, i, u = C.c_double, C.c_int, C.c_uint32
    L.refgg_create.restype = _P
    L.refgg_create.argtypes = [d] * 7
    for name in ("refgg_build", "refgg_find_fluid_nodes", "refgg_destroy"):
        getattr(L, name).argtypes = [_P]
    L.refgg_add_refinement.argtypes = [_P] + [d] * 6 + [i]
    L.refgg_add_geometry.argtypes = [_P, i] + [d] * 6
    L.refgg_set_periodic.argtypes = [_P, i, i, i]
    L.refgg_set_noslip.argtypes = [_P, i]
    L.refgg_set_velocity.argtypes = [_P, i, d, d, d]
    L.refgg_set_pressure.argtypes = [_P, i, d]
    L.refgg_levels.argtypes = [_P]
    L.refgg_delta.argtypes = [_P, i]
    L.refgg_delta.restype = d
    for name in ("refgg_nodes", "refgg_fluid_count", "refgg_velocity_size", "refgg_geometry_size", "refgg_cf_count",
                 "refgg_fc_count"):
        getattr(L, name).argtypes = [_P, i]
        getattr(L, name).restype = u
    L.refgg_node_values.argtypes = [_P, i] + [_P] * 8
    L.refgg_fluid.argtypes = [_P, i, _P]
    L.refgg_velocity.argtypes = [_P, i] + [_P] * 5
    L.refgg_pressure_count.argtypes = [_P, i]
    L.refgg_pressure_size.argtypes = [_P, i, i]
    L.refgg_pressure_size.restype = u
    L.refgg_pressure.argtypes = [_P, i, i] + [_P] * 4
    L.refgg_geometry.argtypes = [_P, i] + [_P] * 5
    L.refgg_interface.argtypes = [_P, i] + [_P] * 10
    assert L.refgg_real_bytes() == 8
    return L


def reference_grid(box, delta, refinements=(), geometries=(), periodic=(False, False, False), noslip=(),
                   velocity=(), pressure=(), geometry_noslip=False):
    """Build a grid with the reference's MultipleGridBuilder and return the arrays its getters hand
    to the solver (the dicts virtualfluids_b200.gridgen.import_levels takes), as
    (levels, interfaces). box: (x0, y0, z0, x1, y1, z1); refinements: ((x0..z1), level_fine);
    geometries: ("sphere", cx, cy, cz, r) or ("cuboid", x0, y0, z0, x1, y1, z1); noslip: side names;
    velocity: (side, vx, vy, vz); pressure: (side, rho). The order of the calls is the reference
    apps' (DrivenCavity.cpp:95-146): grids, periodicity, build, then boundary conditions."""
    L = refgg()
    if L is None:
        raise FileNotFoundError("oracle/_ref/libvfref_gridgen.so is not built (make -C oracle ref)")
    h = L.refgg_create(*(float(x) for x in box), float(delta))
    try:
        for b, lev in refinements:
            L.refgg_add_refinement(h, *(float(x) for x in b), int(lev))
        for g in geometries:
            vals = [float(x) for x in g[1:]] + [0.0] * (7 - len(g))
            L.refgg_add_geometry(h, 0 if g[0] == "sphere" else 1, *vals[:6])
        L.refgg_set_periodic(h, *(int(bool(p)) for p in periodic))
        L.refgg_build(h)
        for s in noslip:
            L.refgg_set_noslip(h, SIDE_INDEX[s])
        for s, vx, vy, vz in velocity:
            L.refgg_set_velocity(h, SIDE_INDEX[s], vx, vy, vz)
        for s, rho in pressure:
            L.refgg_set_pressure(h, SIDE_INDEX[s], rho)
        if geometry_noslip:
            L.refgg_set_noslip(h, SIDE_INDEX["GEOMETRY"])
        L.refgg_find_fluid_nodes(h)
        levels, interfaces = [], []
        for lev in range(L.refgg_levels(h)):
            n = L.refgg_nodes(h, lev)
            xyz = [np.zeros(n) for _ in range(3)]
            nb = [np.zeros(n, dtype=np.uint32) for _ in range(5)]
            L.refgg_node_values(h, lev, *(ptr(a) for a in xyz), *(ptr(a) for a in nb))
            fl = np.zeros(L.refgg_fluid_count(h, lev), dtype=np.uint32)
            L.refgg_fluid(h, lev, ptr(fl))
            nv = L.refgg_velocity_size(h, lev)
            vel = {"k": np.zeros(nv, dtype=np.int32), "q27": np.zeros(27 * nv),
                   **{c: np.zeros(nv) for c in ("vx", "vy", "vz")}}
            if nv:
                L.refgg_velocity(h, lev, ptr(vel["vx"]), ptr(vel["vy"]), ptr(vel["vz"]), ptr(vel["k"]), ptr(vel["q27"]))
            press = []
            for j in range(L.refgg_pressure_count(h, lev)):
                m = L.refgg_pressure_size(h, lev, j)
                p = {"k": np.zeros(m, dtype=np.int32), "k_neighbor": np.zeros(m, dtype=np.int32), "rho": np.zeros(m),
                     "q27": np.zeros(27 * m)}
                if m:
                    p["direction"] = L.refgg_pressure(h, lev, j, ptr(p["rho"]), ptr(p["k"]), ptr(p["k_neighbor"]),
                                                      ptr(p["q27"]))
                    press.append(p)
            ng = L.refgg_geometry_size(h, lev)
            geom = {"k": np.zeros(ng, dtype=np.int32), "q27": np.zeros(27 * ng),
                    **{c: np.zeros(ng) for c in ("vx", "vy", "vz")}}
            if ng:
                L.refgg_geometry(h, lev, ptr(geom["k"]), ptr(geom["q27"]), ptr(geom["vx"]), ptr(geom["vy"]),
                                 ptr(geom["vz"]))
            levels.append({"number_of_nodes": n, "delta": L.refgg_delta(h, lev), "coords": xyz, "neighbor": nb[:3],
                           "neighbor_inverse": nb[3], "geo": nb[4], "fluid": fl, "velocity": vel, "pressure": press,
                           "geometry": geom})
        for lev in range(L.refgg_levels(h) - 1):
            ncf, nfc = L.refgg_cf_count(h, lev), L.refgg_fc_count(h, lev)
            idx = [np.zeros(m, dtype=np.uint32) for m in (ncf, ncf, nfc, nfc)]
            off = [np.zeros(m) for m in (ncf, ncf, ncf, nfc, nfc, nfc)]
            L.refgg_interface(h, lev, *(ptr(a) for a in idx), *(ptr(a) for a in off))
            interfaces.append({"cf_coarse": idx[0], "cf_fine": idx[1], "fc_coarse": idx[2], "fc_fine": idx[3],
                               "offsets_cf": np.stack(off[:3]), "offsets_fc": np.stack(off[3:])})
        return levels, interfaces
    finally:
        L.refgg_destroy(h)
