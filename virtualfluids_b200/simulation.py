"""Python mirror of the reference's set-up surface for the hot path, over the C ABI.

Names and meanings follow the reference so that a set-up reads like one of its apps
(apps/gpu/DrivenCavity/DrivenCavity.cpp:95-146):

* :class:`Parameter` — the subset of ``Parameter`` the time step reads (viscosity, main kernel,
  quadric limiters, forcing; src/gpu/core/Parameter/Parameter.h, Parameter.cpp:69-70, 395-422);
* :class:`BoundaryConditionFactory` — the enums and setters of
  src/gpu/core/BoundaryConditions/BoundaryConditionFactory.h:50-178;
* :class:`Simulation` — allocation, initialisation (PreProcessorImp::init) and the time loop
  (UpdateGrid27::updateGrid) of one level or of nested refinement levels, driving
  ``vfb_simulation_*`` of the native library.

Device memory is held in torch tensors (plumbing only); every kernel runs in ``libvfb.so``.
"""
from __future__ import annotations

import ctypes as C
import enum
import warnings

import numpy as np

from . import _native as N
from .grid import ListGrid, MultiLevelGrid

STORAGE = {"f64": N.STORAGE_F64, "f32": N.STORAGE_F32, "f16": N.STORAGE_F16, "bf16": N.STORAGE_BF16,
           "e3m12": N.STORAGE_E3M12}


def _torch():
    import torch
    return torch


def storage_dtype(storage: int):
    t = _torch()
    return {N.STORAGE_F64: t.float64, N.STORAGE_F32: t.float32, N.STORAGE_F16: t.float16, N.STORAGE_BF16: t.bfloat16,
            N.STORAGE_E3M12: t.int16}[storage]


def real_dtype(storage: int):
    t = _torch()
    return t.float64 if storage == N.STORAGE_F64 else t.float32


class Parameter:
    """Subset of the reference Parameter used by the collision, BC and init kernels."""

    def __init__(self):
        self.viscosity_lb = 0.0
        self.velocity_lb = 0.0
        self.main_kernel = None
        self.quadric_limiters = (0.01, 0.01, 0.01)  # Parameter.cpp:69 defaults
        self.forcing = (0.0, 0.0, 0.0)
        self.storage = N.STORAGE_F64
        self.arith = N.ARITH_FAST
        self.outflow_pressure_correction_factor = 0.0
        self.use_init_neq = False

    def set_viscosity_lb(self, nu: float):
        self.viscosity_lb = float(nu)

    def set_velocity_lb(self, u: float):
        self.velocity_lb = float(u)

    def configure_main_kernel(self, name: str):
        """Parameter::configureMainKernel (Parameter.cpp:1216); unknown names fail at once."""
        kid = C.c_int32()
        N.check(N.lib().vfb_kernel_lookup(name.encode(), C.byref(kid)))
        self.main_kernel = name

    def set_quadric_limiters(self, p: float, m: float, d: float):
        self.quadric_limiters = (float(p), float(m), float(d))

    def set_use_init_neq(self, use: bool):
        """Parameter::setUseInitNeq: Simulation.init adds the non-equilibrium part from the velocity
        gradients to the equilibrium (InitNavierStokesCompressibleNonEquilibrium_Device)."""
        self.use_init_neq = bool(use)

    def set_outflow_pressure_correction_factor(self, factor: float):
        """Parameter::setOutflowPressureCorrectionFactor (OutflowNonReflectivePressureCorrection)."""
        self.outflow_pressure_correction_factor = float(factor)

    def set_forcing(self, fx: float, fy: float, fz: float):
        self.forcing = (float(fx), float(fy), float(fz))

    @property
    def omega(self) -> float:
        """omega = 1 / (3 nu + 1/2) (Parameter.cpp:406)."""
        return 1.0 / (3.0 * self.viscosity_lb + 0.5)

    def omega_of_level(self, level: int) -> float:
        """omega of a refinement level: nu 2^level in that level's units (Parameter.cpp:404-406)."""
        return 1.0 / (3.0 * (self.viscosity_lb * 2.0 ** level) + 0.5)

    @classmethod
    def from_configuration_file(cls, path) -> "Parameter":
        """A Parameter from a configuration file of the reference (basics/config/ConfigurationFile
        read by Parameter::readConfigData, Parameter.cpp:80-300): the keys of this path --
        Viscosity_LB, Velocity_LB, ForcingX/Y/Z (0 when absent), QuadricLimiterP/M/D (0.01 when
        absent), UseInitNeq and MainKernelName -- with the reference's meaning. Every key of the file
        stays readable in ``config`` (strings)."""
        cfg = load_configuration_file(path)
        p = cls()
        p.config = cfg
        if "Viscosity_LB" in cfg:
            p.set_viscosity_lb(float(cfg["Viscosity_LB"]))
        if "Velocity_LB" in cfg:
            p.set_velocity_lb(float(cfg["Velocity_LB"]))
        p.set_forcing(*(float(cfg.get(k, 0.0)) for k in ("ForcingX", "ForcingY", "ForcingZ")))
        p.set_quadric_limiters(*(float(cfg.get(k, 0.01)) for k in ("QuadricLimiterP", "QuadricLimiterM",
                                                                     "QuadricLimiterD")))
        if "UseInitNeq" in cfg:
            p.set_use_init_neq(config_bool(cfg["UseInitNeq"]))
        if "MainKernelName" in cfg:
            p.configure_main_kernel(cfg["MainKernelName"])
        return p

    # Parameter::checkParameterValidityCumulantK17 (Parameter.cpp:424-445): K17 with its
    # 4th-order modified equilibrium is unstable above these values
    K17_VISCOSITY_LIMIT = 1.0 / 42.0
    K17_VELOCITY_LIMIT = 0.1

    def check_parameter_validity_cumulant_k17(self, finest_level: int = 0) -> list:
        """The reference's K17 checks: a warning (K17ParameterWarning) when the viscosity of the
        finest level exceeds 1/42 or the velocity set by set_velocity_lb exceeds 0.1, nothing for
        another main kernel. Simulation runs it once, as the reference's initLBMSimulationParameter
        does. Returns the warning texts."""
        if self.main_kernel != "K17CompressibleNavierStokes":
            return []
        out = []
        nu = self.viscosity_lb * 2.0 ** finest_level
        if nu > self.K17_VISCOSITY_LIMIT:
            out.append(f"The viscosity (in LB units) at level {finest_level} is {nu:1.3g}. It is recommended to keep "
                       f"it smaller than {self.K17_VISCOSITY_LIMIT:1.3g} for the CumulantK17 collision kernel.")
        if self.velocity_lb > self.K17_VELOCITY_LIMIT:
            out.append(f"The velocity (in LB units) is {self.velocity_lb:1.4g}. It is recommended to keep it smaller "
                       f"than {self.K17_VELOCITY_LIMIT:1.4g} for the CumulantK17 collision kernel.")
        for msg in out:
            warnings.warn(msg, K17ParameterWarning, stacklevel=2)
        return out


def load_configuration_file(path) -> dict:
    """key = value lines as the reference's ConfigurationFile::load reads them
    (basics/config/ConfigurationFile.cpp:60-100): everything after '#' is a comment, key and value
    are trimmed of spaces, tabs and line ends, lines without '=' or with an empty key or value are
    skipped, a later line wins. A missing file is an error (std::invalid_argument there,
    FileNotFoundError here)."""
    out = {}
    with open(path, "r") as f:
        for line in f:
            line = line.split("#", 1)[0]
            if "=" not in line:
                continue
            key, value = line.split("=", 1)
            key, value = key.strip(" \t\n\r"), value.strip(" \t\n\r")
            if key and value:
                out[key] = value
    return out


def config_bool(value: str) -> bool:
    """ConfigurationFile's bool: true only for the text 'true' (ConfigurationFile.cpp:50-53)."""
    return value == "true"


class K17ParameterWarning(UserWarning):
    """A K17 parameter outside the range the reference recommends (the reference logs a warning)."""


class BoundaryConditionFactory:
    """Enums and setters of the reference BoundaryConditionFactory."""

    class VelocityBC(enum.IntEnum):
        VelocityBounceBack = N.VELOCITY_BOUNCE_BACK
        VelocityInterpolatedIncompressible = N.VELOCITY_INTERPOLATED_INCOMPRESSIBLE
        VelocityInterpolatedCompressible = N.VELOCITY_INTERPOLATED_COMPRESSIBLE
        VelocityWithPressureInterpolatedCompressible = N.VELOCITY_WITH_PRESSURE_INTERPOLATED_COMPRESSIBLE
        NotSpecified = N.VELOCITY_NOT_SPECIFIED

    class NoSlipBC(enum.IntEnum):
        NoSlipDelayBounceBack = N.NOSLIP_DELAY_BOUNCE_BACK
        NoSlipBounceBack = N.NOSLIP_BOUNCE_BACK
        NoSlipInterpolatedIncompressible = N.NOSLIP_INTERPOLATED_INCOMPRESSIBLE
        NoSlipInterpolatedCompressible = N.NOSLIP_INTERPOLATED_COMPRESSIBLE

    class SlipBC(enum.IntEnum):
        SlipCompressible = N.SLIP_COMPRESSIBLE
        SlipTurbulentViscosityCompressible = N.SLIP_TURBULENT_VISCOSITY_COMPRESSIBLE
        NotSpecified = N.SLIP_NOT_SPECIFIED

    class PressureBC(enum.IntEnum):
        PressureNonEquilibriumIncompressible = N.PRESSURE_NON_EQUILIBRIUM_INCOMPRESSIBLE
        PressureNonEquilibriumCompressible = N.PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE
        OutflowNonReflective = N.PRESSURE_OUTFLOW_NON_REFLECTIVE
        OutflowNonReflectivePressureCorrection = N.PRESSURE_OUTFLOW_NON_REFLECTIVE_PRESSURE_CORRECTION
        NotSpecified = N.PRESSURE_NOT_SPECIFIED

    def __init__(self):
        # defaults of the reference (BoundaryConditionFactory.h:168-176)
        self.velocity = self.VelocityBC.NotSpecified
        self.noslip = self.NoSlipBC.NoSlipDelayBounceBack
        self.pressure = self.PressureBC.NotSpecified
        self.slip = self.SlipBC.NotSpecified
        self.geometry = self.NoSlipBC.NoSlipDelayBounceBack

    def set_velocity_boundary_condition(self, v):
        self.velocity = self.VelocityBC(v)

    def set_no_slip_boundary_condition(self, v):
        self.noslip = self.NoSlipBC(v)

    def set_pressure_boundary_condition(self, v):
        self.pressure = self.PressureBC(v)

    def set_slip_boundary_condition(self, v):
        self.slip = self.SlipBC(v)

    def set_geometry_boundary_condition(self, v):
        """setGeometryBoundaryCondition: a VelocityBC, NoSlipBC or SlipBC value (a plain int is a NoSlipBC)."""
        if isinstance(v, (self.VelocityBC, self.SlipBC)):
            self.geometry = v
        else:
            self.geometry = self.NoSlipBC(v)

    def geometry_family(self) -> int:
        """The family of the geometry BC for vfb_simulation_set_geometry_bc_of."""
        if isinstance(self.geometry, self.VelocityBC):
            return N.GEOMETRY_VELOCITY
        if isinstance(self.geometry, self.SlipBC):
            return N.GEOMETRY_SLIP
        return N.GEOMETRY_NOSLIP

    def velocity_function(self):
        fn = C.c_void_p()
        N.check(N.lib().vfb_bc_factory_velocity(int(self.velocity), C.byref(fn)))
        return fn.value

    def noslip_function(self):
        fn = C.c_void_p()
        N.check(N.lib().vfb_bc_factory_noslip(int(self.noslip), C.byref(fn)))
        return fn.value

    def pressure_function(self):
        fn = C.c_void_p()
        N.check(N.lib().vfb_bc_factory_pressure(int(self.pressure), C.byref(fn)))
        return fn.value


class GridScalingFactory:
    """GridScalingFactory (src/gpu/core/GridScaling/GridScalingFactory.h:47-66): the choice of the
    interpolation between levels; NotSpecified by default."""

    class GridScaling(enum.IntEnum):
        ScaleCompressible = N.SCALE_COMPRESSIBLE
        NotSpecified = N.SCALE_NOT_SPECIFIED

    def __init__(self):
        self.grid_scaling_type = self.GridScaling.NotSpecified

    def set_scaling_factory(self, grid_scaling_type):
        self.grid_scaling_type = self.GridScaling(grid_scaling_type)

    def get_grid_scaling_fc(self, has_turbulent_viscosity: bool = False):
        fn = C.c_void_p()
        N.check(N.lib().vfb_scaling_factory_fine_to_coarse(int(self.grid_scaling_type), int(has_turbulent_viscosity),
                                                             C.byref(fn)))
        return fn.value

    def get_grid_scaling_cf(self, has_turbulent_viscosity: bool = False):
        fn = C.c_void_p()
        N.check(N.lib().vfb_scaling_factory_coarse_to_fine(int(self.grid_scaling_type), int(has_turbulent_viscosity),
                                                             C.byref(fn)))
        return fn.value


class InterpolationCells:
    """ICells + ICellNeigh (src/gpu/core/Calculation/Calculation.h:72-87) on the device.

    fine_cell_indices: MMM node of each cell on the fine level; coarse_cell_indices: the MMM node
    of the coarse cell (coarse to fine) or the coarse node at the cell centre (fine to coarse);
    offsets: (3, n) offsets of the expansion point, 0 in the bulk."""

    def __init__(self, fine_cell_indices, coarse_cell_indices, offsets=None, storage=N.STORAGE_F64, device="cuda"):
        t = _torch()
        fine_cell_indices = np.asarray(fine_cell_indices)
        coarse_cell_indices = np.asarray(coarse_cell_indices)
        n = fine_cell_indices.size
        if coarse_cell_indices.size != n:
            raise ValueError("fine and coarse cell lists differ in length")
        off = np.zeros((3, n)) if offsets is None else np.asarray(offsets, dtype=np.float64).reshape(3, n)
        rd = real_dtype(storage)
        self.fine = t.from_numpy(fine_cell_indices.astype(np.int32)).to(device)
        self.coarse = t.from_numpy(coarse_cell_indices.astype(np.int32)).to(device)
        self.offsets = [t.from_numpy(off[a].copy()).to(device=device, dtype=rd) for a in range(3)]
        self.cells = N.InterpolationCells(self.fine.data_ptr(), self.coarse.data_ptr(), n)
        self.neighbor = N.InterpolationCellNeighbor(*(o.data_ptr() for o in self.offsets))

    @property
    def number_of_cells(self) -> int:
        return int(self.cells.number_of_cells)


def _run_scaling(name, coarse, fine, cells, stream):
    N.check(getattr(N.lib(), name)(C.byref(coarse.level), C.byref(fine.level), C.byref(cells.cells),
                                   C.byref(cells.neighbor), stream))


def scale_coarse_to_fine(coarse, fine, cells: InterpolationCells, stream=None):
    """scaleCoarseToFineCompressible (GridScaling/Scaling.cu:106) between two Simulation levels."""
    _run_scaling("vfb_scale_coarse_to_fine_compressible", coarse, fine, cells, stream)


def scale_fine_to_coarse(coarse, fine, cells: InterpolationCells, stream=None):
    """scaleFineToCoarseCompressible (GridScaling/Scaling.cu:156) between two Simulation levels."""
    _run_scaling("vfb_scale_fine_to_coarse_compressible", coarse, fine, cells, stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


class _LevelState:
    """Device arrays of one level (LBMSimulationParameter of that level) and its BC lists."""

    def neighbor_inverse_device(self):
        """neighborInverse of the level's grid on the device, uploaded on first use."""
        inv = getattr(self, "_nb_inv", None)
        if inv is None:
            host = getattr(self.grid, "neighbor_inverse", None)
            if host is None:                      # an imported grid without it: from the +1 lists
                from .grid import inverse_neighbors
                host = inverse_neighbors(self.grid.neighbor)
            inv = _torch().from_numpy(np.asarray(host).astype(np.int32)).to(self.dist.device)
            self._nb_inv = inv
        return inv

    def __init__(self, para: Parameter, grid: ListGrid, level: int, device):
        t = _torch()
        self.grid = grid
        sd, rd = storage_dtype(para.storage), real_dtype(para.storage)
        n = grid.number_of_nodes
        self.dist = t.zeros(27 * n, dtype=sd, device=device)
        self.nb = [t.from_numpy(grid.neighbor[a].astype(np.int32)).to(device) for a in range(3)]
        self.geo = t.from_numpy(grid.geo.astype(np.int32)).to(device)
        self.fluid = t.from_numpy(grid.fluid.astype(np.int32)).to(device)
        self.rho = t.zeros(n, dtype=rd, device=device)
        self.vx = t.zeros(n, dtype=rd, device=device)
        self.vy = t.zeros(n, dtype=rd, device=device)
        self.vz = t.zeros(n, dtype=rd, device=device)
        self.press = t.zeros(n, dtype=rd, device=device)
        L = N.Level()
        L.storage = para.storage
        L.arith = para.arith
        L.is_even_timestep = 1
        L.level = level
        L.number_of_nodes = n
        L.distributions = self.dist.data_ptr()
        L.neighbor_x, L.neighbor_y, L.neighbor_z = (x.data_ptr() for x in self.nb)
        L.type_of_grid_node = self.geo.data_ptr()
        L.omega = para.omega_of_level(level)
        for i in range(3):
            L.forces[i] = para.forcing[i]
            L.quadric_limiters[i] = para.quadric_limiters[i]
        L.rho, L.velocity_x, L.velocity_y, L.velocity_z = (x.data_ptr() for x in (self.rho, self.vx, self.vy, self.vz))
        L.pressure = self.press.data_ptr()
        L.outflow_pressure_correction_factor = para.outflow_pressure_correction_factor
        self.level = L
        self.keep = []
        self.bcs = {}
        for kind in ("velocity", "noslip", "slip", "geometry"):
            m = grid.merged(kind)
            if m is None:
                continue
            k, q, vel = m
            kt = t.from_numpy(k.astype(np.int32)).to(device)
            qt = t.from_numpy(q.reshape(-1)).to(device=device, dtype=rd)
            vt = [t.from_numpy(vel[a].copy()).to(device=device, dtype=rd) for a in range(3)]
            bc = N.BC(kt.data_ptr(), qt.data_ptr(), k.size, vt[0].data_ptr(), vt[1].data_ptr(), vt[2].data_ptr())
            self.keep += [kt, qt] + vt
            self.bcs[kind] = bc
        self.pressure = []
        from .grid import SIDE_DIR
        for b in grid.bcs:
            if b.kind != "pressure":
                continue
            kt = t.from_numpy(b.k.astype(np.int32)).to(device)
            knt = t.from_numpy(b.k_neighbor.astype(np.int32)).to(device)
            rt = t.from_numpy(np.broadcast_to(np.asarray(b.rho, dtype=np.float64), (b.k.size,)).copy()).to(device, rd)
            self.keep += [kt, knt, rt]
            self.pressure.append(N.DirectionalBC(kt.data_ptr(), knt.data_ptr(), rt.data_ptr(), b.k.size, SIDE_DIR[b.side]))


class Simulation:
    """The time loop (UpdateGrid27::updateGrid) of a uniform grid or of nested refinement levels,
    driven by ``vfb_simulation_*`` of the native library.

    grid is a :class:`ListGrid` (one level) or a :class:`MultiLevelGrid`; with more than one level
    the scaling factory (GridScalingFactory) chooses the interpolation between them, as the
    reference's ``Simulation(para, gridBuilder, bcFactory, scalingFactory)``. neighbor_tables selects
    the collision's neighbour slot tables (``vfb_simulation_set_neighbor_tables``: 0 none, 1 direct
    loads, 2 staged by bulk copies; True = 1). The attributes
    ``grid``, ``level``, ``dist``, ``rho`` ... are those of the coarsest level; ``levels`` holds all."""

    def __init__(self, para: Parameter, grid, bc_factory: BoundaryConditionFactory,
                 scaling_factory: GridScalingFactory | None = None, device="cuda", neighbor_tables=True):
        if para.main_kernel is None:
            raise N.VfbError(N.VFB_ERR_UNKNOWN_KERNEL, "no main kernel configured")
        t = _torch()
        self.para, self.bcf, self.device = para, bc_factory, device
        finest = len(grid.levels) - 1 if hasattr(grid, "levels") else 0
        para.check_parameter_validity_cumulant_k17(finest)
        # nested levels (MultiLevelGrid, or an imported gridgen.ImportedGrid), or a single level
        self.multilevel = grid if hasattr(grid, "interfaces") else MultiLevelGrid.uniform(grid)
        self.levels = [_LevelState(para, g, i, device) for i, g in enumerate(self.multilevel.levels)]
        base = self.levels[0]
        self.grid, self.level, self.dist, self.fluid = base.grid, base.level, base.dist, base.fluid
        self.nb, self.geo = base.nb, base.geo
        self.rho, self.vx, self.vy, self.vz, self.press = base.rho, base.vx, base.vy, base.vz, base.press
        self._bcs = base.bcs
        sim = C.c_void_p()
        N.check(N.lib().vfb_simulation_create(para.main_kernel.encode(), C.byref(sim)))
        self._sim = sim
        N.check(N.lib().vfb_simulation_set_neighbor_tables(sim, int(neighbor_tables)))
        for i, S in enumerate(self.levels):
            N.check(N.lib().vfb_simulation_use_level(sim, i))
            N.check(N.lib().vfb_simulation_set_level(sim, C.byref(S.level), _ptr(S.fluid), int(S.grid.fluid.size)))
            if "velocity" in S.bcs:
                N.check(N.lib().vfb_simulation_set_velocity_bc(sim, C.byref(S.bcs["velocity"]), int(bc_factory.velocity)))
            if "noslip" in S.bcs:
                N.check(N.lib().vfb_simulation_set_noslip_bc(sim, C.byref(S.bcs["noslip"]), int(bc_factory.noslip)))
            if "slip" in S.bcs:
                N.check(N.lib().vfb_simulation_set_slip_bc(sim, C.byref(S.bcs["slip"]), int(bc_factory.slip)))
            if "geometry" in S.bcs:
                N.check(N.lib().vfb_simulation_set_geometry_bc_of(sim, C.byref(S.bcs["geometry"]),
                                                                  bc_factory.geometry_family(),
                                                                  int(bc_factory.geometry)))
            for p in S.pressure:
                N.check(N.lib().vfb_simulation_add_pressure_bc(sim, C.byref(p), int(bc_factory.pressure)))
        self._cells = []
        if scaling_factory is not None:
            N.check(N.lib().vfb_simulation_set_scaling_factory(sim, int(scaling_factory.grid_scaling_type), 0))
        for i, iface in enumerate(self.multilevel.interfaces):
            fc = InterpolationCells(iface.fine_fc, iface.coarse_fc, iface.offsets_fc, storage=para.storage, device=device)
            cf = InterpolationCells(iface.fine_cf, iface.coarse_cf, iface.offsets_cf, storage=para.storage, device=device)
            self._cells.append((fc, cf))
            N.check(N.lib().vfb_simulation_set_interpolation_cells(sim, i, C.byref(fc.cells), C.byref(fc.neighbor),
                                                                   C.byref(cf.cells), C.byref(cf.neighbor)))
        N.check(N.lib().vfb_simulation_use_level(sim, 0))
        self._drag = None
        N.check(N.lib().vfb_simulation_check(sim))

    def close(self):
        if getattr(self, "_sim", None):
            N.lib().vfb_simulation_destroy(self._sim)
            self._sim = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self, rho=None, vx=None, vy=None, vz=None, level=0):
        """PreProcessorImp::init of one level: equilibrium for the odd, then the even parity; starts even.
        With Parameter.use_init_neq the non-equilibrium part from the velocity gradients is added
        (InitNavierStokesCompressibleNonEquilibrium_Device; the grid's neighborInverse is needed)."""
        t = _torch()
        S = self.levels[level]
        rd = real_dtype(self.para.storage)
        for arr, dst in ((rho, S.rho), (vx, S.vx), (vy, S.vy), (vz, S.vz)):
            if arr is None:
                dst.zero_()
            else:
                dst.copy_(t.as_tensor(np.asarray(arr), dtype=rd))
        L = S.level
        if self.para.use_init_neq:
            inv = S.neighbor_inverse_device()
            init = lambda: N.lib().vfb_init_navier_stokes_compressible_non_equilibrium(C.byref(L), _ptr(inv), None)
        else:
            init = lambda: N.lib().vfb_init_navier_stokes_compressible(C.byref(L), None)
        L.is_even_timestep = 0
        N.check(init())
        L.is_even_timestep = 1
        N.check(init())
        N.check(N.lib().vfb_simulation_use_level(self._sim, level))
        N.check(N.lib().vfb_simulation_set_level(self._sim, C.byref(L), _ptr(S.fluid), int(S.grid.fluid.size)))
        N.check(N.lib().vfb_simulation_use_level(self._sim, 0))

    PHASES = ("collision", "postCollisionBC", "preCollisionBC", "scalingFineToCoarse", "scalingCoarseToFine")

    def set_timing(self, on: bool = True):
        """Phase timers of the step driver (the reference's TimeStepTimer phases plus the two
        interpolation directions): device time per phase from CUDA events, added up once at the end
        of every run call (which then synchronises)."""
        N.check(N.lib().vfb_simulation_set_timing(self._sim, int(bool(on))))

    def phase_times(self, reset: bool = False):
        """{phase: milliseconds} summed over the timed runs and all levels, and the coarse steps."""
        ms = (C.c_double * len(self.PHASES))()
        steps = C.c_uint64()
        N.check(N.lib().vfb_simulation_phase_times(self._sim, ms, C.byref(steps), int(bool(reset))))
        return dict(zip(self.PHASES, ms)), steps.value

    def set_graph(self, steps: int = 16):
        """Run the step loop as a CUDA graph of `steps` coarse steps (even; 0 turns it off), replayed
        on a stream of this simulation's own (vfb_simulation_set_graph). Results are the same bits."""
        N.check(N.lib().vfb_simulation_set_graph(self._sim, int(steps)))
        self._graph_stream = _torch().cuda.Stream() if steps else None

    def run(self, steps: int):
        """steps time steps of the coarsest level (each finer level takes twice its coarser one's)."""
        gs = getattr(self, "_graph_stream", None)
        if gs is None:
            N.check(N.lib().vfb_simulation_run(self._sim, int(steps), None))
        else:
            t = _torch()
            gs.wait_stream(t.cuda.current_stream())
            N.check(N.lib().vfb_simulation_run(self._sim, int(steps), C.c_void_p(gs.cuda_stream)))
            t.cuda.current_stream().wait_stream(gs)
        self._drag_steps = getattr(self, "_drag_steps", 0) + int(steps) if self._drag is not None else 0
        for i, S in enumerate(self.levels):
            ev = C.c_int32()
            N.check(N.lib().vfb_simulation_level_is_even_timestep(self._sim, i, C.byref(ev)))
            S.level.is_even_timestep = ev.value

    def macroscopic(self, level=0):
        """drho, vx, vy, vz, pressure of every node of a level (zeros on non-fluid nodes), as numpy."""
        S = self.levels[level]
        N.check(N.lib().vfb_calc_macroscopic_compressible(C.byref(S.level), None))
        N.check(N.lib().vfb_synchronize(None))
        return {k: v.double().cpu().numpy() for k, v in
                (("rho", S.rho), ("vx", S.vx), ("vy", S.vy), ("vz", S.vz), ("pressure", S.press))}

    def mass_energy(self, level=0):
        t = _torch()
        S = self.levels[level]
        nf = int(S.grid.fluid.size)
        nbytes = N.lib().vfb_mass_energy_workspace_bytes(nf)
        ws = t.empty((nbytes + 7) // 8, dtype=t.float64, device=self.device)
        out = (C.c_double * 2)()
        N.check(N.lib().vfb_mass_energy(C.byref(S.level), _ptr(S.fluid), nf, C.c_void_p(ws.data_ptr()), nbytes, out,
                                        None))
        return out[0], out[1]

    def enable_drag_lift(self, history_steps: int):
        """Parameter::setCalcDragLift: the drag/lift force on the geometry every step, kept on the
        device for the last history_steps steps."""
        t = _torch()
        if "geometry" not in self._bcs:
            raise N.VfbError(N.VFB_ERR_INVALID_ARGUMENT, "drag and lift need a geometry boundary condition")
        ng = int(self._bcs["geometry"].number_of_bc_nodes)
        nbytes = N.lib().vfb_simulation_drag_lift_workspace_bytes(ng)
        ws = t.zeros((nbytes + 7) // 8, dtype=t.float64, device=self.device)
        hist = t.zeros(3 * int(history_steps), dtype=t.float64, device=self.device)
        N.check(N.lib().vfb_simulation_set_drag_lift(self._sim, C.c_void_p(ws.data_ptr()), nbytes,
                                                     C.c_void_p(hist.data_ptr()), int(history_steps)))
        self._drag = (ws, hist, int(history_steps), 0)

    def drag_lift_history(self):
        """(steps, 3) forces of the steps run since drag/lift was enabled (the last history_steps)."""
        ws, hist, length, _ = self._drag
        N.check(N.lib().vfb_synchronize(None))
        h = hist.view(length, 3).cpu().numpy()
        done = self._drag_steps
        if done <= length:
            return h[:done].copy()
        start = done % length
        return np.concatenate([h[start:], h[:start]])

    def populations(self, level=0):
        """The population array of a level as float64 values: f - w for F64 / F32 storage, (f - w)/w
        for the 16-bit forms (E3M12 decoded)."""
        N.check(N.lib().vfb_synchronize(None))
        if self.para.storage == N.STORAGE_E3M12:
            from .formats import decode
            return decode(self._raw(level))
        return self.levels[level].dist.double().cpu().numpy()

    def _raw(self, level):
        """The population array of a level as stored (16-bit storage as raw uint16)."""
        t = _torch()
        N.check(N.lib().vfb_synchronize(None))
        d = self.levels[level].dist
        if d.dtype in (t.float16, t.bfloat16, t.int16):
            return d.view(t.int16).cpu().numpy().view(np.uint16)
        return d.cpu().numpy()

    def write_vtk(self, path, level=0):
        """drho, velocity and pressure of a level's fluid nodes at their positions (units of the
        coarsest spacing), as a legacy VTK file."""
        from .output import write_vtk_points
        m = self.macroscopic(level)
        f = self.levels[level].grid.fluid
        write_vtk_points(path, self.multilevel.positions(level)[:, f],
                         {"drho": m["rho"][f], "velocity": np.stack([m["vx"][f], m["vy"][f], m["vz"][f]]),
                          "pressure": m["pressure"][f]}, title=f"level {level}")

    def check_slots(self):
        """The host check of every level's esoteric-twist write pattern (checks.check_grid): each
        slot written once per step by the collision and by the BC lists, in both parities. Returns
        the per-level reports; raises ValueError on the first level with a conflict."""
        from .checks import assert_slots_written_once
        return [assert_slots_written_once(S.grid) for S in self.levels]

    def write_vtu(self, prefix, timestep, last=False, writer=None):
        """Every level's fields in the reference's output files (FileWriter::writeTimestep,
        Output/FileWriter.cpp:104-137): part files of octs with press, rho, vx1, vx2, vx3 and geo,
        the time step's .pvtu collection and, with last=True, the .pvd time series. Positions are
        in units of the coarsest spacing. Pass the same `writer` (output.FileWriter) for every time
        step of a run so that the time series lists them all; returns (writer, files)."""
        from .output import FileWriter
        writer = writer or FileWriter(prefix)
        levels = []
        for lev, S in enumerate(self.levels):
            m = self.macroscopic(lev)
            g = S.grid
            levels.append(dict(coords=self.multilevel.positions(lev), spacing=float(self.multilevel.spacing[lev]),
                               geo=g.geo, neighbor=g.neighbor, rho=m["rho"], vx=m["vx"], vy=m["vy"], vz=m["vz"],
                               pressure=m["pressure"]))
        return writer, writer.write_timestep(timestep, levels, last=last)

    def save_restart(self, path):
        """RestartObject::serialize (binary): every level's population array, `path` + ".bin"."""
        from .output import save_restart
        save_restart(path, [self._raw(i) for i in range(len(self.levels))])

    def load_restart(self, path, timestep=0):
        """RestartObject::deserialize: the population arrays of every level; the coarsest level is
        at the parity of `timestep` (even when it is even), finer levels at the even parity."""
        from .output import load_restart
        t = _torch()
        dts = [self._raw(i).dtype for i in range(len(self.levels))]
        arrs = load_restart(path, dts)
        for i, (S, a) in enumerate(zip(self.levels, arrs)):
            if a.size != S.dist.numel():
                raise ValueError(f"level {i}: {a.size} values in the file, {S.dist.numel()} expected")
            src = t.from_numpy(a.view(np.int16) if a.dtype == np.uint16 else a)
            if S.dist.dtype in (t.float16, t.bfloat16):
                S.dist.view(t.int16).copy_(src)
            else:
                S.dist.copy_(src)
            S.level.is_even_timestep = int(timestep % 2 == 0) if i == 0 else 1
            N.check(N.lib().vfb_simulation_use_level(self._sim, i))
            N.check(N.lib().vfb_simulation_set_level(self._sim, C.byref(S.level), _ptr(S.fluid),
                                                     int(S.grid.fluid.size)))
        N.check(N.lib().vfb_simulation_use_level(self._sim, 0))
