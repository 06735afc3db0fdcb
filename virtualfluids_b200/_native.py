"""ctypes binding of the C ABI in ``include/vfb.h`` (the native library ``libvfb.so``).

Loading fails loudly: there is no Python or CPU fallback for any kernel. Structures mirror the
C declarations field for field.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# VFB_LIBRARY=checked loads the bounds-checked build (libvfb_checked.so) instead of the default one
_LIB_PATH = Path(__file__).resolve().parent / (
    "libvfb_checked.so" if os.environ.get("VFB_LIBRARY", "") == "checked" else "libvfb.so")

VFB_OK = 0
VFB_ERR_INVALID_ARGUMENT = 1
VFB_ERR_UNKNOWN_KERNEL = 2
VFB_ERR_BC_UNSET = 3
VFB_ERR_SCALING_UNSET = 4
VFB_ERR_CUDA = 5
VFB_ERR_OUT_OF_MEMORY = 6
VFB_ERR_UNSUPPORTED = 7
VFB_ERR_WATCHDOG = 8

STORAGE_F64, STORAGE_F32, STORAGE_F16, STORAGE_BF16, STORAGE_E3M12 = 0, 1, 2, 3, 4
VFB_IPC_HANDLE_BYTES = 64
ARITH_FAST, ARITH_EXACT = 0, 1

COLLISION_DEFAULT = 0
COLLISION_WRITE_MACRO_VARS = 1
COLLISION_APPLY_BODY_FORCE = 2
COLLISION_ALL_FEATURES = 3
COLLISION_SUBDOMAIN_BORDER = 4

DIR_P00, DIR_M00, DIR_0P0, DIR_0M0, DIR_00P, DIR_00M = 1, 2, 3, 4, 5, 6
GEO_SOLID, GEO_VOID, GEO_FLUID = 15, 16, 19

# BoundaryConditionFactory enums (BoundaryConditionFactory.h:60-130)
VELOCITY_BOUNCE_BACK = 0
VELOCITY_INTERPOLATED_INCOMPRESSIBLE = 1
VELOCITY_INTERPOLATED_COMPRESSIBLE = 2
VELOCITY_WITH_PRESSURE_INTERPOLATED_COMPRESSIBLE = 3
VELOCITY_NOT_SPECIFIED = 4
NOSLIP_DELAY_BOUNCE_BACK = 0
NOSLIP_BOUNCE_BACK = 1
NOSLIP_INTERPOLATED_INCOMPRESSIBLE = 2
NOSLIP_INTERPOLATED_COMPRESSIBLE = 3
SLIP_COMPRESSIBLE, SLIP_TURBULENT_VISCOSITY_COMPRESSIBLE, SLIP_NOT_SPECIFIED = 0, 1, 2
GEOMETRY_VELOCITY, GEOMETRY_NOSLIP, GEOMETRY_SLIP = 0, 1, 2
PRESSURE_NON_EQUILIBRIUM_INCOMPRESSIBLE = 0
PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE = 1
PRESSURE_OUTFLOW_NON_REFLECTIVE = 2
PRESSURE_OUTFLOW_NON_REFLECTIVE_PRESSURE_CORRECTION = 3
PRESSURE_NOT_SPECIFIED = 4
# GridScalingFactory::GridScaling (GridScalingFactory.h:50-56)
BOX_BC_VELOCITY, BOX_BC_NOSLIP, BOX_BC_GEOMETRY, BOX_BC_SLIP = 0, 1, 2, 3
SCALE_COMPRESSIBLE = 0
SCALE_NOT_SPECIFIED = 1


class VfbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class Level(C.Structure):
    _fields_ = [
        ("storage", C.c_int32), ("arith", C.c_int32), ("is_even_timestep", C.c_int32), ("level", C.c_int32),
        ("number_of_nodes", C.c_uint64), ("distributions", C.c_void_p),
        ("neighbor_x", C.c_void_p), ("neighbor_y", C.c_void_p), ("neighbor_z", C.c_void_p),
        ("type_of_grid_node", C.c_void_p), ("omega", C.c_double), ("forces", C.c_double * 3),
        ("quadric_limiters", C.c_double * 3), ("rho", C.c_void_p), ("velocity_x", C.c_void_p),
        ("velocity_y", C.c_void_p), ("velocity_z", C.c_void_p), ("pressure", C.c_void_p),
        ("body_force_x", C.c_void_p), ("body_force_y", C.c_void_p), ("body_force_z", C.c_void_p),
        ("outflow_pressure_correction_factor", C.c_double),
    ]


class BC(C.Structure):
    _fields_ = [("k", C.c_void_p), ("q27", C.c_void_p), ("number_of_bc_nodes", C.c_uint32),
                ("vx", C.c_void_p), ("vy", C.c_void_p), ("vz", C.c_void_p)]


class DirectionalBC(C.Structure):
    _fields_ = [("k", C.c_void_p), ("k_neighbor", C.c_void_p), ("rho_bc", C.c_void_p),
                ("number_of_bc_nodes", C.c_uint32), ("direction", C.c_int32)]


class InterpolationCells(C.Structure):
    _fields_ = [("fine_cell_indices", C.c_void_p), ("coarse_cell_indices", C.c_void_p),
                ("number_of_cells", C.c_uint32)]


class InterpolationCellNeighbor(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p)]


class BoxDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("periodic_z", C.c_int32),
                ("storage", C.c_int32), ("arith", C.c_int32), ("omega", C.c_double),
                ("forces", C.c_double * 3), ("quadric_limiters", C.c_double * 3), ("mask", C.c_void_p)]


class PoolDesc(C.Structure):
    _fields_ = [("storage", C.c_int32), ("arith", C.c_int32), ("arena_bytes", C.c_uint64), ("max_domains", C.c_uint32)]


class DomainDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("periodic_z", C.c_int32),
                ("omega", C.c_double), ("forces", C.c_double * 3), ("quadric_limiters", C.c_double * 3)]


class DomainBCs(C.Structure):
    _fields_ = [("noslip_variant", C.c_int32), ("noslip_k", C.c_void_p), ("noslip_q27", C.c_void_p),
                ("number_of_noslip_nodes", C.c_uint32), ("pressure_variant", C.c_int32), ("pressure_k", C.c_void_p),
                ("pressure_k_neighbor", C.c_void_p), ("pressure_rho", C.c_void_p), ("pressure_direction", C.c_void_p),
                ("number_of_pressure_nodes", C.c_uint32)]


BC_FN = C.CFUNCTYPE(C.c_int, C.POINTER(Level), C.POINTER(BC), C.c_void_p)
DBC_FN = C.CFUNCTYPE(C.c_int, C.POINTER(Level), C.POINTER(DirectionalBC), C.c_void_p)

# exported symbols and their signatures (restype, argtypes); also the list tests check against vfb.h
SIGNATURES = {
    "vfb_abi_version": (C.c_int, []),
    "vfb_last_error": (C.c_char_p, []),
    "vfb_status_string": (C.c_char_p, [C.c_int]),
    "vfb_synchronize": (C.c_int, [C.c_void_p]),
    "vfb_bounds_checked": (C.c_int, []),
    "vfb_bounds_check_status": (C.c_int, [C.c_void_p, C.c_void_p]),
    "vfb_lattice_tables": (C.c_int, [C.c_void_p] * 5),
    "vfb_k17_rates": (C.c_int, [C.c_double, C.c_void_p]),
    "vfb_kernel_lookup": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32)]),
    "vfb_kernel_count": (C.c_int, []),
    "vfb_kernel_name": (C.c_char_p, [C.c_int]),
    "vfb_k17_run_on_indices": (C.c_int, [C.POINTER(Level), C.c_void_p, C.c_uint32, C.c_int32, C.c_void_p]),
    "vfb_k17_plan_create": (C.c_int, [C.POINTER(Level), C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "vfb_k17_plan_run": (C.c_int, [C.c_void_p, C.POINTER(Level), C.c_int32, C.c_void_p]),
    "vfb_k17_plan_box_addressing": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "vfb_k17_plan_destroy": (C.c_int, [C.c_void_p]),
    "vfb_noslip_bounce_back": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p]),
    "vfb_noslip_interpolated_compressible": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p]),
    "vfb_slip_compressible": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p]),
    "vfb_velocity_bounce_back": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p]),
    "vfb_velocity_interpolated_compressible": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p]),
    "vfb_pressure_non_equilibrium_compressible": (C.c_int, [C.POINTER(Level), C.POINTER(DirectionalBC), C.c_void_p]),
    "vfb_scale_coarse_to_fine_compressible": (C.c_int, [C.POINTER(Level), C.POINTER(Level),
                                                        C.POINTER(InterpolationCells),
                                                        C.POINTER(InterpolationCellNeighbor), C.c_void_p]),
    "vfb_scale_fine_to_coarse_compressible": (C.c_int, [C.POINTER(Level), C.POINTER(Level),
                                                        C.POINTER(InterpolationCells),
                                                        C.POINTER(InterpolationCellNeighbor), C.c_void_p]),
    "vfb_drag_lift_post_27": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "vfb_drag_lift_pre_27": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "vfb_drag_lift_workspace_bytes": (C.c_size_t, [C.c_uint32]),
    "vfb_drag_lift_force": (C.c_int, [C.c_void_p] * 6 + [C.c_uint32, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "vfb_pressure_non_equilibrium_incompressible": (C.c_int, [C.POINTER(Level), C.POINTER(DirectionalBC), C.c_void_p]),
    "vfb_outflow_non_reflecting": (C.c_int, [C.POINTER(Level), C.POINTER(DirectionalBC), C.c_void_p]),
    "vfb_outflow_non_reflecting_pressure_correction": (C.c_int, [C.POINTER(Level), C.POINTER(DirectionalBC),
                                                                 C.c_void_p]),
    "vfb_noslip_interpolated_incompressible": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p]),
    "vfb_velocity_interpolated_incompressible": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p]),
    "vfb_velocity_with_pressure_interpolated_compressible": (C.c_int, [C.POINTER(Level), C.POINTER(BC), C.c_void_p]),
    "vfb_init_navier_stokes_compressible": (C.c_int, [C.POINTER(Level), C.c_void_p]),
    "vfb_init_navier_stokes_compressible_non_equilibrium": (C.c_int, [C.POINTER(Level), C.c_void_p, C.c_void_p]),
    "vfb_calc_macroscopic_compressible": (C.c_int, [C.POINTER(Level), C.c_void_p]),
    "vfb_mass_energy_workspace_bytes": (C.c_size_t, [C.c_uint32]),
    "vfb_mass_energy": (C.c_int, [C.POINTER(Level), C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t, C.c_void_p,
                                  C.c_void_p]),
    "vfb_mass_energy_no_alloc": (C.c_int, [C.POINTER(Level), C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "vfb_bc_factory_velocity": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    "vfb_bc_factory_noslip": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    "vfb_bc_factory_slip": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    "vfb_bc_factory_pressure": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    "vfb_scaling_factory_fine_to_coarse": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "vfb_scaling_factory_coarse_to_fine": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "vfb_simulation_create": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "vfb_simulation_destroy": (C.c_int, [C.c_void_p]),
    "vfb_simulation_set_level": (C.c_int, [C.c_void_p, C.POINTER(Level), C.c_void_p, C.c_uint32]),
    "vfb_simulation_set_velocity_bc": (C.c_int, [C.c_void_p, C.POINTER(BC), C.c_int32]),
    "vfb_simulation_set_noslip_bc": (C.c_int, [C.c_void_p, C.POINTER(BC), C.c_int32]),
    "vfb_simulation_add_pressure_bc": (C.c_int, [C.c_void_p, C.POINTER(DirectionalBC), C.c_int32]),
    "vfb_simulation_set_geometry_bc": (C.c_int, [C.c_void_p, C.POINTER(BC), C.c_int32]),
    "vfb_simulation_set_geometry_bc_of": (C.c_int, [C.c_void_p, C.POINTER(BC), C.c_int32, C.c_int32]),
    "vfb_simulation_set_slip_bc": (C.c_int, [C.c_void_p, C.POINTER(BC), C.c_int32]),
    "vfb_simulation_level_box_addressing": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "vfb_simulation_drag_lift_workspace_bytes": (C.c_size_t, [C.c_uint32]),
    "vfb_simulation_set_drag_lift": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_uint32]),
    "vfb_simulation_check": (C.c_int, [C.c_void_p]),
    "vfb_simulation_run": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "vfb_simulation_set_timing": (C.c_int, [C.c_void_p, C.c_int32]),
    "vfb_simulation_set_graph": (C.c_int, [C.c_void_p, C.c_int32]),
    "vfb_simulation_phase_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.c_int32]),
    "vfb_simulation_is_even_timestep": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "vfb_simulation_level_is_even_timestep": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "vfb_simulation_use_level": (C.c_int, [C.c_void_p, C.c_int32]),
    "vfb_pool_domain_mass": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "vfb_pool_watchdog": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32),
                                    C.c_void_p]),
    "vfb_box_read_populations": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_void_p]),
    "vfb_box_write_populations": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "vfb_simulation_set_neighbor_tables": (C.c_int, [C.c_void_p, C.c_int32]),
    "vfb_simulation_status": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.c_void_p]),
    "vfb_simulation_number_of_levels": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "vfb_simulation_set_scaling_factory": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "vfb_simulation_set_interpolation_cells": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(InterpolationCells),
                                                         C.POINTER(InterpolationCellNeighbor),
                                                         C.POINTER(InterpolationCells),
                                                         C.POINTER(InterpolationCellNeighbor)]),
    "vfb_box_create": (C.c_int, [C.POINTER(BoxDesc), C.POINTER(C.c_void_p)]),
    "vfb_box_destroy": (C.c_int, [C.c_void_p]),
    "vfb_box_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "vfb_box_init": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "vfb_box_step": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_int32, C.c_void_p]),
    "vfb_box_fields": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "vfb_box_status": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.c_void_p]),
    "vfb_box_set_kernel_variant": (C.c_int, [C.c_void_p, C.c_int32]),
    "vfb_box_set_bc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
    "vfb_box_add_pressure_bc": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                          C.c_int32]),
    "vfb_box_set_outflow_pressure_correction": (C.c_int, [C.c_void_p, C.c_double]),
    "vfb_box_set_velocity_perturbation": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double]),
    "vfb_box_set_drag_lift": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "vfb_box_kernel_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "vfb_box_set_launch_shape": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "vfb_box_collide_planes": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "vfb_box_collide_border": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "vfb_box_ipc_handle": (C.c_int, [C.c_void_p, C.c_void_p]),
    "vfb_ipc_open": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "vfb_ipc_close": (C.c_int, [C.c_void_p]),
    "vfb_box_toggle_parity": (C.c_int, [C.c_void_p]),
    "vfb_box_populations": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64),
                                      C.POINTER(C.c_int32)]),
    "vfb_pool_create": (C.c_int, [C.POINTER(PoolDesc), C.POINTER(C.c_void_p)]),
    "vfb_pool_destroy": (C.c_int, [C.c_void_p]),
    "vfb_pool_domain_bytes": (C.c_int, [C.c_void_p, C.POINTER(DomainDesc), C.c_int32, C.POINTER(C.c_uint64)]),
    "vfb_pool_add_domain": (C.c_int, [C.c_void_p, C.POINTER(DomainDesc), C.c_void_p, C.POINTER(C.c_uint32)]),
    "vfb_pool_add_domain_with_bcs": (C.c_int, [C.c_void_p, C.POINTER(DomainDesc), C.c_void_p, C.POINTER(DomainBCs),
                                               C.POINTER(C.c_uint32)]),
    "vfb_pool_domain_bytes_with_bcs": (C.c_int, [C.c_void_p, C.POINTER(DomainDesc), C.c_int32, C.POINTER(DomainBCs),
                                                 C.POINTER(C.c_uint64)]),
    "vfb_pool_remove_domain": (C.c_int, [C.c_void_p, C.c_uint32]),
    "vfb_pool_synchronize": (C.c_int, [C.c_void_p, C.c_void_p]),
    "vfb_pool_init_domain": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int32, C.c_void_p]),
    "vfb_pool_step": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "vfb_pool_domain_fields": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_int32, C.c_void_p]),
    "vfb_pool_set_launch": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "vfb_pool_get_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "vfb_pool_autotune": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_double)]),
    "vfb_pool_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                 C.POINTER(C.c_uint64)]),
    "vfb_pool_kernel_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
}

_lib = None


def lib():
    """The loaded native library. Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise ImportError(f"{_LIB_PATH} is missing: build it with `python -m virtualfluids_b200.build`")
        handle = C.CDLL(str(_LIB_PATH), mode=os.RTLD_NOW)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int) -> None:
    if status != VFB_OK:
        msg = lib().vfb_last_error()
        raise VfbError(status, (msg or b"").decode() or lib().vfb_status_string(status).decode())


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
