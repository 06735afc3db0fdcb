"""The C ABI library loads, exports what include/vfb.h declares, and its host logic follows the
reference's registry / factory / manager semantics. No kernel runs here (CPU only)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared_symbols():
    text = (ROOT / "include" / "vfb.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vfb_[a-z0-9_]+)\s*\(", text)) - {"vfb_bc_fn", "vfb_directional_bc_fn"})


def test_library_exports_every_declared_symbol():
    from virtualfluids_b200 import _native as N
    lib = N.lib()
    declared = _declared_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding covers the whole header
    assert set(declared) == set(N.SIGNATURES), set(declared) ^ set(N.SIGNATURES)


def test_abi_version_and_status_strings():
    from virtualfluids_b200 import _native as N
    assert N.lib().vfb_abi_version() == 1
    assert N.lib().vfb_status_string(N.VFB_ERR_UNKNOWN_KERNEL) == b"KernelFactory does not know the KernelType."


def test_lattice_tables_match_oracle(oracle):
    from virtualfluids_b200 import _native as N
    t = [np.zeros(27, dtype=np.int32) for _ in range(4)] + [np.zeros(27)]
    N.check(N.lib().vfb_lattice_tables(*(C.c_void_p(a.ctypes.data) for a in t)))
    L = C.CDLL(str(oracle.LIB))
    for name, arr in zip(("ORC_CX", "ORC_CY", "ORC_CZ", "ORC_INV"), t[:4]):
        ref = np.frombuffer((C.c_int * 27).in_dll(L, name), dtype=np.int32)
        assert np.array_equal(arr, ref), name
    w = np.frombuffer((C.c_double * 27).in_dll(L, "ORC_W"), dtype=np.float64)
    assert np.array_equal(t[4], w)


def test_host_rates_match_oracle_bitwise(oracle):
    """The omega-only K17 rates precomputed on the host equal the per-node reference expressions."""
    from virtualfluids_b200 import _native as N
    lib = oracle.lib()
    lib.orc_k17_rates_f64.argtypes = [C.c_double, C.c_void_p]
    for om in np.linspace(0.55, 1.99, 97):
        a, b = np.zeros(6), np.zeros(6)
        N.check(N.lib().vfb_k17_rates(float(om), C.c_void_p(a.ctypes.data)))
        lib.orc_k17_rates_f64(float(om), oracle.ptr(b))
        assert np.array_equal(a, b), om


def test_kernel_registry():
    from virtualfluids_b200 import _native as N
    kid = C.c_int32()
    N.check(N.lib().vfb_kernel_lookup(b"K17CompressibleNavierStokes", C.byref(kid)))
    assert kid.value == 1
    assert N.lib().vfb_kernel_lookup(b"K15CompressibleNavierStokes", C.byref(kid)) == N.VFB_ERR_UNKNOWN_KERNEL
    assert b"KernelFactory does not know the KernelType" in N.lib().vfb_last_error()
    assert N.lib().vfb_kernel_count() == 1
    assert N.lib().vfb_kernel_name(0) == b"K17CompressibleNavierStokes"
    with pytest.raises(N.VfbError):
        from virtualfluids_b200 import Parameter
        Parameter().configure_main_kernel("NoSuchKernel")


def test_bc_factory_semantics():
    """BoundaryConditionFactoryTest.cpp: defaults give no kernel; each enum maps to its function."""
    from virtualfluids_b200 import _native as N
    lib = N.lib()
    fn = C.c_void_p()
    N.check(lib.vfb_bc_factory_noslip(N.NOSLIP_DELAY_BOUNCE_BACK, C.byref(fn)))
    assert fn.value is None
    N.check(lib.vfb_bc_factory_noslip(N.NOSLIP_BOUNCE_BACK, C.byref(fn)))
    assert fn.value == C.cast(lib.vfb_noslip_bounce_back, C.c_void_p).value
    N.check(lib.vfb_bc_factory_noslip(N.NOSLIP_INTERPOLATED_COMPRESSIBLE, C.byref(fn)))
    assert fn.value == C.cast(lib.vfb_noslip_interpolated_compressible, C.c_void_p).value
    N.check(lib.vfb_bc_factory_velocity(N.VELOCITY_BOUNCE_BACK, C.byref(fn)))
    assert fn.value == C.cast(lib.vfb_velocity_bounce_back, C.c_void_p).value
    N.check(lib.vfb_bc_factory_velocity(N.VELOCITY_INTERPOLATED_COMPRESSIBLE, C.byref(fn)))
    assert fn.value == C.cast(lib.vfb_velocity_interpolated_compressible, C.c_void_p).value
    N.check(lib.vfb_bc_factory_velocity(N.VELOCITY_NOT_SPECIFIED, C.byref(fn)))
    assert fn.value is None
    N.check(lib.vfb_bc_factory_pressure(N.PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE, C.byref(fn)))
    assert fn.value == C.cast(lib.vfb_pressure_non_equilibrium_compressible, C.c_void_p).value
    for factory, variant, name in (
            (lib.vfb_bc_factory_velocity, N.VELOCITY_INTERPOLATED_INCOMPRESSIBLE, "vfb_velocity_interpolated_incompressible"),
            (lib.vfb_bc_factory_velocity, N.VELOCITY_WITH_PRESSURE_INTERPOLATED_COMPRESSIBLE,
             "vfb_velocity_with_pressure_interpolated_compressible"),
            (lib.vfb_bc_factory_noslip, N.NOSLIP_INTERPOLATED_INCOMPRESSIBLE, "vfb_noslip_interpolated_incompressible"),
            (lib.vfb_bc_factory_pressure, N.PRESSURE_NON_EQUILIBRIUM_INCOMPRESSIBLE,
             "vfb_pressure_non_equilibrium_incompressible"),
            (lib.vfb_bc_factory_pressure, N.PRESSURE_OUTFLOW_NON_REFLECTIVE, "vfb_outflow_non_reflecting"),
            (lib.vfb_bc_factory_pressure, N.PRESSURE_OUTFLOW_NON_REFLECTIVE_PRESSURE_CORRECTION,
             "vfb_outflow_non_reflecting_pressure_correction")):
        N.check(factory(variant, C.byref(fn)))
        assert fn.value == C.cast(getattr(lib, name), C.c_void_p).value, name
    assert lib.vfb_bc_factory_noslip(99, C.byref(fn)) == N.VFB_ERR_INVALID_ARGUMENT
    assert lib.vfb_bc_factory_pressure(99, C.byref(fn)) == N.VFB_ERR_INVALID_ARGUMENT


def _fake_level(N):
    """A level description with placeholder device addresses: only host checks run on it."""
    L = N.Level()
    L.storage, L.arith, L.is_even_timestep, L.level = N.STORAGE_F64, N.ARITH_FAST, 1, 0
    L.number_of_nodes = 10
    L.distributions = L.neighbor_x = L.neighbor_y = L.neighbor_z = 0x1000
    L.omega = 1.5
    return L


def test_simulation_manager_rules():
    """BCKernelManagerTest.cpp: a BC with nodes but no kernel is an error; none without nodes is fine."""
    from virtualfluids_b200 import _native as N
    lib = N.lib()
    sim = C.c_void_p()
    assert lib.vfb_simulation_create(b"K15CompressibleNavierStokes", C.byref(sim)) == N.VFB_ERR_UNKNOWN_KERNEL
    N.check(lib.vfb_simulation_create(b"K17CompressibleNavierStokes", C.byref(sim)))
    try:
        N.check(lib.vfb_simulation_set_neighbor_tables(sim, 0))   # host checks only: no device tables
        assert lib.vfb_simulation_check(sim) == N.VFB_ERR_INVALID_ARGUMENT  # no level yet
        L = _fake_level(N)
        N.check(lib.vfb_simulation_set_level(sim, C.byref(L), C.c_void_p(0x2000), 5))
        N.check(lib.vfb_simulation_check(sim))
        bc = N.BC(0x3000, 0x4000, 0, 0, 0, 0)
        N.check(lib.vfb_simulation_set_velocity_bc(sim, C.byref(bc), N.VELOCITY_NOT_SPECIFIED))
        N.check(lib.vfb_simulation_check(sim))        # no nodes, no kernel: fine
        bc.number_of_bc_nodes = 4
        N.check(lib.vfb_simulation_set_velocity_bc(sim, C.byref(bc), N.VELOCITY_NOT_SPECIFIED))
        assert lib.vfb_simulation_check(sim) == N.VFB_ERR_BC_UNSET
        N.check(lib.vfb_simulation_set_velocity_bc(sim, C.byref(bc), N.VELOCITY_BOUNCE_BACK))
        N.check(lib.vfb_simulation_check(sim))
        nbc = N.BC(0x3000, 0x4000, 4, 0, 0, 0)
        N.check(lib.vfb_simulation_set_noslip_bc(sim, C.byref(nbc), N.NOSLIP_DELAY_BOUNCE_BACK))
        N.check(lib.vfb_simulation_check(sim))        # delayed bounce-back needs no kernel
        pbc = N.DirectionalBC(0x3000, 0x3100, 0x3200, 3, N.DIR_P00)
        N.check(lib.vfb_simulation_add_pressure_bc(sim, C.byref(pbc), N.PRESSURE_NOT_SPECIFIED))
        assert lib.vfb_simulation_check(sim) == N.VFB_ERR_BC_UNSET
    finally:
        lib.vfb_simulation_destroy(sim)


def test_multilevel_driver_rules():
    """Levels are added one at a time; vfb_level::level must be the level's index; more than one
    level needs the scaling factory (GridScalingKernelManager.cpp:45-62) and, where a pair of levels
    has interpolation cells, a function for them (checkScalingFunction); one storage for all."""
    from virtualfluids_b200 import _native as N
    lib = N.lib()
    sim = C.c_void_p()
    N.check(lib.vfb_simulation_create(b"K17CompressibleNavierStokes", C.byref(sim)))
    try:
        N.check(lib.vfb_simulation_set_neighbor_tables(sim, 0))
        L0, L1 = _fake_level(N), _fake_level(N)
        N.check(lib.vfb_simulation_set_level(sim, C.byref(L0), C.c_void_p(0x2000), 5))
        assert lib.vfb_simulation_use_level(sim, 2) == N.VFB_ERR_INVALID_ARGUMENT     # skips level 1
        assert lib.vfb_simulation_use_level(sim, -1) == N.VFB_ERR_INVALID_ARGUMENT
        N.check(lib.vfb_simulation_use_level(sim, 1))
        n = C.c_int32()
        N.check(lib.vfb_simulation_number_of_levels(sim, C.byref(n)))
        assert n.value == 2
        assert lib.vfb_simulation_check(sim) == N.VFB_ERR_INVALID_ARGUMENT           # level 1 not set
        assert lib.vfb_simulation_set_level(sim, C.byref(L1), C.c_void_p(0x2000), 5) == N.VFB_ERR_INVALID_ARGUMENT
        L1.level = 1
        N.check(lib.vfb_simulation_set_level(sim, C.byref(L1), C.c_void_p(0x2000), 5))
        assert lib.vfb_simulation_check(sim) == N.VFB_ERR_SCALING_UNSET
        assert "no scalingFactory" in N.lib().vfb_last_error().decode()
        cells = N.InterpolationCells(0x5000, 0x5100, 7)
        offs = N.InterpolationCellNeighbor(0x5200, 0x5300, 0x5400)
        assert lib.vfb_simulation_set_interpolation_cells(sim, 1, C.byref(cells), C.byref(offs), C.byref(cells),
                                                          C.byref(offs)) == N.VFB_ERR_INVALID_ARGUMENT  # finest level
        N.check(lib.vfb_simulation_set_interpolation_cells(sim, 0, C.byref(cells), C.byref(offs), C.byref(cells),
                                                           C.byref(offs)))
        N.check(lib.vfb_simulation_set_scaling_factory(sim, N.SCALE_NOT_SPECIFIED, 0))
        assert lib.vfb_simulation_check(sim) == N.VFB_ERR_SCALING_UNSET               # cells but no function
        assert lib.vfb_simulation_set_scaling_factory(sim, N.SCALE_COMPRESSIBLE, 1) == N.VFB_ERR_UNSUPPORTED
        N.check(lib.vfb_simulation_set_scaling_factory(sim, N.SCALE_COMPRESSIBLE, 0))
        N.check(lib.vfb_simulation_check(sim))
        L1.storage = N.STORAGE_F32
        N.check(lib.vfb_simulation_set_level(sim, C.byref(L1), C.c_void_p(0x2000), 5))
        assert lib.vfb_simulation_check(sim) == N.VFB_ERR_INVALID_ARGUMENT            # mixed storage
        ev = C.c_int32()
        N.check(lib.vfb_simulation_level_is_even_timestep(sim, 1, C.byref(ev)))
        assert ev.value == 1
        assert lib.vfb_simulation_level_is_even_timestep(sim, 2, C.byref(ev)) == N.VFB_ERR_INVALID_ARGUMENT
    finally:
        lib.vfb_simulation_destroy(sim)


def test_argument_validation_without_launching():
    from virtualfluids_b200 import _native as N
    lib = N.lib()
    L = _fake_level(N)
    L.omega = 2.5
    assert lib.vfb_k17_run_on_indices(C.byref(L), C.c_void_p(0x2000), 5, 0, None) == N.VFB_ERR_INVALID_ARGUMENT
    L.omega = 1.5
    L.storage = N.STORAGE_F16
    L.arith = N.ARITH_EXACT
    assert lib.vfb_k17_run_on_indices(C.byref(L), C.c_void_p(0x2000), 5, 0, None) == N.VFB_ERR_UNSUPPORTED
    L.arith = N.ARITH_FAST
    assert lib.vfb_k17_run_on_indices(C.byref(L), C.c_void_p(0x2000), 5, 9, None) == N.VFB_ERR_INVALID_ARGUMENT
    assert lib.vfb_k17_run_on_indices(C.byref(L), None, 5, 0, None) == N.VFB_ERR_INVALID_ARGUMENT
    # a write-macro template without output arrays
    assert lib.vfb_k17_run_on_indices(C.byref(L), C.c_void_p(0x2000), 5, 1, None) == N.VFB_ERR_INVALID_ARGUMENT
    pbc = N.DirectionalBC(0x3000, 0x3100, 0x3200, 3, 19)
    assert lib.vfb_pressure_non_equilibrium_compressible(C.byref(L), C.byref(pbc), None) == N.VFB_ERR_INVALID_ARGUMENT
    d = N.BoxDesc()
    d.nx = d.ny = d.nz = 8
    d.storage, d.omega = N.STORAGE_F64, 1.8
    h = C.c_void_p()
    assert lib.vfb_box_create(C.byref(d), C.byref(h)) == N.VFB_ERR_INVALID_ARGUMENT  # walls need a mask


def test_grid_scaling_factory_semantics():
    """GridScalingFactoryTest.cpp: NotSpecified gives no function; ScaleCompressible gives the
    compressible scaling of each direction; turbulent viscosity is not built here."""
    from virtualfluids_b200 import _native as N
    lib = N.lib()
    fn = C.c_void_p()
    N.check(lib.vfb_scaling_factory_fine_to_coarse(N.SCALE_NOT_SPECIFIED, 0, C.byref(fn)))
    assert fn.value is None
    N.check(lib.vfb_scaling_factory_coarse_to_fine(N.SCALE_NOT_SPECIFIED, 0, C.byref(fn)))
    assert fn.value is None
    N.check(lib.vfb_scaling_factory_fine_to_coarse(N.SCALE_COMPRESSIBLE, 0, C.byref(fn)))
    assert fn.value == C.cast(lib.vfb_scale_fine_to_coarse_compressible, C.c_void_p).value
    N.check(lib.vfb_scaling_factory_coarse_to_fine(N.SCALE_COMPRESSIBLE, 0, C.byref(fn)))
    assert fn.value == C.cast(lib.vfb_scale_coarse_to_fine_compressible, C.c_void_p).value
    assert lib.vfb_scaling_factory_coarse_to_fine(N.SCALE_COMPRESSIBLE, 1, C.byref(fn)) == N.VFB_ERR_UNSUPPORTED
    assert lib.vfb_scaling_factory_fine_to_coarse(7, 0, C.byref(fn)) == N.VFB_ERR_INVALID_ARGUMENT


def test_scaling_argument_validation_without_launching():
    from virtualfluids_b200 import _native as N
    lib = N.lib()
    coarse, fine = _fake_level(N), _fake_level(N)
    fine.distributions = 0x5000
    cells = N.InterpolationCells(0x6000, 0x6100, 4)
    off = N.InterpolationCellNeighbor(0x6200, 0x6300, 0x6400)
    for name in ("vfb_scale_coarse_to_fine_compressible", "vfb_scale_fine_to_coarse_compressible"):
        f = getattr(lib, name)
        assert f(C.byref(coarse), C.byref(fine), None, C.byref(off), None) == N.VFB_ERR_INVALID_ARGUMENT
        fine.storage = N.STORAGE_F32
        assert f(C.byref(coarse), C.byref(fine), C.byref(cells), C.byref(off), None) == N.VFB_ERR_INVALID_ARGUMENT
        fine.storage = N.STORAGE_F64
        fine.distributions = coarse.distributions
        assert f(C.byref(coarse), C.byref(fine), C.byref(cells), C.byref(off), None) == N.VFB_ERR_INVALID_ARGUMENT
        fine.distributions = 0x5000
        bad = N.InterpolationCellNeighbor(0x6200, 0, 0x6400)
        assert f(C.byref(coarse), C.byref(fine), C.byref(cells), C.byref(bad), None) == N.VFB_ERR_INVALID_ARGUMENT
        # no cells: nothing to launch, nothing to check
        empty = N.InterpolationCells(0, 0, 0)
        assert f(C.byref(coarse), C.byref(fine), C.byref(empty), C.byref(bad), None) == N.VFB_OK


def test_bounds_checked_build_loads_and_reports_itself():
    """libvfb_checked.so (built by build(checked=True)) exports the same ABI and says it is the
    checked build; the default build answers that it has no checks. No CUDA call is made."""
    from virtualfluids_b200 import _native as N
    from virtualfluids_b200 import build as vbuild
    if not vbuild.LIB_CHECKED.exists():
        pytest.skip("libvfb_checked.so not built here")
    checked = C.CDLL(str(vbuild.LIB_CHECKED))
    assert checked.vfb_bounds_checked() == 1
    assert N.lib().vfb_bounds_checked() == 0
    bad, n = C.c_uint64(7), C.c_uint64(7)
    assert N.lib().vfb_bounds_check_status(C.byref(bad), C.byref(n)) == N.VFB_ERR_UNSUPPORTED
    assert bad.value == 0 and n.value == 0
    missing = [name for name in _declared_symbols() if not hasattr(checked, name)]
    assert not missing, missing
