/*
 * vfb.h — C ABI of the B200-native VirtualFluids GPU time-step hot path.
 *
 * Plain C: pointers, sizes and status codes; no exceptions and no C++ or torch types cross
 * this boundary. Every entry point returns a vfb_status; vfb_last_error() gives a message for the
 * calling thread. CUDA launches are asynchronous on the given stream (NULL = legacy stream);
 * launch-configuration errors are reported at once, execution errors at the next synchronising
 * call (vfb_synchronize, a reduction, a copy to the host).
 *
 * Two layers:
 *  (1) Reference-layout entry points that take caller-owned device memory laid out as the
 *      reference's LBMSimulationParameter (src/gpu/core/Parameter/Parameter.h:66-330): one
 *      population array of 27*numberOfNodes, neighborX/Y/Z index lists, dummy node 0, BC node
 *      lists with SoA q27 arrays. Each replaces one reference launcher (cited at the
 *      declaration) and allocates nothing.
 *  (2) Library-owned objects: a step driver with the reference's kernel/BC/scaling factory
 *      semantics (vfb_simulation_*), and structured boxes (vfb_box_*) for full-box domains with
 *      arithmetic neighbours, runtime storage formats and a fused FP64 energy reduction.
 *
 * "real" arrays (q27, boundary velocities, rhoBC, macroscopic outputs) are double when the
 * level's storage is VFB_STORAGE_F64 and float for every other storage format, as the
 * reference's `real` is double or float (src/basics/DataTypes.h:39-43).
 */
#ifndef VFB_H
#define VFB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VFB_ABI_VERSION 1

typedef enum vfb_status {
    VFB_OK = 0,
    VFB_ERR_INVALID_ARGUMENT = 1,
    VFB_ERR_UNKNOWN_KERNEL = 2,   /* KernelFactoryImp::makeKernel throws (KernelFactoryImp.cpp:92-139) */
    VFB_ERR_BC_UNSET = 3,         /* BoundaryConditionKernelManager ctor throws (BoundaryConditionKernelManager.cpp:67-80) */
    VFB_ERR_SCALING_UNSET = 4,    /* GridScalingKernelManager ctor throws (GridScalingKernelManager.cpp:45-62) */
    VFB_ERR_CUDA = 5,
    VFB_ERR_OUT_OF_MEMORY = 6,
    VFB_ERR_UNSUPPORTED = 7,      /* a variant the reference has that this build does not implement */
    VFB_ERR_WATCHDOG = 8          /* non-finite populations or mass drift detected */
} vfb_status;

/* population storage (runtime choice; the reference fixes it at compile time) */
typedef enum vfb_storage {
    VFB_STORAGE_F64 = 0,   /* f - w in double, arithmetic in double */
    VFB_STORAGE_F32 = 1,   /* f - w in float, arithmetic in float */
    VFB_STORAGE_F16 = 2,   /* (f - w)/w in IEEE half, arithmetic in float */
    VFB_STORAGE_BF16 = 3,  /* (f - w)/w in bfloat16, arithmetic in float */
    VFB_STORAGE_E3M12 = 4  /* (f - w)/w in a 16-bit float of 1 sign, 3 exponent, 12 significand bits
                              (|values| < 2, subnormal steps of 2^-18, no infinity or NaN: out-of-range
                              values saturate), arithmetic in float; no counterpart in the reference */
} vfb_storage;

/* rounding mode of the arithmetic */
typedef enum vfb_arith {
    VFB_ARITH_FAST = 0,    /* products contracted into FMAs (the Python classes' default) */
    VFB_ARITH_EXACT = 1    /* every operation rounded separately, as the reference built without FMA
                              (the reference-side adapter's default): bit for bit the reference's
                              host arithmetic */
} vfb_arith;

/* CollisionTemplate (src/gpu/core/Calculation/Calculation.h:55-67) */
typedef enum vfb_collision_template {
    VFB_COLLISION_DEFAULT = 0,
    VFB_COLLISION_WRITE_MACRO_VARS = 1,
    VFB_COLLISION_APPLY_BODY_FORCE = 2,
    VFB_COLLISION_ALL_FEATURES = 3,
    VFB_COLLISION_SUBDOMAIN_BORDER = 4
} vfb_collision_template;

/* D3Q27 directions used as outlet normals (src/lbm/constants/D3Q27.h:42-48) */
enum { VFB_DIR_P00 = 1, VFB_DIR_M00 = 2, VFB_DIR_0P0 = 3, VFB_DIR_0M0 = 4, VFB_DIR_00P = 5, VFB_DIR_00M = 6 };

/* GEO node types (src/gpu/core/Calculation/Calculation.h:39-45) */
enum { VFB_GEO_SOLID = 15, VFB_GEO_VOID = 16, VFB_GEO_FLUID = 19 };

/* One refinement level: the fields of LBMSimulationParameter the hot path reads. Device pointers. */
typedef struct vfb_level {
    int32_t storage;                  /* vfb_storage */
    int32_t arith;                    /* vfb_arith */
    int32_t is_even_timestep;         /* isEvenTimestep */
    int32_t level;                    /* refinement level: forces are scaled by 2^-level */
    uint64_t number_of_nodes;         /* numberOfNodes, including the dummy node 0 */
    void *distributions;              /* distributions.f[0]: 27 * number_of_nodes elements */
    const uint32_t *neighbor_x;       /* neighborX: node at +1 in x (0 = dummy) */
    const uint32_t *neighbor_y;
    const uint32_t *neighbor_z;
    const uint32_t *type_of_grid_node;/* typeOfGridNode (init and macroscopic output) */
    double omega;                     /* omega = 1 / (3 nu + 1/2) */
    double forces[3];                 /* Parameter forcing (getForcesDev), by value */
    double quadric_limiters[3];       /* P, M, D (getQuadricLimitersDev), by value; reference default 0.01 */
    void *rho;                        /* real[number_of_nodes] macroscopic outputs (drho) */
    void *velocity_x;
    void *velocity_y;
    void *velocity_z;
    void *pressure;                   /* may be NULL */
    void *body_force_x;               /* forceX_SP etc., only for body-force collision templates */
    void *body_force_y;
    void *body_force_z;
    double outflow_pressure_correction_factor; /* outflowPressureCorrectionFactor (OutflowNonReflectivePressureCorrection) */
} vfb_level;

/* QforBoundaryConditions (src/gpu/core/Calculation/Calculation.h:105-117). Device pointers. */
typedef struct vfb_bc {
    const int32_t *k;                 /* BC node indices */
    const void *q27;                  /* real[27 * number_of_bc_nodes], q of direction d at [d * n + i]; q in [0,1] = link cut */
    uint32_t number_of_bc_nodes;
    const void *vx, *vy, *vz;         /* real[n] wall velocity (velocity BCs only) */
} vfb_bc;

/* QforDirectionalBoundaryCondition (Calculation.h:119-127). Device pointers. */
typedef struct vfb_directional_bc {
    const int32_t *k;                 /* BC node indices */
    const int32_t *k_neighbor;        /* kN: the neighbour one node inwards */
    const void *rho_bc;               /* real[n] prescribed drho */
    uint32_t number_of_bc_nodes;
    int32_t direction;                /* VFB_DIR_*: outward normal of the outlet */
} vfb_directional_bc;

/* ---- library ------------------------------------------------------------------------------ */
int vfb_abi_version(void);
const char *vfb_last_error(void);
const char *vfb_status_string(int status);
int vfb_synchronize(void *stream);
/* Bounds-checked build (libvfb_checked.so, compiled with -DVFB_BOUNDS_CHECK; no counterpart in the
   reference, which range-checks host containers only): every node index a kernel takes from the
   caller's arrays (fluid-node lists, neighborX/Y/Z, BC node lists, interpolation cells) is compared
   with its level's node count; an index out of range is replaced by the dummy node 0, so no access
   leaves the arrays, and the first one is recorded. vfb_bounds_checked() is 1 in that build.
   vfb_bounds_check_status synchronises the device, returns the first recorded index and the node
   count it exceeded (VFB_ERR_INVALID_ARGUMENT when there is one, VFB_OK when none) and clears the
   record; in the default build it returns VFB_ERR_UNSUPPORTED. */
int vfb_bounds_checked(void);
int vfb_bounds_check_status(uint64_t *bad_index, uint64_t *node_count);
/* D3Q27 tables as the kernels use them (for host-side checks) */
int vfb_lattice_tables(int32_t cx[27], int32_t cy[27], int32_t cz[27], int32_t inv[27], double w[27]);
/* the omega-only K17 relaxation rates as precomputed on the host:
   {OxyyPxzz, OxyyMxzz, Oxyz, factorA, factorB, 1/omega - 1/2} (K17CompressibleNavierStokes.h:251-273) */
int vfb_k17_rates(double omega, double rates[6]);

/* ---- kernel registry (Kernel/KernelTypes.h:35-46, KernelFactoryImp.cpp:92-139) -------------- */
enum { VFB_KERNEL_K17_COMPRESSIBLE_NAVIER_STOKES = 1 };
/* name -> id; unknown names give VFB_ERR_UNKNOWN_KERNEL ("KernelFactory does not know the KernelType.") */
int vfb_kernel_lookup(const char *name, int32_t *kernel_id);
/* number of registered kernels and their names */
int vfb_kernel_count(void);
const char *vfb_kernel_name(int index);

/* ---- (1) reference-layout entry points ----------------------------------------------------- */

/* K17CompressibleNavierStokes<None>::runOnIndices (Kernel/Compressible/NavierStokes/K17/
   K17CompressibleNavierStokes.cu:102-145) launching runCollision (Utilities/RunCollision.cuh:75):
   collision + esoteric-twist streaming of the listed fluid nodes, in place. */
int vfb_k17_run_on_indices(const vfb_level *level, const uint32_t *fluid_node_indices, uint32_t size,
                           int32_t collision_template, void *stream);
/* A prepared collision for a caller that keeps its own step loop (KernelImp::run / runOnIndices):
   one fluid-node list of a level, with its slot table (library-owned device memory, 32 bytes per
   entry) and, for an F64 or F32 list that is a whole periodic box numbered x fastest, box
   addressing; both are built from the list and neighborX/Y/Z as they are at creation. Same results
   as vfb_k17_run_on_indices. vfb_k17_plan_run takes the level of each call (parity, omega, forces,
   arrays); its node count, neighbour arrays and storage must be the plan's. Create the plan again
   after changing the list or the neighbour arrays. */
typedef struct vfb_k17_plan vfb_k17_plan;
int vfb_k17_plan_create(const vfb_level *level, const uint32_t *fluid_node_indices, uint32_t size,
                        vfb_k17_plan **plan);
int vfb_k17_plan_run(vfb_k17_plan *plan, const vfb_level *level, int32_t collision_template, void *stream);
/* 1 when the plan's default-template collision runs with box addressing */
int vfb_k17_plan_box_addressing(const vfb_k17_plan *plan, int32_t *box_addressing);
int vfb_k17_plan_destroy(vfb_k17_plan *plan);

/* NoSlipBounceBack (BoundaryConditions/NoSlip/NoSlip.cu:44) */
int vfb_noslip_bounce_back(const vfb_level *level, const vfb_bc *bc, void *stream);
/* NoSlipInterpolatedCompressible (NoSlip/NoSlip.cu:81) */
int vfb_noslip_interpolated_compressible(const vfb_level *level, const vfb_bc *bc, void *stream);
/* VelocityBounceBack (BoundaryConditions/Velocity/Velocity.cu:44) */
int vfb_velocity_bounce_back(const vfb_level *level, const vfb_bc *bc, void *stream);
/* VelocityInterpolatedCompressible (Velocity/Velocity.cu:87) */
int vfb_velocity_interpolated_compressible(const vfb_level *level, const vfb_bc *bc, void *stream);
/* SlipCompressible (BoundaryConditions/Slip/Slip.cu:42, SlipCompressible_Device): the interpolated
   velocity BC whose wall velocity is the node's own velocity, with the x (y, z) component zeroed when
   the node's P00 or M00 (0P0 or 0M0, 00P or 00M) link is cut; no wall velocities are read */
int vfb_slip_compressible(const vfb_level *level, const vfb_bc *bc, void *stream);
/* PressureNonEquilibriumCompressible (BoundaryConditions/Pressure/Pressure.cu:63) */
int vfb_pressure_non_equilibrium_compressible(const vfb_level *level, const vfb_directional_bc *bc, void *stream);
/* PressureNonEquilibriumIncompressible (Pressure/Pressure.cu:43) */
int vfb_pressure_non_equilibrium_incompressible(const vfb_level *level, const vfb_directional_bc *bc, void *stream);
/* OutflowNonReflecting (BoundaryConditions/Outflow/Outflow.cu:43) */
int vfb_outflow_non_reflecting(const vfb_level *level, const vfb_directional_bc *bc, void *stream);
/* OutflowNonReflectingPressureCorrection (Outflow/Outflow.cu:64), with the level's
   outflow_pressure_correction_factor */
int vfb_outflow_non_reflecting_pressure_correction(const vfb_level *level, const vfb_directional_bc *bc, void *stream);
/* NoSlipInterpolatedIncompressible (NoSlip/NoSlip.cu:62) */
int vfb_noslip_interpolated_incompressible(const vfb_level *level, const vfb_bc *bc, void *stream);
/* VelocityInterpolatedIncompressible (Velocity/Velocity.cu:65) */
int vfb_velocity_interpolated_incompressible(const vfb_level *level, const vfb_bc *bc, void *stream);
/* VelocityWithPressureInterpolatedCompressible (Velocity/Velocity.cu:109); the BC's q27 / velocity
   arrays as the velocity BC */
int vfb_velocity_with_pressure_interpolated_compressible(const vfb_level *level, const vfb_bc *bc, void *stream);

/* ICells and ICellNeigh (src/gpu/core/Calculation/Calculation.h:72-87): the interpolation cells
   between a coarse level and the fine level nested in it. Device pointers. */
typedef struct vfb_interpolation_cells {
    const uint32_t *fine_cell_indices;    /* fineCellIndices: MMM node of the cell on the fine level */
    const uint32_t *coarse_cell_indices;  /* coarseCellIndices: coarse-to-fine: MMM node of the coarse cell;
                                             fine-to-coarse: the coarse node at the cell centre */
    uint32_t number_of_cells;
} vfb_interpolation_cells;
typedef struct vfb_interpolation_cell_neighbor {
    const void *x, *y, *z;                /* real[number_of_cells]: offset of the expansion point (0 in the bulk) */
} vfb_interpolation_cell_neighbor;

/* scaleCoarseToFineCompressible<false> (GridScaling/Scaling.cu:106-138, kernel
   scaleCoarseToFineCompressible.cu:305-528): second-order moment interpolation of each coarse cell
   at the coarse level's parity (omega of the coarse level) into the pre-collision populations of
   its eight fine nodes at the even parity (omega of the fine level). Both levels share storage and
   arithmetic. Turbulent viscosity (the <true> instantiation) is not built. */
int vfb_scale_coarse_to_fine_compressible(const vfb_level *coarse, const vfb_level *fine,
                                          const vfb_interpolation_cells *cells,
                                          const vfb_interpolation_cell_neighbor *offsets, void *stream);
/* scaleFineToCoarseCompressible<false> (GridScaling/Scaling.cu:156-188, kernel
   scaleFineToCoarseCompressible.cu:76-124): each fine cell at the even parity into the coarse node
   at its centre, written at the coarse level's parity. */
int vfb_scale_fine_to_coarse_compressible(const vfb_level *coarse, const vfb_level *fine,
                                          const vfb_interpolation_cells *cells,
                                          const vfb_interpolation_cell_neighbor *offsets, void *stream);

/* DragLiftPostD27 (PostProcessor/DragLift.cu:558-567, kernel :50-301): per geometry BC node, minus
   the momentum carried by the post-collision populations that leave the node through its cut
   links (q in [0, 1]), in double; called after the collision and before the geometry BC
   (BoundaryConditionKernelManager.cpp:258-276). drag_x/y/z: double[number_of_bc_nodes], device. */
int vfb_drag_lift_post_27(const vfb_level *level, const vfb_bc *geometry_bc, double *drag_x, double *drag_y,
                          double *drag_z, void *stream);
/* DragLiftPreD27 (DragLift.cu:569-578, kernel :304-555): after the parity swap, minus the momentum of
   the populations each geometry node reads next, each weighted by the cut link of the opposite
   direction (BoundaryConditionKernelManager.cpp:148-172). */
int vfb_drag_lift_pre_27(const vfb_level *level, const vfb_bc *geometry_bc, double *drag_x, double *drag_y,
                         double *drag_z, void *stream);
/* calcDragLift (PostProcessor/DragLift.cpp:52-73): the force on the geometry, the FP64 sum over the
   nodes of pre - post, formed on the device in a fixed order and copied to force[3] on the host
   (the coefficient 2 F / (rho u^2 A) is left to the caller, whose area it needs). Device
   workspace of vfb_drag_lift_workspace_bytes(n) bytes. Synchronises the stream. */
size_t vfb_drag_lift_workspace_bytes(uint32_t n);
int vfb_drag_lift_force(const double *pre_x, const double *pre_y, const double *pre_z, const double *post_x,
                        const double *post_y, const double *post_z, uint32_t n, void *workspace, size_t workspace_bytes,
                        double force[3], void *stream);

/* InitNavierStokesCompressible::init (PreProcessor/PreProcessorStrategy/InitNavierStokesCompressible/
   InitNavierStokesCompressible.cu:45): equilibrium from level->rho/velocity_* for the level's
   current parity. PreProcessorImp::init (PreProcessorImp.cpp:50-58) calls it for the odd, then
   the even parity. */
int vfb_init_navier_stokes_compressible(const vfb_level *level, void *stream);
/* The same with Parameter::getUseInitNeq() (InitNavierStokesCompressible.cu:65-83,
   InitNavierStokesCompressibleNonEquilibrium_Device): the equilibrium plus (1 + drho) times a
   non-equilibrium part per direction pair, formed from central differences of the velocities at the
   six face neighbours and level->omega, for the level's current parity. neighbor_inverse is
   neighborInverse: per node, the node at -1 in x, y and z (device memory). Solid and void nodes get
   96 in their rest slot, as in the reference. */
int vfb_init_navier_stokes_compressible_non_equilibrium(const vfb_level *level, const uint32_t *neighbor_inverse,
                                                        void *stream);
/* calculateMacroscopicQuantitiesCompressible (PostProcessor/MacroscopicQuantities.cu:194) */
int vfb_calc_macroscopic_compressible(const vfb_level *level, void *stream);
/* FP64 sum over the listed nodes of (1 + drho) and 0.5 (1 + drho) |u|^2, into out[2] on the host.
   The per-block partial sums go to caller-provided device workspace of
   vfb_mass_energy_workspace_bytes(size) bytes. Synchronises the stream. */
size_t vfb_mass_energy_workspace_bytes(uint32_t size);
int vfb_mass_energy(const vfb_level *level, const uint32_t *node_indices, uint32_t size, void *workspace,
                    size_t workspace_bytes, double out[2], void *stream);

/* The same reduction for callers that cannot allocate device memory or hand the library any: no
   counterpart in the reference. The per-block partial sums live in a fixed array inside the
   library's device memory (about 1 MiB on every GPU that loads the library, held until the
   process exits), so the node count is limited to VFB_NO_ALLOC_MAX_NODES; larger sizes are
   rejected with VFB_ERR_INVALID_ARGUMENT; the level is checked as vfb_mass_energy checks it.
   Every call looks the array's device address up on the current device; the first call on a
   device also loads the library's device code there, so make it before any stream capture. All
   calls share the array, so calls that overlap on the GPU race; each call overwrites what it
   reads back. Synchronises the stream. */
#define VFB_NO_ALLOC_MAX_NODES (1u << 24)
int vfb_mass_energy_no_alloc(const vfb_level *level, const uint32_t *node_indices, uint32_t size, double out[2],
                             void *stream);

/* ---- boundary-condition factory (BoundaryConditions/BoundaryConditionFactory.h:50-130) ------ */
typedef int (*vfb_bc_fn)(const vfb_level *level, const vfb_bc *bc, void *stream);
typedef int (*vfb_directional_bc_fn)(const vfb_level *level, const vfb_directional_bc *bc, void *stream);
/* enum values of BoundaryConditionFactory::VelocityBC / NoSlipBC / PressureBC */
enum { VFB_VELOCITY_BOUNCE_BACK = 0, VFB_VELOCITY_INTERPOLATED_INCOMPRESSIBLE = 1, VFB_VELOCITY_INTERPOLATED_COMPRESSIBLE = 2,
       VFB_VELOCITY_WITH_PRESSURE_INTERPOLATED_COMPRESSIBLE = 3, VFB_VELOCITY_NOT_SPECIFIED = 4 };
enum { VFB_NOSLIP_DELAY_BOUNCE_BACK = 0, VFB_NOSLIP_BOUNCE_BACK = 1, VFB_NOSLIP_INTERPOLATED_INCOMPRESSIBLE = 2,
       VFB_NOSLIP_INTERPOLATED_COMPRESSIBLE = 3 };
/* SlipBC (BoundaryConditionFactory.h:87-94) */
enum { VFB_SLIP_COMPRESSIBLE = 0, VFB_SLIP_TURBULENT_VISCOSITY_COMPRESSIBLE = 1, VFB_SLIP_NOT_SPECIFIED = 2 };
enum { VFB_PRESSURE_NON_EQUILIBRIUM_INCOMPRESSIBLE = 0, VFB_PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE = 1,
       VFB_PRESSURE_OUTFLOW_NON_REFLECTIVE = 2, VFB_PRESSURE_OUTFLOW_NON_REFLECTIVE_PRESSURE_CORRECTION = 3,
       VFB_PRESSURE_NOT_SPECIFIED = 4 };
/* The function for an enum value; every variant of the three enums has one. *fn = NULL with
   VFB_OK means "no kernel" (NoSlipDelayBounceBack, whose bounce-back happens through the dummy
   node; NotSpecified). A value outside the enum gives VFB_ERR_INVALID_ARGUMENT. */
int vfb_bc_factory_velocity(int32_t variant, vfb_bc_fn *fn);
int vfb_bc_factory_noslip(int32_t variant, vfb_bc_fn *fn);
/* SlipCompressible -> vfb_slip_compressible; NotSpecified -> NULL; SlipTurbulentViscosityCompressible
   (it needs a turbulence model, outside this path) -> VFB_ERR_UNSUPPORTED */
int vfb_bc_factory_slip(int32_t variant, vfb_bc_fn *fn);
int vfb_bc_factory_pressure(int32_t variant, vfb_directional_bc_fn *fn);

/* ---- grid-scaling factory (GridScaling/GridScalingFactory.h:47-66) ----------------------- */
typedef int (*vfb_scaling_fn)(const vfb_level *coarse, const vfb_level *fine, const vfb_interpolation_cells *cells,
                              const vfb_interpolation_cell_neighbor *offsets, void *stream);
/* enum values of GridScalingFactory::GridScaling */
enum { VFB_SCALE_COMPRESSIBLE = 0, VFB_SCALE_NOT_SPECIFIED = 1 };
/* getGridScalingFC / getGridScalingCF. NotSpecified gives *fn = NULL with VFB_OK; a turbulent
   viscosity request gives VFB_ERR_UNSUPPORTED. */
int vfb_scaling_factory_fine_to_coarse(int32_t variant, int32_t has_turbulent_viscosity, vfb_scaling_fn *fn);
int vfb_scaling_factory_coarse_to_fine(int32_t variant, int32_t has_turbulent_viscosity, vfb_scaling_fn *fn);

/* ---- (2a) step driver: UpdateGrid27::updateGrid (Calculation/UpdateGrid27.cpp:54-95) over one or more
   refinement levels ----------------------------------------------------------------------------- */
typedef struct vfb_simulation vfb_simulation;
#define VFB_MAX_LEVELS 16
/* kernel_name as Parameter::configureMainKernel; VFB_ERR_UNKNOWN_KERNEL for unknown names */
int vfb_simulation_create(const char *kernel_name, vfb_simulation **out);
int vfb_simulation_destroy(vfb_simulation *sim);
/* the level that vfb_simulation_set_level and the BC, geometry and drag/lift setters below
   configure: 0 (the coarsest, the default) up to the number of levels, which adds a finer level
   (Parameter::getParD(level)) */
int vfb_simulation_use_level(vfb_simulation *sim, int32_t level);
int vfb_simulation_number_of_levels(const vfb_simulation *sim, int32_t *number_of_levels);
/* Neighbour slot tables: vfb_simulation_set_level builds, in library-owned device memory (32 bytes
   per fluid node), each fluid node and its seven +1 neighbours, and the driver's collision reads
   them instead of walking the neighborX/Y/Z chain, with the same results. mode 1 (default): one
   coalesced load per slot; 2: the tables staged in shared memory by bulk asynchronous copies two
   tiles ahead (persistent warps); 0: no tables (the chain). Set the level again after changing its
   neighbour arrays or fluid-node list.
   With modes 1 and 2, an F64 or F32 level whose fluid list is a whole periodic box numbered x
   fastest from its first node (as the reference's grid builder numbers a box without solids;
   checked by vfb_simulation_set_level against every neighbour entry) is collided by the structured
   box kernel over the same arrays: arithmetic neighbours instead of index loads, the same results.
   The 16-bit forms keep the list kernel (their stochastic rounding hashes the slot offsets). */
int vfb_simulation_set_neighbor_tables(vfb_simulation *sim, int32_t mode);
/* 1 when the level's collision runs with that box addressing, else 0 */
int vfb_simulation_level_box_addressing(const vfb_simulation *sim, int32_t level, int32_t *box_addressing);
/* synchronises the stream and reads the status word the staged collision sets when a bounded wait
   for its copies gave up (0 = fine); returns VFB_ERR_CUDA when it is nonzero */
int vfb_simulation_status(vfb_simulation *sim, int32_t *device_status, void *stream);
/* the selected level's description, copied; device memory stays caller-owned; level->level must be
   the selected level (forces are scaled by 2^-level) */
int vfb_simulation_set_level(vfb_simulation *sim, const vfb_level *level, const uint32_t *fluid_node_indices,
                             uint32_t number_of_fluid_nodes);
/* GridScalingFactory::setScalingFactory (VFB_SCALE_*); with more than one level a run without it is
   VFB_ERR_SCALING_UNSET ("There is more than one level, but no scalingFactory was provided.") */
int vfb_simulation_set_scaling_factory(vfb_simulation *sim, int32_t variant, int32_t has_turbulent_viscosity);
/* the interpolation cells between coarse_level and coarse_level + 1 (both added before), the coarse level's
   fineToCoarse / neighborFineToCoarse and coarseToFine / neighborCoarseToFine (descriptors copied,
   device arrays caller-owned); unset pairs have no cells */
int vfb_simulation_set_interpolation_cells(vfb_simulation *sim, int32_t coarse_level,
                                           const vfb_interpolation_cells *fine_to_coarse,
                                           const vfb_interpolation_cell_neighbor *fine_to_coarse_offsets,
                                           const vfb_interpolation_cells *coarse_to_fine,
                                           const vfb_interpolation_cell_neighbor *coarse_to_fine_offsets);
/* BC lists of the selected level (copied descriptors) and factory choices */
int vfb_simulation_set_velocity_bc(vfb_simulation *sim, const vfb_bc *bc, int32_t variant);
int vfb_simulation_set_noslip_bc(vfb_simulation *sim, const vfb_bc *bc, int32_t variant);
/* the slip BC list (slipBC, a SlipBC value); it runs after the no-slip BC and before the geometry BC,
   as runSlipBCKernelPost (UpdateGrid27.cpp:240) */
int vfb_simulation_set_slip_bc(vfb_simulation *sim, const vfb_bc *bc, int32_t variant);
int vfb_simulation_add_pressure_bc(vfb_simulation *sim, const vfb_directional_bc *bc, int32_t variant);
/* the geometry BC list (BoundaryConditionFactory::setGeometryBoundaryCondition with a NoSlipBC
   value); it runs after the no-slip BC, as runGeoBCKernelPost (UpdateGrid27.cpp:247-248) */
int vfb_simulation_set_geometry_bc(vfb_simulation *sim, const vfb_bc *bc, int32_t variant);
/* the same with the variant's family, as setGeometryBoundaryCondition takes a VelocityBC, NoSlipBC or
   SlipBC value (BoundaryConditionFactory.cpp:206-216); a velocity family needs the list's velocities */
enum { VFB_GEOMETRY_VELOCITY = 0, VFB_GEOMETRY_NOSLIP = 1, VFB_GEOMETRY_SLIP = 2 };
int vfb_simulation_set_geometry_bc_of(vfb_simulation *sim, const vfb_bc *bc, int32_t family, int32_t variant);
/* drag and lift on the geometry nodes every step (Parameter::setCalcDragLift): DragLiftPost27 before
   the geometry BC, DragLiftPre27 and the FP64 sum after the parity swap, the force of step t into
   force_history[3 * (t % history_steps)] (device, no host synchronisation). Caller-owned device
   workspace of vfb_simulation_drag_lift_workspace_bytes(geometry nodes) bytes; NULL disables. */
size_t vfb_simulation_drag_lift_workspace_bytes(uint32_t number_of_geometry_nodes);
int vfb_simulation_set_drag_lift(vfb_simulation *sim, void *workspace, size_t workspace_bytes, double *force_history,
                                 uint32_t history_steps);
/* checks the BoundaryConditionKernelManager rules (a BC with nodes but no kernel is VFB_ERR_BC_UNSET)
   and the GridScalingKernelManager ones (VFB_ERR_SCALING_UNSET); every level set, one storage and
   arithmetic for all */
int vfb_simulation_check(const vfb_simulation *sim);
/* run steps of the coarsest level. A level's step: collision, velocity, no-slip, slip then geometry BCs,
   parity toggle, drag/lift, pressure BCs. A level with a finer one lets that one take two steps
   first and after its own step interpolates fine to coarse, then coarse to fine. */
int vfb_simulation_run(vfb_simulation *sim, uint32_t steps, void *stream);

/* Phase timers (Output/TimeStepTimer.h: the reference's collision, post- and pre-collision BC
   timers, here with the two interpolation directions). Every phase of a run is an NVTX range of
   the phase's name (visible to ncu --nvtx and other NVTX tools). With timing on, each phase is also
   bracketed by CUDA events on the run's stream, and vfb_simulation_run synchronises that stream
   once at its end to add the device times up; phase_times returns the sums in milliseconds, over
   all levels, and the coarse steps they cover (reset != 0 clears them). Off by default. */
enum {
    VFB_PHASE_COLLISION = 0,
    VFB_PHASE_POST_COLLISION_BC = 1,   /* velocity, no-slip, slip, geometry BCs and the drag's post part */
    VFB_PHASE_PRE_COLLISION_BC = 2,    /* the drag's pre part and sum, pressure BCs */
    VFB_PHASE_SCALING_FC = 3,
    VFB_PHASE_SCALING_CF = 4,
    VFB_PHASES = 5
};
int vfb_simulation_set_timing(vfb_simulation *sim, int32_t on);
/* The step loop as a CUDA graph (the step loop of the reference launches every kernel of every step
   from the host, UpdateGrid27.cpp:54-95): with steps > 0 (even, up to 1024), vfb_simulation_run on
   a non-NULL stream runs its first step directly after any configuration change (so that buffers
   made on first use exist), then captures `steps` coarse steps once and replays the graph while
   enough steps remain, the rest directly. Every setter drops the graph; a run whose level
   parities differ from those at capture captures again. Not used on the legacy (NULL) stream, with
   timing on, or while a drag/lift history is kept (its per-step slot is chosen on the host).
   Results are those of the direct loop, bit for bit. 0 (the default) turns it off.
   The boundary-condition and scaling functions set on the simulation run once per captured step,
   during the capture only: what they enqueue on the stream is replayed, but their host code is not
   run again. Functions that change host-side state from step to step, or that synchronise the
   stream, need the graph off. The library's own functions only enqueue work. */
int vfb_simulation_set_graph(vfb_simulation *sim, int32_t steps);
int vfb_simulation_phase_times(vfb_simulation *sim, double *ms, uint64_t *steps, int32_t reset);
/* parity of the coarsest level / of a given level */
int vfb_simulation_is_even_timestep(const vfb_simulation *sim, int32_t *is_even);
int vfb_simulation_level_is_even_timestep(const vfb_simulation *sim, int32_t level, int32_t *is_even);

/* ---- (2b) structured boxes --------------------------------------------------------------- */
/* A full box of nx*ny*nz nodes, node k = x + nx (y + ny z), neighbours by index arithmetic.
   Non-periodic axes need a mask whose border nodes are 0 (not collided). */
typedef struct vfb_box_desc {
    int32_t nx, ny, nz;
    int32_t periodic_x, periodic_y, periodic_z;
    int32_t storage;                  /* vfb_storage */
    int32_t arith;                    /* vfb_arith */
    double omega;
    double forces[3];                 /* acceleration, applied as forces * 1/2 */
    double quadric_limiters[3];
    const uint8_t *mask;              /* optional host mask, nonzero = fluid; NULL = every node */
} vfb_box_desc;
typedef struct vfb_box vfb_box;
int vfb_box_create(const vfb_box_desc *desc, vfb_box **out);
int vfb_box_destroy(vfb_box *box);
/* bytes the box holds on the device */
int vfb_box_device_bytes(const vfb_box *box, uint64_t *bytes);
/* equilibrium initialisation from drho, ux, uy, uz (real[nx*ny*nz]); host memory when from_host,
   else device memory. Leaves the box at an even step. */
int vfb_box_init(vfb_box *box, const void *rho, const void *ux, const void *uy, const void *uz, int32_t from_host,
                 void *stream);
/* advance `steps` time steps. energy (optional): FP64 {sum(1+drho), sum(0.5 (1+drho)|u|^2)} per
   step, 2*steps doubles, host (pinned for asynchrony) when energy_on_host, else device. */
int vfb_box_step(vfb_box *box, uint32_t steps, double *energy, int32_t energy_on_host, void *stream);
/* macroscopic drho, ux, uy, uz (real[nx*ny*nz]) of the current state, to host or device memory */
int vfb_box_fields(vfb_box *box, void *rho, void *ux, void *uy, void *uz, int32_t to_host, void *stream);
/* synchronises the stream and reads the status word the box's kernels set on a failed internal wait
   (0 = fine); returns VFB_ERR_CUDA when it is nonzero */
int vfb_box_status(vfb_box *box, int32_t *device_status, void *stream);
/* collision kernel: 0 = choose (direct loads, the fastest measured on B200 for every storage),
   1 = direct loads, 2 = TMA-staged warp tiles (nx % 32 == 0),
   3 = per-thread asynchronous copies (F64 and F32 storage),
   4 = two nodes per thread in packed FP32x2 arithmetic (F32, F16, BF16 storage, FMA arithmetic),
   5 = persistent blocks with the next node's loads in flight while the current node is collided */
int vfb_box_set_kernel_variant(vfb_box *box, int32_t variant);
/* Boundary conditions on a box, run by vfb_box_step in the order of vfb_simulation_run: velocity,
   no-slip, slip, geometry (with the drag's post part before it), parity toggle, the drag's pre part
   and sum, pressure. Node indices are box indices k = x + nx (y + ny z) of fluid (mask nonzero) nodes;
   q27[d * n + i], velocities and rho are host arrays of the box's real type, copied into the box.
   variant: the VelocityBC / NoSlipBC / SlipBC / PressureBC enum values (the geometry list takes a
   NoSlipBC value). A new call replaces the list. */
enum { VFB_BOX_BC_VELOCITY = 0, VFB_BOX_BC_NOSLIP = 1, VFB_BOX_BC_GEOMETRY = 2, VFB_BOX_BC_SLIP = 3 };
int vfb_box_set_bc(vfb_box *box, int32_t kind, int32_t variant, const int32_t *k, const void *q27, uint32_t n,
                   const void *ux, const void *uy, const void *uz);
int vfb_box_add_pressure_bc(vfb_box *box, int32_t variant, const int32_t *k, const int32_t *k_neighbor, const void *rho,
                            uint32_t n, int32_t direction);
/* outflowPressureCorrectionFactor of the box's OutflowNonReflectivePressureCorrection lists */
int vfb_box_set_outflow_pressure_correction(vfb_box *box, double factor);
/* a seeded perturbation of the velocity BC every step: u_i(t) = u_i (1 + amplitude (2 U - 1)), U
   uniform in [0, 1) from the counter-based Philox-4x32-10 generator keyed by seed and counted by
   (BC node, step) */
int vfb_box_set_velocity_perturbation(vfb_box *box, uint64_t seed, double amplitude);
/* FP64 drag/lift on the geometry list every step (DragLiftPost27 / DragLiftPre27 / calcDragLift):
   the force of step t (counted from this call) into force_history[3 * (t % history_steps)], device */
int vfb_box_set_drag_lift(vfb_box *box, double *force_history, uint32_t history_steps);
/* number of kernels vfb_box_step has launched for this box so far (collision and reductions) */
int vfb_box_kernel_launches(const vfb_box *box, uint64_t *count);
/* launch shape of the per-thread asynchronous-copy kernel: resident blocks per SM (0 = 3) and the
   shared-memory configuration in KB each block pads its staging to a share of (0 = no padding,
   only a carve-out hint; else 64, 100, 132, 164, 196 or 228). Results do not depend on it. */
int vfb_box_set_launch_shape(vfb_box *box, int32_t blocks_per_sm, int32_t smem_kb);
/* raw access to the population planes for checks: pointer, plane pitch (elements), parity */
int vfb_box_populations(const vfb_box *box, void **dist, uint64_t *pitch, int32_t *is_even);
/* A time step in parts, for drivers that overlap work with the collision (no counterpart in the
   reference, whose CollisionAndExchange_streams splits the step by node lists instead,
   Calculation/CollisisionStrategy.cpp:100-135): vfb_box_collide_planes collides the box's planes
   z in [z_begin, z_end) at its current parity (direct-load kernel, the box's mask respected; no BC
   lists, no energy), on `stream`; vfb_box_toggle_parity ends the step. A step is the planes in any
   order and any split, then one toggle: every slot is read and written by one node per step. */
int vfb_box_collide_planes(vfb_box *box, int32_t z_begin, int32_t z_end, void *stream);
int vfb_box_toggle_parity(vfb_box *box);
/* The border plane z (0 <= z < nz - 1) of a box that is one slab of a domain cut along z, with the
   halo exchange fused into its stores (the counterpart of the reference's border collision plus
   ExchangeData27's collect / send / scatter, Communication/ExchangeData27.cpp:52-226): the slots the
   plane writes in plane z + 1 for directions with a negative z component at this parity are stored
   into plane 0 of `up` (the population array of the slab above), and the slots it writes in its own
   plane for directions with a positive z component into the last plane of `down` (the slab below's
   ghost plane); a null `up` or `down` keeps those stores local. `up` and `down` are population
   arrays of boxes of the same extents and storage (this process's, or another GPU's opened with
   vfb_ipc_open: the stores then cross NVLink as peer writes). No node of the receiving slab touches
   those slots in the same step; the caller puts a barrier between steps (after every rank's border
   planes, before any rank's next step). */
int vfb_box_collide_border(vfb_box *box, int32_t z, void *up, void *down, void *stream);
/* CUDA IPC of population arrays between the processes of one node: the handle
   (VFB_IPC_HANDLE_BYTES bytes) of a box's population array, and its mapping in another process
   (peer access enabled) and the mapping's release. */
#define VFB_IPC_HANDLE_BYTES 64
int vfb_box_ipc_handle(const vfb_box *box, void *handle);
int vfb_ipc_open(const void *handle, void **ptr);
int vfb_ipc_close(void *ptr);
/* the 27 population planes without their padding (plane d at d * nx*ny*nz, the storage type, as
   stored) and the parity, out of or into the box: restart files (RestartObject::serialize /
   deserialize). Host memory when to_host / from_host (the call then synchronises the stream). */
int vfb_box_read_populations(vfb_box *box, void *out, int32_t to_host, int32_t *is_even, void *stream);
int vfb_box_write_populations(vfb_box *box, const void *src, int32_t from_host, int32_t is_even, void *stream);

/* ---- (2c) domain pools: batches of independent boxes in one launch per step ---------------
   No counterpart in the reference (one level of one domain per Simulation there). A pool owns one
   device arena sized at creation; domains of uneven sizes are carved from it and released again,
   so a serving loop can admit solves against the HBM budget. Every step advances all active
   domains with one kernel launch over a work list of node blocks (domain, first node): one block
   per item, or a persistent grid that walks the list (vfb_pool_set_launch);
   each domain computes exactly what a vfb_box of the same description computes. */
typedef struct vfb_pool_desc {
    int32_t storage;                  /* vfb_storage */
    int32_t arith;                    /* vfb_arith */
    uint64_t arena_bytes;             /* device bytes for populations, masks and BC lists */
    uint32_t max_domains;
} vfb_pool_desc;
typedef struct vfb_domain_desc {
    int32_t nx, ny, nz;
    int32_t periodic_x, periodic_y, periodic_z;  /* on a non-periodic axis the first and last layers
                                                    are solid walls (NoSlipDelayBounceBack) */
    double omega;
    double forces[3];                 /* acceleration, applied as forces * 1/2 */
    double quadric_limiters[3];
} vfb_domain_desc;
typedef struct vfb_pool vfb_pool;
int vfb_pool_create(const vfb_pool_desc *desc, vfb_pool **out);
int vfb_pool_destroy(vfb_pool *pool);
/* device bytes one domain of this description takes in the arena (admission checks) */
int vfb_pool_domain_bytes(const vfb_pool *pool, const vfb_domain_desc *desc, int32_t has_mask, uint64_t *bytes);
/* carve a domain from the arena; mask (optional, host, nx*ny*nz bytes, nonzero = fluid) adds solid
   nodes inside. VFB_ERR_OUT_OF_MEMORY when the arena has no room: nothing is changed then. The
   domain takes part in steps once it is initialised. */
int vfb_pool_add_domain(vfb_pool *pool, const vfb_domain_desc *desc, const uint8_t *mask, uint32_t *id);
/* Boundary-condition lists of a pool domain, host arrays copied into the arena with the domain (they
   count against the budget and stay resident). Node indices are box indices k = x + nx (y + ny z) of
   fluid nodes. Every step runs them for all domains at once: the no-slip list after the collision
   (NoSlipInterpolatedCompressible, NoSlipInterpolatedCompressible.cu:44-381), the pressure list after
   the parity swap (PressureNonEquilibriumCompressible, PressureNonEquilibriumCompressible.cu:45-314,
   one outward normal per node, so inlet and outlet share a list). Other variants give
   VFB_ERR_UNSUPPORTED. A domain computes what a vfb_box with the same lists computes. Where a
   link joins two no-slip nodes and is cut from both ends (curved geometry), the values each reads
   and the other overwrites are saved before the writes (a per-node direction mask built here), so
   the result does not depend on thread order. */
typedef struct vfb_domain_bcs {
    int32_t noslip_variant;           /* VFB_NOSLIP_INTERPOLATED_COMPRESSIBLE */
    const int32_t *noslip_k;
    const double *noslip_q27;         /* q of direction d of node i at [d * n + i]; q in [0, 1] = cut link */
    uint32_t number_of_noslip_nodes;
    int32_t pressure_variant;         /* VFB_PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE */
    const int32_t *pressure_k;
    const int32_t *pressure_k_neighbor; /* the node one step inwards */
    const double *pressure_rho;       /* prescribed drho */
    const int32_t *pressure_direction;  /* VFB_DIR_*: outward normal */
    uint32_t number_of_pressure_nodes;
} vfb_domain_bcs;
int vfb_pool_add_domain_with_bcs(vfb_pool *pool, const vfb_domain_desc *desc, const uint8_t *mask,
                                 const vfb_domain_bcs *bcs, uint32_t *id);
/* device bytes of a domain with these BC lists (NULL: none) */
int vfb_pool_domain_bytes_with_bcs(const vfb_pool *pool, const vfb_domain_desc *desc, int32_t has_mask,
                                   const vfb_domain_bcs *bcs, uint64_t *bytes);
/* the domain stops taking part in steps; its arena range and id become reusable once the pool's
   stream has drained (the next vfb_pool_step that changes the work list, or vfb_pool_synchronize).
   All calls on one pool must use one stream. */
int vfb_pool_remove_domain(vfb_pool *pool, uint32_t id);
/* waits for the pool's stream and makes the ranges of removed domains reusable */
int vfb_pool_synchronize(vfb_pool *pool, void *stream);
/* equilibrium initialisation of both parities from drho, ux, uy, uz (real[nx*ny*nz], host when
   from_host, else device); activates the domain. Host fields pass through a staging buffer the
   pool keeps outside the arena (grown when a larger domain than before is staged). */
int vfb_pool_init_domain(vfb_pool *pool, uint32_t id, const void *rho, const void *ux, const void *uy, const void *uz,
                         int32_t from_host, void *stream);
/* advance every active domain by `steps` time steps (one collision launch per step; with the
   graph option the launches of 16 steps are replayed from one captured CUDA graph) */
int vfb_pool_step(vfb_pool *pool, uint32_t steps, void *stream);
/* drho, ux, uy, uz (real[nx*ny*nz]) of one domain, to host or device memory */
int vfb_pool_domain_fields(vfb_pool *pool, uint32_t id, void *rho, void *ux, void *uy, void *uz, int32_t to_host,
                           void *stream);
/* launch shape: threads per block (64, 128 or 256), nodes per thread per work item (1..32), resident
   blocks per SM of the persistent launch (0 = as many as fit; -1 = no persistent loop: one block per
   work item, the grid following the work list, so a change of the list's length captures the step
   graph again), CUDA-graph replay (0/1); a new pool starts at 128, 8, -1, 1 */
int vfb_pool_set_launch(vfb_pool *pool, int32_t threads_per_block, int32_t nodes_per_thread, int32_t blocks_per_sm,
                        int32_t use_graph);
int vfb_pool_get_launch(const vfb_pool *pool, int32_t out4[4]);
/* the autotuner: times trial_steps steps of the current domains for each launch shape of a fixed
   candidate set and keeps the fastest (results do not depend on the shape). It advances the active
   domains by the steps it runs: call it before initialising them, or accept the extra steps. */
int vfb_pool_autotune(vfb_pool *pool, uint32_t trial_steps, void *stream, double *best_ms_per_step);
/* active domains, their nodes, and arena bytes in use / free */
int vfb_pool_stats(const vfb_pool *pool, uint32_t *active_domains, uint64_t *active_nodes, uint64_t *used_bytes,
                   uint64_t *free_bytes);
/* kernels the pool has launched (graph replays count their kernels) */
int vfb_pool_kernel_launches(const vfb_pool *pool, uint64_t *count);
/* FP64 mass sum(1 + drho) over the fluid nodes of every active domain, at the state the next step
   reads: mass[id] for id < max_domains (0 for inactive ids), host memory; synchronises the stream.
   Per domain the sum runs in a fixed order. */
int vfb_pool_domain_mass(vfb_pool *pool, double *mass, void *stream);
/* The watchdog: the domain masses as above; a domain fails when its mass is not finite (a NaN or
   infinite population anywhere in it) or has drifted by more than max_relative_drift from its
   mass at the first check after its initialisation. Up to `capacity` failing ids go to `failed`,
   their number to *n_failed; VFB_ERR_WATCHDOG when any failed. Nothing is removed: the caller
   decides (a serving loop fails the request, not the process). */
int vfb_pool_watchdog(vfb_pool *pool, double max_relative_drift, uint32_t *failed, uint32_t capacity,
                      uint32_t *n_failed, void *stream);

#ifdef __cplusplus
}
#endif
#endif
