/*
 * ORACLE — test infrastructure, not product code.
 *
 * A plain-C CPU restatement of the VirtualFluids GPU time-step hot path (D3Q27 K17 cumulant
 * collision with in-place esoteric-twist streaming, the no-slip / velocity / pressure boundary
 * kernels, equilibrium initialisation, macroscopic output, the FP64 reductions and the
 * interpolation between refinement levels). It exists
 * only so tests, the smoke check and the benchmark's CPU-baseline leg can check the CUDA
 * library against the reference algorithm. Nothing in the shipped library links or calls it.
 *
 * Data layout is the reference GPU layout (src/gpu/core/Utilities/KernelUtilities.h:66-132,
 * src/gpu/core/Cuda/CudaMemoryManager.cpp:146-168): populations are one array of 27*n reals,
 * direction-major (f[dir*n + k]); n counts the dummy node 0; neighborX/Y/Z[k] give the node at
 * +1 in x/y/z (src/gpu/GridGenerator/grid/GridImp.cpp:1012-1080).
 */
#ifndef VFB_ORACLE_H
#define VFB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* D3Q27 direction numbering of src/lbm/constants/D3Q27.h:42-72 */
enum {
    D_000 = 0, D_P00, D_M00, D_0P0, D_0M0, D_00P, D_00M,
    D_PP0, D_MM0, D_PM0, D_MP0, D_P0P, D_M0M, D_P0M, D_M0P,
    D_0PP, D_0MM, D_0PM, D_0MP,
    D_PPP, D_MPP, D_PMP, D_MMP, D_PPM, D_MPM, D_PMM, D_MMM
};

extern const int ORC_CX[27], ORC_CY[27], ORC_CZ[27], ORC_INV[27];
extern const double ORC_W[27];

/* per-node K17 (src/lbm/collision/K17CompressibleNavierStokes.h:88) */
void orc_k17_f64(double *f, double omega, const double *lim, double fx, double fy, double fz, double *macro);
void orc_k17_f32(float *f, float omega, const float *lim, float fx, float fy, float fz, float *macro);
void orc_k17_rates_f64(double omega, double rates[6]);
void orc_k17_rates_f32(float omega, float rates[6]);
double orc_density_f64(const double *f);
void orc_macro_compressible_f64(const double *f, double *drho, double *one_over_rho, double *vx, double *vy, double *vz);

/* chimera transforms, exposed for the reference's known-answer tests */
void orc_chimera_f64(int which, double *abc, double v, double v2, double kinv, double k);

/* one refinement level in the reference layout */
typedef struct {
    uint64_t n;             /* numberOfNodes, including the dummy node 0 */
    double *f;              /* distributions.f[0], 27*n */
    const uint32_t *nbx;    /* neighborX */
    const uint32_t *nby;    /* neighborY */
    const uint32_t *nbz;    /* neighborZ */
} orc_level;

/* esoteric-twist addressing (KernelUtilities.h:66-132, 221-378) */
void orc_pointer_map(int is_even, int map[27]);
uint32_t orc_read_index(const orc_level *L, uint32_t k, int dir);
void orc_read_pre(const orc_level *L, uint32_t k, int is_even, double out[27]);
void orc_write_post(orc_level *L, uint32_t k, int is_even, const double in[27]);

/* RunCollision.cuh:75-143 with the K17 functor; force = forces*0.5*2^-level; macros optional */
void orc_collision(orc_level *L, const uint32_t *idx, uint32_t n_idx, int is_even, double omega,
                   const double lim[3], const double forces[3], int level,
                   double *rho, double *vx, double *vy, double *vz, int n_threads);
/* the same with the features of a CollisionTemplate (K17CompressibleNavierStokes.cu:114-139):
   body_force reads (forces + bodyForce[k]) * 0.5 * 2^-level and resets bodyForce[k] to zero
   (RunCollision.cuh:88-98); write_macro stores drho and u at k (:133-138) */
void orc_collision_template(orc_level *L, const uint32_t *idx, uint32_t n_idx, int is_even, double omega,
                            const double lim[3], const double forces[3], int level, int write_macro, int body_force,
                            double *rho, double *vx, double *vy, double *vz, double *bfx, double *bfy, double *bfz);

/* boundary conditions, QforBoundaryConditions layout: k[nbc], q27[dir*nbc + i] */
void orc_bc_noslip_bounce_back(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even);
void orc_bc_noslip_interpolated(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even, double omega);
void orc_bc_velocity_bounce_back(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                                 const double *ux, const double *uy, const double *uz);
void orc_bc_velocity_interpolated(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                                  double omega, const double *ux, const double *uy, const double *uz);
/* SlipCompressible (Slip/SlipCompressible.cu:44-550): the interpolated velocity BC with the node's own
   velocity as the wall velocity, its component along an axis zeroed where that axis's links are cut */
void orc_bc_slip(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even, double omega);
void orc_bc_pressure_neq(orc_level *L, const int32_t *k, const int32_t *kN, const double *rho_bc, uint32_t nbc,
                         int is_even, int direction);

/* InitNavierStokesCompressible_Device.cu:44-215 for one parity; geo: skip 15 (solid) and 16 (void) */
void orc_init(orc_level *L, const uint32_t *geo, const double *rho, const double *ux, const double *uy,
              const double *uz, int is_even);
/* InitNavierStokesCompressible_Device.cu:216-501 (the non-equilibrium init) for one parity; nb_inverse
   is neighborInverse (the node at -1 in x, y and z); solid and void nodes get 96 in their rest slot */
void orc_init_neq(orc_level *L, const uint32_t *geo, const uint32_t *nb_inverse, const double *rho, const double *ux,
                  const double *uy, const double *uz, double omega, int is_even);
/* MacroscopicQuantities.cu:194 compressible macros (rho, vx, vy, vz, pressure) for geo == 19 nodes */
void orc_macros(const orc_level *L, const uint32_t *geo, int is_even, double *rho, double *vx, double *vy,
                double *vz, double *press);
/* FP64 global mass sum(1+drho) and kinetic energy sum(0.5*(1+drho)*u^2) over a node list */
void orc_mass_energy(const orc_level *L, const uint32_t *idx, uint32_t n_idx, int is_even, double out[2]);

/* one time step of a single level in the order of UpdateGrid27::updateGrid (UpdateGrid27.cpp:54-95) */
typedef struct {
    int32_t *k; double *q; uint32_t n;                 /* no-slip list */
    int kind;                                          /* 0 none, 1 bounce-back, 2 interpolated */
} orc_noslip;
typedef struct {
    int32_t *k; double *q; uint32_t n; double *ux, *uy, *uz;
    int kind;                                          /* 0 none, 1 bounce-back, 2 interpolated */
} orc_velocity;
typedef struct {
    int32_t *k; int32_t *kN; double *rho; uint32_t n; int direction;
} orc_pressure;

/* ---- refinement: interpolation between levels ----
   Second-order moment interpolation of src/lbm/interpolation/InterpolationCoefficients.h:74-438 and
   src/lbm/refinement/Interpolation{CF,FC}.h, restated with the coefficients written as sign-pattern
   sums over the eight cell corners. Corner c = ix + 2 iy + 4 iz sits at (ix, iy, iz) - 1/2. */
/* moments of one source node: {drho, ux, uy, uz, kxy, kyz, kxz, kxxMyy, kxxMzz} */
void orc_interp_node_moments(const double *f, double omega, double out9[9]);
/* coefficients of the cell from the eight corners' moments, in the member order of
   InterpolationCoefficients: a, b, c (000 100 010 001 200 020 002 110 101 011 each),
   d000 d100 d010 d001 d110 d101 d011, a111 b111 c111 d111, LaplaceRho */
void orc_interp_coefficients(const double *mom8x9, double xoff, double yoff, double zoff, double out42[42]);
/* populations (f - w) at (x, y, z) of the cell from its coefficients; fc != 0: the fine-to-coarse form */
void orc_interp_point(const double *coef42, double omega_target, double eps, double x, double y, double z, int fc,
                      double out27[27]);
/* scaleCoarseToFineCompressible / scaleFineToCoarseCompressible (GridScaling/scale*.cu) for a list of cells */
void orc_scale_cf(orc_level *coarse, orc_level *fine, const uint32_t *coarse_cells, const uint32_t *fine_cells,
                  uint32_t n_cells, const double *ox, const double *oy, const double *oz, int coarse_is_even,
                  double omega_coarse, double omega_fine);
void orc_scale_fc(orc_level *coarse, orc_level *fine, const uint32_t *coarse_cells, const uint32_t *fine_cells,
                  uint32_t n_cells, const double *ox, const double *oy, const double *oz, int coarse_is_even,
                  double omega_coarse, double omega_fine);

/* drag and lift (PostProcessor/DragLift.cu:50-555, DragLift.cpp:52-73): per geometry BC node, the
   post part (after the collision, current parity) and the pre part (after the parity swap); the
   force is the node-ordered FP64 sum of pre - post */
void orc_drag_lift_post(const orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                        double *dx, double *dy, double *dz);
void orc_drag_lift_pre(const orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                       double *dx, double *dy, double *dz);
void orc_drag_lift_sum(const double *pre_x, const double *pre_y, const double *pre_z, const double *post_x,
                       const double *post_y, const double *post_z, uint32_t nbc, double force[3]);

/* the step with a geometry BC list (no-slip kinds) and, when drag_history is given, the drag force
   of every step into drag_history[3 * step] */
int orc_run_geo(orc_level *L, const uint32_t *fluid, uint32_t n_fluid, int *is_even, double omega, const double lim[3],
                const double forces[3], const orc_velocity *vel, const orc_noslip *ns, const orc_noslip *geo,
                double *drag_history, const orc_pressure *pr, int n_pr, int steps, int n_threads);

/* the same for a refinement level: forces scaled by 2^-level (KernelUtilities.h getForceFactor) */
int orc_run_level(orc_level *L, int level, const uint32_t *fluid, uint32_t n_fluid, int *is_even, double omega,
                  const double lim[3], const double forces[3], const orc_velocity *vel, const orc_noslip *ns,
                  const orc_noslip *geo, double *drag_history, const orc_pressure *pr, int n_pr, int steps,
                  int n_threads);

int orc_run(orc_level *L, const uint32_t *fluid, uint32_t n_fluid, int *is_even, double omega, const double lim[3],
            const double forces[3], const orc_velocity *vel, const orc_noslip *ns, const orc_pressure *pr, int n_pr,
            int steps, int n_threads);

#ifdef __cplusplus
}
#endif
#endif
