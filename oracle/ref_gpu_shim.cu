/*
 * ORACLE PIN — test infrastructure, not product code.
 *
 * The reference's own GPU kernels of the hot path, compiled with nvcc from the reference source
 * tree where it lies (the kernel sources are included by path; nothing is copied) into
 * _ref/libvfref_gpu64.so (FP64, real = double) and _ref/libvfref_gpu32.so (FP32, real = float; the
 * collision entry points only are used from it). Plain C entry points take device pointers and
 * launch the reference kernels with a one-dimensional grid, which their index calculation
 * (cuda_helper/CudaIndexCalculation.h get1DIndexFrom2DBlock) maps onto the same node indices as
 * the reference's own launchers. Built with -fmad=false, so every operation rounds on its own as
 * in the reference's host build; the tests compare the library's kernels against these.
 *
 * Kernels wrapped (all under src/gpu/core):
 *   runCollision + runK17CompressibleNavierStokes  Utilities/RunCollision.cuh:75, Kernel/Compressible/
 *                                                  NavierStokes/K17/K17CompressibleNavierStokes.cu:85-100
 *   NoSlipBounceBack_Device                        BoundaryConditions/NoSlip/NoSlipBounceBack.cu:44
 *   NoSlipInterpolatedCompressible_Device          BoundaryConditions/NoSlip/NoSlipInterpolatedCompressible.cu:44
 *   VelocityBounceBack_Device                      BoundaryConditions/Velocity/VelocityBounceBack.cu:44
 *   VelocityInterpolatedCompressible_Device        BoundaryConditions/Velocity/VelocityInterpolatedCompressible.cu:44
 *   PressureNonEquilibriumCompressible_Device      BoundaryConditions/Pressure/PressureNonEquilibriumCompressible.cu:45
 *   NoSlipInterpolatedIncompressible_Device, VelocityInterpolatedIncompressible_Device,
 *   VelocityWithPressureInterpolatedCompressible_Device, PressureNonEquilibriumIncompressible_Device,
 *   OutflowNonReflecting_Device, OutflowNonReflectingPressureCorrection_Device
 *                                                  BoundaryConditions/{NoSlip,Velocity,Pressure,Outflow}/
 *   InitNavierStokesCompressible_Device            PreProcessor/PreProcessorStrategy/InitNavierStokesCompressible/
 *                                                  InitNavierStokesCompressible_Device.cu:44
 *   calculateMacroscopicQuantitiesCompressible_device  PostProcessor/MacroscopicQuantities.cu:194
 *   scaleCoarseToFineCompressible_Device<false>    GridScaling/scaleCoarseToFineCompressible.cu:305
 *   scaleFineToCoarseCompressible_Device<false>    GridScaling/scaleFineToCoarseCompressible.cu:76
 *   DragLiftPost27 / DragLiftPre27                 PostProcessor/DragLift.cu:50, :304
 */
#include <cstdint>
#include <cstdlib>

#include "Utilities/KernelUtilities.h"
#include "Utilities/RunCollision.cuh"
#include <lbm/collision/K17CompressibleNavierStokes.h>

#include "BoundaryConditions/NoSlip/NoSlipBounceBack.cu"
#include "BoundaryConditions/NoSlip/NoSlipInterpolatedCompressible.cu"
#include "BoundaryConditions/Pressure/PressureNonEquilibriumCompressible.cu"
#include "BoundaryConditions/Velocity/VelocityBounceBack.cu"
#include "BoundaryConditions/Velocity/VelocityInterpolatedCompressible.cu"
#include "BoundaryConditions/Velocity/VelocityInterpolatedIncompressible.cu"
#include "BoundaryConditions/Velocity/VelocityWithPressureInterpolatedCompressible.cu"
#include "BoundaryConditions/NoSlip/NoSlipInterpolatedIncompressible.cu"
#include "BoundaryConditions/Slip/SlipCompressible.cu"
#include "BoundaryConditions/Pressure/PressureNonEquilibriumIncompressible.cu"
#include "BoundaryConditions/Outflow/OutflowNonReflecting.cu"
#include "BoundaryConditions/Outflow/OutflowNonReflectingPressureCorrection.cu"
#include "GridScaling/scaleCoarseToFineCompressible.cu"
#include "GridScaling/scaleFineToCoarseCompressible.cu"
#include "PostProcessor/DragLift.cu"
#include "PostProcessor/MacroscopicQuantities.cu"
#include "PreProcessor/PreProcessorStrategy/InitNavierStokesCompressible/InitNavierStokesCompressible_Device.cu"

// The host-side launchers of DragLift.cu and MacroscopicQuantities.cu, compiled along with the
// kernels, refer to the grid helper of cuda_helper/CudaGrid.cpp, which pulls in the reference's
// logger. This shim never calls those launchers; the helper is defined here only so the library
// links, and aborts if it is ever reached.
namespace vf::cuda
{
CudaGrid::CudaGrid(unsigned int, unsigned int) { std::abort(); }
void CudaGrid::print() const { std::abort(); }
dim3 getCudaGrid(unsigned int, unsigned int) { std::abort(); }
} // namespace vf::cuda

namespace
{
constexpr unsigned kThreads = 64;
inline unsigned blocks_for(uint64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }
inline int done() { return (int)cudaGetLastError(); }
} // namespace

extern "C" {

int refgpu_real_bytes() { return (int)sizeof(real); }

/* K17CompressibleNavierStokes<None>::runOnIndices with CollisionTemplate::Default; forces and
   quadric limiters are device arrays of 3 reals (getForcesDev, getQuadricLimitersDev) */
int refgpu_k17(real *dist, uint64_t n, unsigned *nbx, unsigned *nby, unsigned *nbz, const unsigned *fluid,
               unsigned n_fluid, int is_even, real omega, real *forces, real *limiters, real force_factor)
{
    if (n_fluid == 0)
        return 0;
    vf::gpu::GPUCollisionParameter p { omega,   nbx,     nby,     nbz,     dist,    nullptr, nullptr,
                                       nullptr, nullptr, nullptr, 0,       (int)n,  force_factor, forces,
                                       nullptr, nullptr, nullptr, limiters, is_even != 0, fluid, n_fluid };
    auto collision = [] __device__(vf::lbm::CollisionParameter & parameter, vf::lbm::MacroscopicValues & macroscopicValues,
                                   vf::lbm::TurbulentViscosity & turbulentViscosity) {
        return vf::lbm::runK17CompressibleNavierStokes<vf::lbm::TurbulenceModel::None>(parameter, macroscopicValues,
                                                                                        turbulentViscosity);
    };
    vf::gpu::runCollision<decltype(collision), vf::lbm::TurbulenceModel::None, false, false>
        <<<blocks_for(n_fluid), kThreads>>>(collision, p);
    return done();
}

/* K17CompressibleNavierStokes<None>::runOnIndices with any CollisionTemplate: the template
   switch of K17CompressibleNavierStokes.cu:114-139 (WriteMacroVars -> runCollision<.., true, false>,
   ApplyBodyForce -> <false, true>, AllFeatures and SubDomainBorder -> <true, true>); rho, vx, vy, vz
   receive the macroscopic values, bfx/bfy/bfz are the per-node body forces (read, then reset) */
int refgpu_k17_template(real *dist, uint64_t n, unsigned *nbx, unsigned *nby, unsigned *nbz, const unsigned *fluid,
                        unsigned n_fluid, int is_even, real omega, real *forces, real *limiters, real force_factor,
                        real *rho, real *vx, real *vy, real *vz, real *bfx, real *bfy, real *bfz, int tmpl)
{
    if (n_fluid == 0)
        return 0;
    vf::gpu::GPUCollisionParameter p { omega,   nbx,  nby,  nbz,  dist, rho,  vx,  vy,  vz,  nullptr, 0, (int)n,
                                       force_factor, forces, bfx,  bfy,  bfz, limiters, is_even != 0, fluid, n_fluid };
    auto collision = [] __device__(vf::lbm::CollisionParameter & parameter, vf::lbm::MacroscopicValues & macroscopicValues,
                                   vf::lbm::TurbulentViscosity & turbulentViscosity) {
        return vf::lbm::runK17CompressibleNavierStokes<vf::lbm::TurbulenceModel::None>(parameter, macroscopicValues,
                                                                                        turbulentViscosity);
    };
    using F = decltype(collision);
    constexpr auto none = vf::lbm::TurbulenceModel::None;
    switch (tmpl) {
    case 0: vf::gpu::runCollision<F, none, false, false><<<blocks_for(n_fluid), kThreads>>>(collision, p); break;
    case 1: vf::gpu::runCollision<F, none, true, false><<<blocks_for(n_fluid), kThreads>>>(collision, p); break;
    case 2: vf::gpu::runCollision<F, none, false, true><<<blocks_for(n_fluid), kThreads>>>(collision, p); break;
    case 3:
    case 4: vf::gpu::runCollision<F, none, true, true><<<blocks_for(n_fluid), kThreads>>>(collision, p); break;
    default: return -1;
    }
    return done();
}

int refgpu_noslip_bounce_back(real *dist, int *k, real *q, unsigned nbc, unsigned *nbx, unsigned *nby, unsigned *nbz,
                              uint64_t n, int is_even)
{
    if (nbc == 0)
        return 0;
    NoSlipBounceBack_Device<<<blocks_for(nbc), kThreads>>>(dist, k, q, nbc, nbx, nby, nbz, n, is_even != 0);
    return done();
}

int refgpu_noslip_interpolated(real *dist, int *k, real *q, unsigned nbc, real omega, unsigned *nbx, unsigned *nby,
                               unsigned *nbz, uint64_t n, int is_even)
{
    if (nbc == 0)
        return 0;
    NoSlipInterpolatedCompressible_Device<<<blocks_for(nbc), kThreads>>>(dist, k, q, nbc, omega, nbx, nby, nbz, n,
                                                                           is_even != 0);
    return done();
}

int refgpu_slip(real *dist, int *k, real *q, unsigned nbc, real omega, unsigned *nbx, unsigned *nby, unsigned *nbz,
                uint64_t n, int is_even)
{
    if (nbc == 0)
        return 0;
    SlipCompressible_Device<<<blocks_for(nbc), kThreads>>>(dist, k, q, nbc, omega, nbx, nby, nbz, n, is_even != 0);
    return done();
}

int refgpu_velocity_bounce_back(real *vx, real *vy, real *vz, real *dist, int *k, real *q, unsigned nbc, unsigned *nbx,
                                unsigned *nby, unsigned *nbz, uint64_t n, int is_even)
{
    if (nbc == 0)
        return 0;
    VelocityBounceBack_Device<<<blocks_for(nbc), kThreads>>>(vx, vy, vz, dist, k, q, nbc, nbx, nby, nbz, n, is_even != 0);
    return done();
}

int refgpu_velocity_interpolated(real *vx, real *vy, real *vz, real *dist, int *k, real *q, unsigned nbc, real omega,
                                 unsigned *nbx, unsigned *nby, unsigned *nbz, uint64_t n, int is_even)
{
    if (nbc == 0)
        return 0;
    VelocityInterpolatedCompressible_Device<<<blocks_for(nbc), kThreads>>>(vx, vy, vz, dist, k, q, nbc, omega, nbx, nby,
                                                                             nbz, n, is_even != 0);
    return done();
}

int refgpu_pressure_neq(real *rho_bc, real *dist, int *k, int *kn, int nbc, unsigned *nbx, unsigned *nby, unsigned *nbz,
                        uint64_t n, int is_even, int direction)
{
    if (nbc == 0)
        return 0;
    PressureNonEquilibriumCompressible_Device<<<blocks_for((uint64_t)nbc), kThreads>>>(
        rho_bc, dist, k, kn, nbc, nbx, nby, nbz, n, is_even != 0, (size_t)direction);
    return done();
}

int refgpu_noslip_interpolated_incompressible(real *dist, int *k, real *q, unsigned nbc, real omega, unsigned *nbx,
                                              unsigned *nby, unsigned *nbz, uint64_t n, int is_even)
{
    if (nbc == 0)
        return 0;
    NoSlipInterpolatedIncompressible_Device<<<blocks_for(nbc), kThreads>>>(dist, k, q, nbc, omega, nbx, nby, nbz, n,
                                                                             is_even != 0);
    return done();
}

int refgpu_velocity_interpolated_incompressible(real *vx, real *vy, real *vz, real *dist, int *k, real *q, unsigned nbc,
                                                real omega, unsigned *nbx, unsigned *nby, unsigned *nbz, uint64_t n,
                                                int is_even)
{
    if (nbc == 0)
        return 0;
    VelocityInterpolatedIncompressible_Device<<<blocks_for(nbc), kThreads>>>(vx, vy, vz, dist, k, q, nbc, omega, nbx,
                                                                               nby, nbz, n, is_even != 0);
    return done();
}

int refgpu_velocity_with_pressure(real *vx, real *vy, real *vz, real *dist, int *k, real *q, unsigned nbc, real omega,
                                  unsigned *nbx, unsigned *nby, unsigned *nbz, uint64_t n, int is_even)
{
    if (nbc == 0)
        return 0;
    VelocityWithPressureInterpolatedCompressible_Device<<<blocks_for(nbc), kThreads>>>(
        vx, vy, vz, dist, k, q, nbc, omega, nbx, nby, nbz, n, is_even != 0);
    return done();
}

int refgpu_pressure_neq_incompressible(real *rho_bc, real *dist, int *k, int *kn, int nbc, unsigned *nbx, unsigned *nby,
                                       unsigned *nbz, uint64_t n, int is_even, int direction)
{
    if (nbc == 0)
        return 0;
    PressureNonEquilibriumIncompressible_Device<<<blocks_for((uint64_t)nbc), kThreads>>>(
        rho_bc, dist, k, kn, nbc, nbx, nby, nbz, n, is_even != 0, (size_t)direction);
    return done();
}

int refgpu_outflow(real *rho_bc, real *dist, int *k, int *kn, int nbc, real omega, unsigned *nbx, unsigned *nby,
                   unsigned *nbz, uint64_t n, int is_even, int direction, int correction, real factor)
{
    if (nbc == 0)
        return 0;
    if (correction)
        OutflowNonReflectingPressureCorrection_Device<<<blocks_for((uint64_t)nbc), kThreads>>>(
            rho_bc, dist, k, kn, nbc, omega, nbx, nby, nbz, n, is_even != 0, direction, factor);
    else
        OutflowNonReflecting_Device<<<blocks_for((uint64_t)nbc), kThreads>>>(rho_bc, dist, k, kn, nbc, omega, nbx, nby,
                                                                              nbz, n, is_even != 0, direction);
    return done();
}

int refgpu_init(unsigned *nbx, unsigned *nby, unsigned *nbz, unsigned *geo, real *rho, real *ux, real *uy, real *uz,
                unsigned n, real *dist, int is_even)
{
    InitNavierStokesCompressible_Device<<<blocks_for(n), kThreads>>>(nbx, nby, nbz, geo, rho, ux, uy, uz, n, dist,
                                                                      is_even != 0);
    return done();
}

int refgpu_init_neq(unsigned *nbx, unsigned *nby, unsigned *nbz, unsigned *nb_inverse, unsigned *geo, real *rho,
                    real *ux, real *uy, real *uz, unsigned n, real *dist, real omega, int is_even)
{
    InitNavierStokesCompressibleNonEquilibrium_Device<<<blocks_for(n), kThreads>>>(
        nbx, nby, nbz, nb_inverse, geo, rho, ux, uy, uz, n, dist, omega, is_even != 0);
    return done();
}

int refgpu_macros(real *vx, real *vy, real *vz, real *rho, real *press, unsigned *geo, unsigned *nbx, unsigned *nby,
                  unsigned *nbz, uint64_t n, real *dist, int is_even)
{
    calculateMacroscopicQuantitiesCompressible_device<<<blocks_for(n), kThreads>>>(vx, vy, vz, rho, press, geo, nbx, nby,
                                                                                    nbz, n, dist, is_even != 0);
    return done();
}

int refgpu_scale_cf(real *dist_c, real *dist_f, unsigned *nbx_c, unsigned *nby_c, unsigned *nbz_c, unsigned *nbx_f,
                    unsigned *nby_f, unsigned *nbz_f, uint64_t n_c, uint64_t n_f, int coarse_is_even, unsigned *coarse_cells,
                    unsigned *fine_cells, unsigned n_cells, real omega_c, real omega_f, real *ox, real *oy, real *oz)
{
    if (n_cells == 0)
        return 0;
    ICellNeigh off { ox, oy, oz };
    scaleCoarseToFineCompressible_Device<false><<<blocks_for(n_cells), kThreads>>>(
        dist_c, dist_f, nbx_c, nby_c, nbz_c, nbx_f, nby_f, nbz_f, n_c, n_f, coarse_is_even != 0, coarse_cells,
        fine_cells, n_cells, omega_c, omega_f, nullptr, nullptr, off);
    return done();
}

int refgpu_scale_fc(real *dist_c, real *dist_f, unsigned *nbx_c, unsigned *nby_c, unsigned *nbz_c, unsigned *nbx_f,
                    unsigned *nby_f, unsigned *nbz_f, uint64_t n_c, uint64_t n_f, int coarse_is_even, unsigned *coarse_cells,
                    unsigned *fine_cells, unsigned n_cells, real omega_c, real omega_f, real *ox, real *oy, real *oz)
{
    if (n_cells == 0)
        return 0;
    ICellNeigh off { ox, oy, oz };
    scaleFineToCoarseCompressible_Device<false><<<blocks_for(n_cells), kThreads>>>(
        dist_c, dist_f, nbx_c, nby_c, nbz_c, nbx_f, nby_f, nbz_f, n_c, n_f, coarse_is_even != 0, coarse_cells,
        fine_cells, n_cells, omega_c, omega_f, nullptr, nullptr, off);
    return done();
}

int refgpu_drag_lift_post(real *dist, int *k, real *q, int nbc, double *dx, double *dy, double *dz, unsigned *nbx,
                          unsigned *nby, unsigned *nbz, uint64_t n, int is_even)
{
    if (nbc == 0)
        return 0;
    DragLiftPost27<<<blocks_for((uint64_t)nbc), kThreads>>>(dist, k, q, nbc, dx, dy, dz, nbx, nby, nbz, n, is_even != 0);
    return done();
}

int refgpu_drag_lift_pre(real *dist, int *k, real *q, int nbc, double *dx, double *dy, double *dz, unsigned *nbx,
                         unsigned *nby, unsigned *nbz, uint64_t n, int is_even)
{
    if (nbc == 0)
        return 0;
    DragLiftPre27<<<blocks_for((uint64_t)nbc), kThreads>>>(dist, k, q, nbc, dx, dy, dz, nbx, nby, nbz, n, is_even != 0);
    return done();
}

} // extern "C"
