/*
 * ORACLE PIN — test infrastructure, not product code.
 *
 * A thin C-ABI shim around the reference's own header-only LBM arithmetic, compiled for the
 * host straight from the reference source tree (include paths point at it; nothing is copied).
 * Built twice by oracle/Makefile: with VF_DOUBLE_ACCURACY (real = double, libvfref64.so) and
 * without (real = float, libvfref32.so), mirroring src/basics/DataTypes.h:39-43. Used to pin the
 * plain-C restatement in oracle.c bit for bit, to generate the golden vectors under
 * tests/golden/, and as the reference arm of the benchmark (reference K17 header driven over
 * the esoteric-twist layout on the host cores).
 *
 * Reference entry points wrapped here:
 *   vf::lbm::runK17CompressibleNavierStokes<None>   src/lbm/collision/K17CompressibleNavierStokes.h:88
 *   vf::lbm::{forward,backward}{Inverse,}Chimera*   src/lbm/ChimeraTransformation.h:58-150
 *   vf::lbm::getDensity / getCompressibleMacroscopicValues  src/lbm/MacroscopicQuantities.h:55-137
 *   vf::lbm::MomentsOnSourceNodeSet::calculate*, calculateCoefficients
 *                                                   src/lbm/interpolation/InterpolationCoefficients.h:74-438
 *   vf::lbm::interpolateCF / interpolateFC          src/lbm/refinement/InterpolationCF.h:57, InterpolationFC.h:56
 */
#include <cstdint>
#include <cstring>

#include <lbm/ChimeraTransformation.h>
#include <lbm/MacroscopicQuantities.h>
#include <lbm/collision/K17CompressibleNavierStokes.h>
#include <lbm/interpolation/InterpolationCoefficients.h>
#include <lbm/refinement/InterpolationCF.h>
#include <lbm/refinement/InterpolationFC.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef VF_DOUBLE_ACCURACY
#define REF_FN(name) ref_##name##_f64
#else
#define REF_FN(name) ref_##name##_f32
#endif

extern "C" {

int REF_FN(real_bytes)() { return (int)sizeof(real); }

void REF_FN(k17)(real *f, real omega, const real *lim, real fx, real fy, real fz, real *macro)
{
    vf::lbm::CollisionParameter p;
    std::memcpy(p.distribution, f, 27 * sizeof(real));
    real limiters[3] = { lim[0], lim[1], lim[2] };
    p.omega = omega;
    p.quadricLimiter = limiters;
    p.forceX = fx;
    p.forceY = fy;
    p.forceZ = fz;
    vf::lbm::MacroscopicValues mv;
    vf::lbm::TurbulentViscosity tv;
    vf::lbm::runK17CompressibleNavierStokes<vf::lbm::TurbulenceModel::None>(p, mv, tv);
    std::memcpy(f, p.distribution, 27 * sizeof(real));
    if (macro) {
        macro[0] = mv.rho;
        macro[1] = mv.vx;
        macro[2] = mv.vy;
        macro[3] = mv.vz;
    }
}

/* which: 0 forwardInverseChimeraWithK, 1 backwardInverseChimeraWithK, 2 forwardChimera,
          3 backwardChimera, 4 forwardChimeraWithK, 5 backwardChimeraWithK */
void REF_FN(chimera)(int which, real *abc, real v, real v2, real kinv, real k)
{
    switch (which) {
    case 0: vf::lbm::forwardInverseChimeraWithK(abc[0], abc[1], abc[2], v, v2, kinv, k); break;
    case 1: vf::lbm::backwardInverseChimeraWithK(abc[0], abc[1], abc[2], v, v2, kinv, k); break;
    case 2: vf::lbm::forwardChimera(abc[0], abc[1], abc[2], v, v2); break;
    case 3: vf::lbm::backwardChimera(abc[0], abc[1], abc[2], v, v2); break;
    case 4: vf::lbm::forwardChimeraWithK(abc[0], abc[1], abc[2], v, v2, k); break;
    default: vf::lbm::backwardChimeraWithK(abc[0], abc[1], abc[2], v, v2, k); break;
    }
}

real REF_FN(density)(const real *f) { return vf::lbm::getDensity(f); }

void REF_FN(macro_compressible)(const real *f, real *out4)
{
    real drho, oneOverRho, vx, vy, vz;
    vf::lbm::getCompressibleMacroscopicValues(f, drho, oneOverRho, vx, vy, vz);
    out4[0] = drho;
    out4[1] = vx;
    out4[2] = vy;
    out4[3] = vz;
}

void REF_FN(incompressible_velocity)(const real *f, real *out3)
{
    out3[0] = vf::lbm::getIncompressibleVelocityX1(f);
    out3[1] = vf::lbm::getIncompressibleVelocityX2(f);
    out3[2] = vf::lbm::getIncompressibleVelocityX3(f);
}

/* the eight source nodes of an interpolation cell, in the order MMM, MMP, PMP, PMM, MPM, MPP, PPP, PPM
   (ScalingUtilities.h:53-200 visits them in this order); f8 = 8 x 27 populations */
static vf::lbm::MomentsOnSourceNodeSet moments_of(const real *f8, real omega)
{
    vf::lbm::MomentsOnSourceNodeSet m;
    m.calculateMMM(f8 + 0 * 27, omega);
    m.calculateMMP(f8 + 1 * 27, omega);
    m.calculatePMP(f8 + 2 * 27, omega);
    m.calculatePMM(f8 + 3 * 27, omega);
    m.calculateMPM(f8 + 4 * 27, omega);
    m.calculateMPP(f8 + 5 * 27, omega);
    m.calculatePPP(f8 + 6 * 27, omega);
    m.calculatePPM(f8 + 7 * 27, omega);
    return m;
}

/* all coefficients in the member order of InterpolationCoefficients (InterpolationCoefficients.h:63-71) */
void REF_FN(interp_coefficients)(const real *f8, real omega, real xoff, real yoff, real zoff, real *out46)
{
    vf::lbm::MomentsOnSourceNodeSet m = moments_of(f8, omega);
    vf::lbm::InterpolationCoefficients c;
    m.calculateCoefficients(c, xoff, yoff, zoff);
    const real v[46] = { c.a000, c.a100, c.a010, c.a001, c.a200, c.a020, c.a002, c.a110, c.a101, c.a011,
                         c.b000, c.b100, c.b010, c.b001, c.b200, c.b020, c.b002, c.b110, c.b101, c.b011,
                         c.c000, c.c100, c.c010, c.c001, c.c200, c.c020, c.c002, c.c110, c.c101, c.c011,
                         c.d000, c.d100, c.d010, c.d001, c.d110, c.d101, c.d011,
                         c.a111, c.b111, c.c111, c.d111, c.LaplaceRho, 0, 0, 0, 0 };
    std::memcpy(out46, v, sizeof(v));
}

/* coarse -> fine for one cell: moments with omega_source, populations at (x, y, z) with omega_target,
   epsilon 1/2 (scaleCoarseToFineCompressible.cu:46-300 / InterpolationCF.h:57) */
void REF_FN(interp_cf)(const real *f8, real omega_coarse, real omega_fine, real xoff, real yoff, real zoff,
                       real x, real y, real z, real *out27)
{
    vf::lbm::MomentsOnSourceNodeSet m = moments_of(f8, omega_coarse);
    vf::lbm::InterpolationCoefficients c;
    m.calculateCoefficients(c, xoff, yoff, zoff);
    vf::lbm::interpolateCF(out27, omega_fine, vf::basics::constant::c1o2, c, x, y, z);
}

/* fine -> coarse for one cell: epsilon 2, evaluated at the cell centre (scaleFineToCoarseCompressible.cu:46-70) */
void REF_FN(interp_fc)(const real *f8, real omega_fine, real omega_coarse, real xoff, real yoff, real zoff, real *out27)
{
    vf::lbm::MomentsOnSourceNodeSet m = moments_of(f8, omega_fine);
    vf::lbm::InterpolationCoefficients c;
    m.calculateCoefficients(c, xoff, yoff, zoff);
    vf::lbm::interpolateFC(out27, vf::basics::constant::c2o1, omega_coarse, c);
}

#ifdef VF_DOUBLE_ACCURACY
/*
 * Reference arm of the benchmark: one collision sweep over a list of fluid nodes of a level in
 * the GPU layout. The per-node arithmetic is the reference header; gather/scatter follow the
 * esoteric-twist addressing of src/gpu/core/Utilities/KernelUtilities.h:221-378 (pure index
 * arithmetic). OpenMP over nodes mirrors the CPU solver's 'omp for' over blocks
 * (src/cpu/core/Simulation/Simulation.cpp:366-392).
 */
static const int kInv[27] = { 0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 26, 25, 24, 23, 22, 21, 20, 19 };
static const int kCx[27] = { 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1 };
static const int kCy[27] = { 0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1 };
static const int kCz[27] = { 0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1 };

void ref_collision_sweep_f64(double *f, uint64_t n, const uint32_t *nbx, const uint32_t *nby, const uint32_t *nbz,
                             const uint32_t *idx, uint32_t n_idx, int is_even, double omega, const double *lim,
                             int n_threads)
{
#ifdef _OPENMP
    if (n_threads > 0)
        omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)n_idx; ++i) {
        const uint32_t k = idx[i];
        uint64_t slot[27];
        for (int d = 0; d < 27; ++d) {
            uint32_t s = k;
            if (kCx[d] < 0) s = nbx[s];
            if (kCy[d] < 0) s = nby[s];
            if (kCz[d] < 0) s = nbz[s];
            const int plane = is_even ? d : kInv[d];
            slot[d] = (uint64_t)plane * n + s;
        }
        double local[27], macro[4];
        for (int d = 0; d < 27; ++d)
            local[d] = f[slot[d]];
        ref_k17_f64(local, omega, lim, 0.0, 0.0, 0.0, macro);
        for (int d = 0; d < 27; ++d)
            f[slot[d]] = local[kInv[d]];
    }
}
#endif

} // extern "C"
