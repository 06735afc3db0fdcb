/*
 * ORACLE — test infrastructure, not product code (see oracle.h).
 *
 * CPU restatement of the VirtualFluids GPU hot path. Each function names the reference
 * file:line it follows. Compiled with -O2 -ffp-contract=off and no -march flags so that every
 * double operation is a separately rounded IEEE-754 operation, like the reference built for
 * the host.
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* src/lbm/constants/D3Q27.h:42-72 numbering; components as the direction names say */
const int ORC_CX[27] = { 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1 };
const int ORC_CY[27] = { 0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1 };
const int ORC_CZ[27] = { 0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1 };
/* D3Q27.h:85-110 inverse directions */
const int ORC_INV[27] = { 0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 26, 25, 24, 23, 22, 21, 20, 19 };
/* lattice weights c8o27, c2o27, c1o54, c1o216 (InitNavierStokesCompressible_Device.cu:175-202) */
const double ORC_W[27] = { 8. / 27.,
                           2. / 27., 2. / 27., 2. / 27., 2. / 27., 2. / 27., 2. / 27.,
                           1. / 54., 1. / 54., 1. / 54., 1. / 54., 1. / 54., 1. / 54.,
                           1. / 54., 1. / 54., 1. / 54., 1. / 54., 1. / 54., 1. / 54.,
                           1. / 216., 1. / 216., 1. / 216., 1. / 216., 1. / 216., 1. / 216., 1. / 216., 1. / 216. };

/* ---------------- K17, in double and in float ---------------- */
#define REAL double
#define SFX(name) name##_f64
#define ORC_ABS fabs
#include "k17_body.inc"
#undef REAL
#undef SFX
#undef ORC_ABS

#define REAL float
#define SFX(name) name##_f32
#define ORC_ABS fabsf
#include "k17_body.inc"
#undef REAL
#undef SFX
#undef ORC_ABS

void orc_chimera_f64(int which, double *abc, double v, double v2, double kinv, double k)
{
    switch (which) {
    case 0: chim_fwd_k_f64(&abc[0], &abc[1], &abc[2], v, v2, kinv, k); break;
    case 1: chim_bwd_k_f64(&abc[0], &abc[1], &abc[2], v, v2, kinv, k); break;
    case 2: chim_fwd_f64(&abc[0], &abc[1], &abc[2], v, v2); break;
    default: chim_bwd_f64(&abc[0], &abc[1], &abc[2], v, v2); break;
    }
}

/* ---------------- esoteric twist (KernelUtilities.h:66-132, 221-378) ---------------- */

/* even step: direction d lives in array plane d; odd step: in the plane of its inverse */
void orc_pointer_map(int is_even, int map[27])
{
    for (int d = 0; d < 27; ++d)
        map[d] = is_even ? d : ORC_INV[d];
}

/* ListIndices: the slot of direction d is at k moved +1 along every axis where d points negative;
   the chain goes x, then y, then z (k_MM0 = nbY[k_M00], k_MMM = nbZ[k_MM0]) */
uint32_t orc_read_index(const orc_level *L, uint32_t k, int d)
{
    if (ORC_CX[d] < 0) k = L->nbx[k];
    if (ORC_CY[d] < 0) k = L->nby[k];
    if (ORC_CZ[d] < 0) k = L->nbz[k];
    return k;
}

/* getPreCollisionDistribution (KernelUtilities.h:252) */
void orc_read_pre(const orc_level *L, uint32_t k, int is_even, double out[27])
{
    int map[27];
    orc_pointer_map(is_even, map);
    for (int d = 0; d < 27; ++d)
        out[d] = L->f[(uint64_t)map[d] * L->n + orc_read_index(L, k, d)];
}

/* setPostCollisionDistribution (KernelUtilities.h:350): inverse direction into the same slot */
void orc_write_post(orc_level *L, uint32_t k, int is_even, const double in[27])
{
    int map[27];
    orc_pointer_map(is_even, map);
    for (int d = 0; d < 27; ++d)
        L->f[(uint64_t)map[d] * L->n + orc_read_index(L, k, d)] = in[ORC_INV[d]];
}

/* getPostCollisionDistribution (KernelUtilities.h:283): post[d] is the population leaving k along d */
static void read_post(const orc_level *L, uint32_t k, int is_even, double post[27])
{
    int map[27];
    orc_pointer_map(is_even, map);
    for (int d = 0; d < 27; ++d) {
        const int e = ORC_INV[d];
        post[d] = L->f[(uint64_t)map[e] * L->n + orc_read_index(L, k, e)];
    }
}

/* setPreCollisionDistribution (KernelUtilities.h:319) for one direction */
static inline void write_pre_dir(orc_level *L, uint32_t k, const int map[27], int d, double v)
{
    L->f[(uint64_t)map[d] * L->n + orc_read_index(L, k, d)] = v;
}

/* ---------------- collision driver (RunCollision.cuh:75-143) ---------------- */
void orc_collision(orc_level *L, const uint32_t *idx, uint32_t n_idx, int is_even, double omega,
                   const double lim[3], const double forces[3], int level,
                   double *rho, double *vx, double *vy, double *vz, int n_threads)
{
    /* KernelUtilities.h:56 getForceFactor: 1 / 2^level */
    double factor = 1.0;
    for (int i = 1; i <= level; ++i)
        factor *= 2.0;
    factor = 1.0 / factor;
    const double fx = forces[0] * 0.5 * factor, fy = forces[1] * 0.5 * factor, fz = forces[2] * 0.5 * factor;
    (void)n_threads;
#ifdef _OPENMP
    if (n_threads > 0)
        omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)n_idx; ++i) {
        const uint32_t k = idx[i];
        double f[27], macro[4];
        orc_read_pre(L, k, is_even, f);
        orc_k17_f64(f, omega, lim, fx, fy, fz, macro);
        if (rho) {
            rho[k] = macro[0];
            vx[k] = macro[1];
            vy[k] = macro[2];
            vz[k] = macro[3];
        }
        orc_write_post(L, k, is_even, f);
    }
}

/* RunCollision.cuh:75-143 for every CollisionTemplate: the body-force variant adds the node's body
   force to the global forcing before the half-force scaling ((forces[c] + bodyForce[k]) * c1o2 *
   forceFactor, :88-90) and resets the node's body force (:93-95); the macroscopic variant writes
   drho and the velocity after the collision (:133-138). Sequential over the list. */
void orc_collision_template(orc_level *L, const uint32_t *idx, uint32_t n_idx, int is_even, double omega,
                            const double lim[3], const double forces[3], int level, int write_macro, int body_force,
                            double *rho, double *vx, double *vy, double *vz, double *bfx, double *bfy, double *bfz)
{
    double factor = 1.0;
    for (int i = 1; i <= level; ++i)
        factor *= 2.0;
    factor = 1.0 / factor;
    for (uint32_t i = 0; i < n_idx; ++i) {
        const uint32_t k = idx[i];
        double fx, fy, fz;
        if (body_force) {
            fx = (forces[0] + bfx[k]) * 0.5 * factor;
            fy = (forces[1] + bfy[k]) * 0.5 * factor;
            fz = (forces[2] + bfz[k]) * 0.5 * factor;
            bfx[k] = 0.0;
            bfy[k] = 0.0;
            bfz[k] = 0.0;
        } else {
            fx = forces[0] * 0.5 * factor;
            fy = forces[1] * 0.5 * factor;
            fz = forces[2] * 0.5 * factor;
        }
        double f[27], macro[4];
        orc_read_pre(L, k, is_even, f);
        orc_k17_f64(f, omega, lim, fx, fy, fz, macro);
        if (write_macro) {
            vx[k] = macro[1];
            vy[k] = macro[2];
            vz[k] = macro[3];
            rho[k] = macro[0];
        }
        orc_write_post(L, k, is_even, f);
    }
}

/* ---------------- boundary conditions ---------------- */

/* c . u as the reference kernels spell it: signed sum in x, y, z order (e.g. -vx1 - vx2 + vx3) */
static inline double signed_sum(int d, double ux, double uy, double uz)
{
    double s = 0.0;
    int first = 1;
    const int c[3] = { ORC_CX[d], ORC_CY[d], ORC_CZ[d] };
    const double u[3] = { ux, uy, uz };
    for (int a = 0; a < 3; ++a) {
        if (c[a] == 0)
            continue;
        if (first) {
            s = c[a] > 0 ? u[a] : -u[a];
            first = 0;
        } else {
            s = c[a] > 0 ? s + u[a] : s - u[a];
        }
    }
    return s;
}

static inline int q_active(double q) { return q >= 0.0 && q <= 1.0; }

/* The post-collision populations of every node of a BC list, read before the list writes anything
   ([i * 27 + d]). Where two nodes of one list are joined by a link cut from both ends, each node's
   write lands in a slot the other reads; reading first gives every node the collision's values,
   as a parallel kernel whose reads all precede its writes does, independent of the list order. */
static double *read_posts(const orc_level *L, const int32_t *k, uint32_t nbc, int is_even)
{
    double *all = (double *)malloc(sizeof(double) * 27 * (size_t)(nbc ? nbc : 1));
    if (!all) {
        fprintf(stderr, "oracle: out of memory for a BC list of %u nodes\n", nbc);
        abort();
    }
    /* each node fills its own row */
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)nbc; ++i)
        read_post(L, (uint32_t)k[i], is_even, all + 27 * (size_t)i);
    return all;
}

/* NoSlipBounceBack_Device (BoundaryConditions/NoSlip/NoSlipBounceBack.cu:44-179) */
void orc_bc_noslip_bounce_back(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even)
{
    int map_next[27];
    orc_pointer_map(!is_even, map_next);
    double *all = read_posts(L, k, nbc, is_even);
    /* all reads are done: every entry writes only its own node's slots */
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)nbc; ++i) {
        const uint32_t node = (uint32_t)k[i];
        const double *post = all + 27 * (size_t)i;
        for (int d = 1; d < 27; ++d)
            if (q_active(q27[(uint64_t)d * nbc + i]))
                write_pre_dir(L, node, map_next, ORC_INV[d], post[d]);
    }
    free(all);
}

/* VelocityBounceBack_Device (BoundaryConditions/Velocity/VelocityBounceBack.cu:44-188):
   f_inv(d) = f_d + 6 w_d (c_inv(d) . u_w) with 6w = 4/9, 1/9, 1/36 */
void orc_bc_velocity_bounce_back(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                                 const double *ux, const double *uy, const double *uz)
{
    int map_next[27];
    orc_pointer_map(!is_even, map_next);
    double *all = read_posts(L, k, nbc, is_even);
    /* all reads are done: every entry writes only its own node's slots */
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)nbc; ++i) {
        const uint32_t node = (uint32_t)k[i];
        const double *post = all + 27 * (size_t)i;
        for (int d = 1; d < 27; ++d) {
            if (!q_active(q27[(uint64_t)d * nbc + i]))
                continue;
            const int e = ORC_INV[d];
            const int nz = (ORC_CX[d] != 0) + (ORC_CY[d] != 0) + (ORC_CZ[d] != 0);
            const double coef = nz == 1 ? 4. / 9. : (nz == 2 ? 1. / 9. : 1. / 36.);
            write_pre_dir(L, node, map_next, e, post[d] + coef * signed_sum(e, ux[i], uy[i], uz[i]));
        }
    }
    free(all);
}

/* macroscopic values the interpolated kernels compute from post-collision populations
   (NoSlipInterpolatedCompressible.cu:134-153): plain sum for drho, grouped differences for j */
static void bc_macros(const double *p, double *drho, double *vx, double *vy, double *vz, double *cu_sq)
{
    static const int order[27] = { D_PMP, D_MPP, D_PPP, D_MMP, D_PMM, D_MPM, D_PPM, D_MMM, D_0PM, D_0MP, D_0PP, D_0MM,
                                   D_P0M, D_M0P, D_P0P, D_M0M, D_PM0, D_MP0, D_PP0, D_MM0, D_00P, D_00M, D_0P0, D_0M0,
                                   D_P00, D_M00, D_000 };
    double s = p[order[0]];
    for (int i = 1; i < 27; ++i)
        s += p[order[i]];
    *drho = s;
    const double r = 1.0 + s;
    *vx = (((((p[D_PMP] - p[D_MPM]) - (p[D_MPP] - p[D_PMM])) + ((p[D_PPP] - p[D_MMM]) - (p[D_MMP] - p[D_PPM])))
           + ((p[D_P0M] - p[D_M0P]) + (p[D_P0P] - p[D_M0M]))) + ((p[D_PM0] - p[D_MP0]) + (p[D_PP0] - p[D_MM0])))
          + (p[D_P00] - p[D_M00]);
    *vx = *vx / r;
    *vy = (((((-(p[D_PMP] - p[D_MPM])) + (p[D_MPP] - p[D_PMM])) + ((p[D_PPP] - p[D_MMM]) - (p[D_MMP] - p[D_PPM])))
           + ((p[D_0PM] - p[D_0MP]) + (p[D_0PP] - p[D_0MM]))) + ((-(p[D_PM0] - p[D_MP0])) + (p[D_PP0] - p[D_MM0])))
          + (p[D_0P0] - p[D_0M0]);
    *vy = *vy / r;
    *vz = (((((p[D_PMP] - p[D_MPM]) + (p[D_MPP] - p[D_PMM])) + ((p[D_PPP] - p[D_MMM]) + (p[D_MMP] - p[D_PPM])))
           + ((-(p[D_0PM] - p[D_0MP])) + (p[D_0PP] - p[D_0MM]))) + ((p[D_P0P] - p[D_M0M]) - (p[D_P0M] - p[D_M0P])))
          + (p[D_00P] - p[D_00M]);
    *vz = *vz / r;
    *cu_sq = 1.5 * (*vx * *vx + *vy * *vy + *vz * *vz) * (1.0 + s);
}

/* getEquilibriumForBC (KernelUtilities.h:171) */
static inline double feq_bc(double drho, double v, double cu_sq, double w)
{
    return w * (drho + 4.5 * v * v * (1.0 + drho) - cu_sq);
}

/* getInterpolatedDistributionForNoSlipBC (KernelUtilities.h:191) */
static inline double interp_noslip(double q, double f, double finv, double feq, double omega)
{
    return (1.0 - q) / (1.0 + q) * (f - finv + (f + finv - 2.0 * feq * omega) / (1.0 - omega)) * 0.5
         + (q * (f + finv)) / (1.0 + q);
}

/* getInterpolatedDistributionForVeloBC (KernelUtilities.h:176) */
static inline double interp_velocity(double q, double f, double finv, double feq, double omega, double v, double w)
{
    return (1.0 - q) / (1.0 + q) * (f - finv + (f + finv - 2.0 * feq * omega) / (1.0 - omega)) * 0.5
         + (q * (f + finv) - 6.0 * w * v) / (1.0 + q);
}

/* NoSlipInterpolatedCompressible_Device (NoSlip/NoSlipInterpolatedCompressible.cu:44-381) */
void orc_bc_noslip_interpolated(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even, double omega)
{
    int map_next[27];
    orc_pointer_map(!is_even, map_next);
    double *all = read_posts(L, k, nbc, is_even);
    /* all reads are done: every entry writes only its own node's slots */
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)nbc; ++i) {
        const uint32_t node = (uint32_t)k[i];
        const double *post = all + 27 * (size_t)i;
        double drho, vx, vy, vz, cu_sq;
        bc_macros(post, &drho, &vx, &vy, &vz, &cu_sq);
        for (int d = 1; d < 27; ++d) {
            const double q = q27[(uint64_t)d * nbc + i];
            if (!q_active(q))
                continue;
            const double feq = feq_bc(drho, signed_sum(d, vx, vy, vz), cu_sq, ORC_W[d]);
            write_pre_dir(L, node, map_next, ORC_INV[d], interp_noslip(q, post[d], post[ORC_INV[d]], feq, omega));
        }
    }
    free(all);
}

/* VelocityInterpolatedCompressible_Device (Velocity/VelocityInterpolatedCompressible.cu:44-420) */
void orc_bc_velocity_interpolated(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                                  double omega, const double *ux, const double *uy, const double *uz)
{
    int map_next[27];
    orc_pointer_map(!is_even, map_next);
    double *all = read_posts(L, k, nbc, is_even);
    /* all reads are done: every entry writes only its own node's slots */
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)nbc; ++i) {
        const uint32_t node = (uint32_t)k[i];
        const double *post = all + 27 * (size_t)i;
        double drho, vx, vy, vz, cu_sq;
        bc_macros(post, &drho, &vx, &vy, &vz, &cu_sq);
        for (int d = 1; d < 27; ++d) {
            const double q = q27[(uint64_t)d * nbc + i];
            if (!q_active(q))
                continue;
            const double feq = feq_bc(drho, signed_sum(d, vx, vy, vz), cu_sq, ORC_W[d]);
            const double vbc = signed_sum(d, ux[i], uy[i], uz[i]);
            write_pre_dir(L, node, map_next, ORC_INV[d],
                          interp_velocity(q, post[d], post[ORC_INV[d]], feq, omega, vbc, ORC_W[d]));
        }
    }
    free(all);
}

/* SlipCompressible_Device (Slip/SlipCompressible.cu:44-550): the interpolated velocity BC above with
   the node's own velocity as the wall velocity (slip length 1), except that the component along an
   axis is zero when the node's link along that axis, either way, is cut. The reference visits the six
   axis links first and zeroes the component there, so every diagonal link sees all three. */
void orc_bc_slip(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even, double omega)
{
    int map_next[27];
    orc_pointer_map(!is_even, map_next);
    double *all = read_posts(L, k, nbc, is_even);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)nbc; ++i) {
        const uint32_t node = (uint32_t)k[i];
        const double *post = all + 27 * (size_t)i;
        double drho, vx, vy, vz, cu_sq;
        bc_macros(post, &drho, &vx, &vy, &vz, &cu_sq);
        const int cut_x = q_active(q27[(uint64_t)D_P00 * nbc + i]) || q_active(q27[(uint64_t)D_M00 * nbc + i]);
        const int cut_y = q_active(q27[(uint64_t)D_0P0 * nbc + i]) || q_active(q27[(uint64_t)D_0M0 * nbc + i]);
        const int cut_z = q_active(q27[(uint64_t)D_00P * nbc + i]) || q_active(q27[(uint64_t)D_00M * nbc + i]);
        const double wx = cut_x ? 0.0 : vx, wy = cut_y ? 0.0 : vy, wz = cut_z ? 0.0 : vz;
        for (int d = 1; d < 27; ++d) {
            const double q = q27[(uint64_t)d * nbc + i];
            if (!q_active(q))
                continue;
            const double feq = feq_bc(drho, signed_sum(d, vx, vy, vz), cu_sq, ORC_W[d]);
            const double vbc = signed_sum(d, wx, wy, wz);
            write_pre_dir(L, node, map_next, ORC_INV[d],
                          interp_velocity(q, post[d], post[ORC_INV[d]], feq, omega, vbc, ORC_W[d]));
        }
    }
    free(all);
}

/* feq - w for one direction in the form of the pressure/init kernels: w (drho + (drho+1)(3cu + 4.5cu^2 - cusq)) */
static inline double feq_dir(int d, double drho, double vx, double vy, double vz, double cusq)
{
    if (d == D_000)
        return ORC_W[0] * (drho - (drho + 1.0) * cusq);
    const double cu = signed_sum(d, vx, vy, vz);
    return ORC_W[d] * (drho + (drho + 1.0) * (3.0 * cu + 4.5 * cu * cu - cusq));
}

/* PressureNonEquilibriumCompressible_Device (Pressure/PressureNonEquilibriumCompressible.cu:45-314):
   take the neighbour's non-equilibrium part, re-centre it on rhoBC, write the 18 populations
   whose component along the outlet axis is zero or points against 'direction' */
void orc_bc_pressure_neq(orc_level *L, const int32_t *k, const int32_t *kN, const double *rho_bc, uint32_t nbc,
                         int is_even, int direction)
{
    int map[27];
    orc_pointer_map(is_even, map);
    const int axis = ORC_CX[direction] != 0 ? 0 : (ORC_CY[direction] != 0 ? 1 : 2);
    const int sgn = axis == 0 ? ORC_CX[direction] : (axis == 1 ? ORC_CY[direction] : ORC_CZ[direction]);
    for (uint32_t i = 0; i < nbc; ++i) {
        double fn[27], drho1, inv, vx, vy, vz;
        orc_read_pre(L, (uint32_t)kN[i], is_even, fn);
        orc_macro_compressible_f64(fn, &drho1, &inv, &vx, &vy, &vz);
        const double cusq = 1.5 * (vx * vx + vy * vy + vz * vz);
        for (int d = 0; d < 27; ++d)
            fn[d] -= feq_dir(d, drho1, vx, vy, vz, cusq);
        drho1 = rho_bc[i];
        for (int d = 0; d < 27; ++d)
            fn[d] += feq_dir(d, drho1, vx, vy, vz, cusq);
        for (int d = 0; d < 27; ++d) {
            const int c = axis == 0 ? ORC_CX[d] : (axis == 1 ? ORC_CY[d] : ORC_CZ[d]);
            if (c != sgn)
                write_pre_dir(L, (uint32_t)k[i], map, d, fn[d]);
        }
    }
}

/* ---------------- initialisation and output ---------------- */

/* InitNavierStokesCompressible_Device (InitNavierStokesCompressible_Device.cu:44-215) */
void orc_init(orc_level *L, const uint32_t *geo, const double *rho, const double *ux, const double *uy,
              const double *uz, int is_even)
{
    int map[27];
    orc_pointer_map(is_even, map);
    /* every node writes its own 27 slots: the loop runs in parallel */
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t k = 0; k < (int64_t)L->n; ++k) {
        if (geo[k] == 15u || geo[k] == 16u)
            continue;
        const double drho = rho[k], vx = ux[k], vy = uy[k], vz = uz[k];
        const double cu_sq = 1.5 * (vx * vx + vy * vy + vz * vz);
        write_pre_dir(L, (uint32_t)k, map, D_000, ORC_W[0] * (drho - cu_sq * (1.0 + drho)));
        for (int d = 1; d < 27; ++d) {
            const double cu = signed_sum(d, vx, vy, vz);
            write_pre_dir(L, (uint32_t)k, map, d, ORC_W[d] * (drho + (1.0 + drho) * (3.0 * cu + 4.5 * cu * cu - cu_sq)));
        }
    }
}

/* InitNavierStokesCompressibleNonEquilibrium_Device (InitNavierStokesCompressible_Device.cu:216-501):
   the equilibrium above plus (1 + drho) times a non-equilibrium part per direction pair, from central
   differences of the velocities at the six face neighbours (the -1 ones reached from neighborInverse,
   the node at -1 in x, y and z, then stepped back up with neighborY/Z, neighborX/Z and neighborX/Y)
   and omega; the equilibrium is the stored value the part is added to. Solid and void nodes get 96 in
   their rest slot. The parts follow the reference's expressions term by term (eps and op are 1). */
void orc_init_neq(orc_level *L, const uint32_t *geo, const uint32_t *nb_inverse, const double *rho, const double *ux,
                  const double *uy, const double *uz, double omega, int is_even)
{
    int map[27];
    orc_pointer_map(is_even, map);
    /* the part of each direction: rest, then the pairs E, N, T, NE, SE, TE, BE, TN, BN, TNE, TSW, TSE, TNW */
    int part_of[27];
    {
        const int pairs[13][2] = { { D_P00, D_M00 }, { D_0P0, D_0M0 }, { D_00P, D_00M }, { D_PP0, D_MM0 },
                                   { D_PM0, D_MP0 }, { D_P0P, D_M0M }, { D_P0M, D_M0P }, { D_0PP, D_0MM },
                                   { D_0PM, D_0MP }, { D_PPP, D_MMM }, { D_PPM, D_MMP }, { D_PMP, D_MPM },
                                   { D_PMM, D_MPP } };
        part_of[D_000] = 0;
        for (int p = 0; p < 13; ++p)
            part_of[pairs[p][0]] = part_of[pairs[p][1]] = p + 1;
    }
    for (uint64_t k = 0; k < L->n; ++k) {
        if (geo[k] == 15u || geo[k] == 16u) {
            L->f[(uint64_t)map[D_000] * L->n + k] = 96.0;
            continue;
        }
        const uint32_t m = nb_inverse[k];
        const uint32_t plus[3] = { L->nbx[k], L->nby[k], L->nbz[k] };
        const uint32_t minus[3] = { L->nbz[L->nby[m]], L->nbz[L->nbx[m]], L->nby[L->nbx[m]] };
        const double *u[3] = { ux, uy, uz };
        double g[3][3]; /* g[i][j] = d u_i / d x_j */
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                g[i][j] = (u[i][plus[j]] - u[i][minus[j]]) / 2.0;
        const double ax = g[0][0], ay = g[0][1], az = g[0][2];
        const double bx = g[1][0], by = g[1][1], bz = g[1][2];
        const double cx = g[2][0], cy = g[2][1], cz = g[2][2];
        const double o = omega, op = 1.0, eps = 1.0;
        double p[14];
        p[1] = eps * ((5. * ax * o + 5. * by * o + 5. * cz * o - 8. * ax * op + 4. * by * op + 4. * cz * op) / (54. * o * op));
        p[2] = p[1] + eps * ((2. * (ax - by)) / (9. * o));
        p[3] = p[1] + eps * ((2. * (ax - cz)) / (9. * o));
        p[4] = eps * (-(5. * cz * o + 3. * (ay + bx) * op - 2. * cz * op + ax * (5. * o + op) + by * (5. * o + op))
                      / (54. * o * op));
        p[5] = p[4] + eps * ((ay + bx) / (9. * o));
        p[6] = eps * (-(5. * cz * o + by * (5. * o - 2. * op) + 3. * (az + cx) * op + cz * op + ax * (5. * o + op))
                      / (54. * o * op));
        p[7] = p[6] + eps * ((az + cx) / (9. * o));
        p[8] = eps * (-(5. * ax * o + 5. * by * o + 5. * cz * o - 2. * ax * op + by * op + 3. * bz * op + 3. * cy * op
                        + cz * op) / (54. * o * op));
        p[9] = p[8] + eps * ((bz + cy) / (9. * o));
        p[0] = eps * ((5. * (ax + by + cz)) / (9. * op));
        p[10] = eps * (-(ay + az + bx + bz + cx + cy) / (72. * o));
        p[11] = -p[10] - eps * ((ay + bx) / (36. * o));
        p[12] = -p[10] - eps * ((az + cx) / (36. * o));
        p[13] = -p[10] - eps * ((bz + cy) / (36. * o));
        const double drho = rho[k], vx = ux[k], vy = uy[k], vz = uz[k];
        const double cu_sq = 1.5 * (vx * vx + vy * vy + vz * vz);
        for (int d = 0; d < 27; ++d) {
            double v;
            if (d == D_000) {
                v = ORC_W[0] * (drho - cu_sq * (1.0 + drho));
            } else {
                const double cu = signed_sum(d, vx, vy, vz);
                v = ORC_W[d] * (drho + (1.0 + drho) * (3.0 * cu + 4.5 * cu * cu - cu_sq));
            }
            v = v + (1.0 + drho) * p[part_of[d]];
            write_pre_dir(L, (uint32_t)k, map, d, v);
        }
    }
}

/* getPressure (MacroscopicQuantities.h:139) */
static double pressure_of(const double *f, double rho, double vx, double vy, double vz)
{
    return (f[D_P00] + f[D_M00] + f[D_0P0] + f[D_0M0] + f[D_00P] + f[D_00M]
            + 2.0 * (f[D_PP0] + f[D_MM0] + f[D_PM0] + f[D_MP0] + f[D_P0P] + f[D_M0M] + f[D_P0M] + f[D_M0P] + f[D_0PP]
                     + f[D_0MM] + f[D_0PM] + f[D_0MP])
            + 3.0 * (f[D_PPP] + f[D_MMP] + f[D_PMP] + f[D_MPP] + f[D_PPM] + f[D_MMM] + f[D_PMM] + f[D_MPM])
            - rho - (vx * vx + vy * vy + vz * vz) * (1.0 + rho)) * 0.5 + rho;
}

/* calculateMacroscopicQuantitiesCompressible_device (PostProcessor/MacroscopicQuantities.cu:194) */
void orc_macros(const orc_level *L, const uint32_t *geo, int is_even, double *rho, double *vx, double *vy,
                double *vz, double *press)
{
    for (uint64_t k = 0; k < L->n; ++k) {
        rho[k] = vx[k] = vy[k] = vz[k] = 0.0;
        if (press)
            press[k] = 0.0;
        if (geo[k] != 19u)
            continue;
        double f[27];
        orc_read_pre(L, (uint32_t)k, is_even, f);
        const double r = orc_density_f64(f);
        rho[k] = r;
        vx[k] = mom_x_f64(f) / (r + 1.0);
        vy[k] = mom_y_f64(f) / (r + 1.0);
        vz[k] = mom_z_f64(f) / (r + 1.0);
        if (press)
            press[k] = pressure_of(f, r, vx[k], vy[k], vz[k]);
    }
}

void orc_mass_energy(const orc_level *L, const uint32_t *idx, uint32_t n_idx, int is_even, double out[2])
{
    double mass = 0.0, ekin = 0.0;
    for (uint32_t i = 0; i < n_idx; ++i) {
        double f[27], drho, inv, vx, vy, vz;
        orc_read_pre(L, idx[i], is_even, f);
        orc_macro_compressible_f64(f, &drho, &inv, &vx, &vy, &vz);
        mass += 1.0 + drho;
        ekin += 0.5 * (1.0 + drho) * (vx * vx + vy * vy + vz * vz);
    }
    out[0] = mass;
    out[1] = ekin;
}

static void run_noslip(orc_level *L, const orc_noslip *ns, int is_even, double omega)
{
    if (!ns || !ns->n)
        return;
    if (ns->kind == 1)
        orc_bc_noslip_bounce_back(L, ns->k, ns->q, ns->n, is_even);
    else if (ns->kind == 2)
        orc_bc_noslip_interpolated(L, ns->k, ns->q, ns->n, is_even, omega);
}

/* UpdateGrid27::updateGrid for one level (UpdateGrid27.cpp:54-95, postCollisionBC :227-252,
   preCollisionBC :288-300): collision; velocity, no-slip and geometry BCs (with the drag's post part
   before the geometry BC); parity toggle; the drag's pre part and sum; pressure BCs */
int orc_run_geo(orc_level *L, const uint32_t *fluid, uint32_t n_fluid, int *is_even, double omega, const double lim[3],
                const double forces[3], const orc_velocity *vel, const orc_noslip *ns, const orc_noslip *geo,
                double *drag_history, const orc_pressure *pr, int n_pr, int steps, int n_threads)
{
    return orc_run_level(L, 0, fluid, n_fluid, is_even, omega, lim, forces, vel, ns, geo, drag_history, pr, n_pr, steps,
                         n_threads);
}

int orc_run_level(orc_level *L, int level, const uint32_t *fluid, uint32_t n_fluid, int *is_even, double omega,
                  const double lim[3], const double forces[3], const orc_velocity *vel, const orc_noslip *ns,
                  const orc_noslip *geo, double *drag_history, const orc_pressure *pr, int n_pr, int steps,
                  int n_threads)
{
    const uint32_t ng = geo ? geo->n : 0;
    double *work = NULL;
    if (drag_history && ng) {
        work = (double *)malloc(sizeof(double) * 6 * ng);
        if (!work)
            return -1;
    }
    for (int t = 0; t < steps; ++t) {
        orc_collision(L, fluid, n_fluid, *is_even, omega, lim, forces, level, NULL, NULL, NULL, NULL, n_threads);
        if (vel && vel->n) {
            if (vel->kind == 1)
                orc_bc_velocity_bounce_back(L, vel->k, vel->q, vel->n, *is_even, vel->ux, vel->uy, vel->uz);
            else if (vel->kind == 2)
                orc_bc_velocity_interpolated(L, vel->k, vel->q, vel->n, *is_even, omega, vel->ux, vel->uy, vel->uz);
        }
        run_noslip(L, ns, *is_even, omega);
        if (work)
            orc_drag_lift_post(L, geo->k, geo->q, ng, *is_even, work + 3 * ng, work + 4 * ng, work + 5 * ng);
        run_noslip(L, geo, *is_even, omega);
        *is_even = !*is_even;
        if (work) {
            orc_drag_lift_pre(L, geo->k, geo->q, ng, *is_even, work, work + ng, work + 2 * ng);
            orc_drag_lift_sum(work, work + ng, work + 2 * ng, work + 3 * ng, work + 4 * ng, work + 5 * ng, ng,
                              drag_history + 3 * (size_t)t);
        }
        for (int p = 0; p < n_pr; ++p)
            orc_bc_pressure_neq(L, pr[p].k, pr[p].kN, pr[p].rho, pr[p].n, *is_even, pr[p].direction);
    }
    free(work);
    return 0;
}

int orc_run(orc_level *L, const uint32_t *fluid, uint32_t n_fluid, int *is_even, double omega, const double lim[3],
            const double forces[3], const orc_velocity *vel, const orc_noslip *ns, const orc_pressure *pr, int n_pr,
            int steps, int n_threads)
{
    return orc_run_geo(L, fluid, n_fluid, is_even, omega, lim, forces, vel, ns, NULL, NULL, pr, n_pr, steps, n_threads);
}

/* ---------------- refinement ---------------- */

/* MomentsOnSourceNode::calculate (InterpolationCoefficients.h:74-146): macroscopic values and the
   non-equilibrium second moments, k_ab = -3 omega (sum c_a c_b f / rho - u_a u_b) and
   k_aaMbb = -3/2 omega (sum (c_a^2 - c_b^2) f / rho - (u_a^2 - u_b^2)) */
void orc_interp_node_moments(const double *f, double omega, double out9[9])
{
    double drho, inv, vx, vy, vz;
    orc_macro_compressible_f64(f, &drho, &inv, &vx, &vy, &vz);
    double sxy = 0.0, syz = 0.0, sxz = 0.0, sxxyy = 0.0, sxxzz = 0.0;
    for (int d = 0; d < 27; ++d) {
        const int cx = ORC_CX[d], cy = ORC_CY[d], cz = ORC_CZ[d];
        sxy += (double)(cx * cy) * f[d];
        syz += (double)(cy * cz) * f[d];
        sxz += (double)(cx * cz) * f[d];
        sxxyy += (double)(cx * cx - cy * cy) * f[d];
        sxxzz += (double)(cx * cx - cz * cz) * f[d];
    }
    out9[0] = drho;
    out9[1] = vx;
    out9[2] = vy;
    out9[3] = vz;
    out9[4] = -3.0 * omega * (sxy * inv - vx * vy);
    out9[5] = -3.0 * omega * (syz * inv - vy * vz);
    out9[6] = -3.0 * omega * (sxz * inv - vx * vz);
    out9[7] = -1.5 * omega * (sxxyy * inv - (vx * vx - vy * vy));
    out9[8] = -1.5 * omega * (sxxzz * inv - (vx * vx - vz * vz));
}

/* coefficient order: for u (a), v (b), w (c): 000 100 010 001 200 020 002 110 101 011 (3 x 10),
   then d000 d100 d010 d001 d110 d101 d011, then a111 b111 c111 d111, LaplaceRho (42) */
enum { C_A = 0, C_B = 10, C_C = 20, C_D = 30, C_111 = 37, C_LAPLACE = 41 };
enum { K000 = 0, K100, K010, K001, K200, K020, K002, K110, K101, K011 };

/* the sum of q over the corners with the sign pattern s_x^px s_y^py s_z^pz */
static double pattern_sum(const double *mom8x9, int q, int px, int py, int pz)
{
    double s = 0.0;
    for (int c = 0; c < 8; ++c) {
        const int sx = (c & 1) ? 1 : -1, sy = (c & 2) ? 1 : -1, sz = (c & 4) ? 1 : -1;
        const int sign = (px ? sx : 1) * (py ? sy : 1) * (pz ? sz : 1);
        s += sign > 0 ? mom8x9[c * 9 + q] : -mom8x9[c * 9 + q];
    }
    return s;
}

void orc_interp_coefficients(const double *m, double xo, double yo, double zo, double out[42])
{
    /* trilinear part of u, v, w (quantities 1..3) and drho (0): mean, gradients, cross terms */
    double mean[4];
    const int base[4] = { C_D, C_A, C_B, C_C };
    for (int q = 0; q < 4; ++q) {
        mean[q] = pattern_sum(m, q, 0, 0, 0) / 8.0;
        const int b = base[q];
        double g100 = pattern_sum(m, q, 1, 0, 0) / 4.0, g010 = pattern_sum(m, q, 0, 1, 0) / 4.0;
        double g001 = pattern_sum(m, q, 0, 0, 1) / 4.0;
        double g110 = pattern_sum(m, q, 1, 1, 0) / 2.0, g101 = pattern_sum(m, q, 1, 0, 1) / 2.0;
        double g011 = pattern_sum(m, q, 0, 1, 1) / 2.0, g111 = pattern_sum(m, q, 1, 1, 1);
        if (q == 0) {
            out[C_D + 0] = mean[0];
            out[C_D + 1] = g100;
            out[C_D + 2] = g010;
            out[C_D + 3] = g001;
            out[C_D + 4] = g110;
            out[C_D + 5] = g101;
            out[C_D + 6] = g011;
            out[C_111 + 3] = g111;
        } else {
            out[b + K100] = g100;
            out[b + K010] = g010;
            out[b + K001] = g001;
            out[b + K110] = g110;
            out[b + K101] = g101;
            out[b + K011] = g011;
            out[C_111 + q - 1] = g111;
        }
    }
    /* quadratic terms from the non-equilibrium moments (4 kxy, 5 kyz, 6 kxz, 7 kxxMyy, 8 kxxMzz)
       and the cross derivatives of the other two components (continuity) */
    const double a110 = out[C_A + K110], a101 = out[C_A + K101];
    const double b110 = out[C_B + K110], b011 = out[C_B + K011];
    const double c101 = out[C_C + K101], c011 = out[C_C + K011];
    out[C_A + K200] = (b110 + c101) / 4.0 + (pattern_sum(m, 7, 1, 0, 0) + pattern_sum(m, 8, 1, 0, 0)) / 16.0;
    out[C_A + K020] = -b110 / 2.0 + pattern_sum(m, 4, 0, 1, 0) / 8.0;
    out[C_A + K002] = -c101 / 2.0 + pattern_sum(m, 6, 0, 0, 1) / 8.0;
    out[C_B + K200] = -a110 / 2.0 + pattern_sum(m, 4, 1, 0, 0) / 8.0;
    out[C_B + K020] = (a110 + c011) / 4.0 + (-2.0 * pattern_sum(m, 7, 0, 1, 0) + pattern_sum(m, 8, 0, 1, 0)) / 16.0;
    out[C_B + K002] = -c011 / 2.0 + pattern_sum(m, 5, 0, 0, 1) / 8.0;
    out[C_C + K200] = -a101 / 2.0 + pattern_sum(m, 6, 1, 0, 0) / 8.0;
    out[C_C + K020] = -b011 / 2.0 + pattern_sum(m, 5, 0, 1, 0) / 8.0;
    out[C_C + K002] = (a101 + b011) / 4.0 + (pattern_sum(m, 7, 0, 0, 1) - 2.0 * pattern_sum(m, 8, 0, 0, 1)) / 16.0;
    /* the corner values see the quadratic terms at x^2 = y^2 = z^2 = 1/4 */
    for (int q = 1; q < 4; ++q) {
        const int b = base[q];
        out[b + K000] = mean[q] - (out[b + K200] + out[b + K020] + out[b + K002]) / 4.0;
    }
    out[C_LAPLACE] = (xo != 0.0 || yo != 0.0 || zo != 0.0)
                         ? 0.0
                         : -3.0 * (out[C_A + K100] * out[C_A + K100] + out[C_B + K010] * out[C_B + K010] + out[C_C + K001] * out[C_C + K001])
                               - 6.0 * (out[C_B + K100] * out[C_A + K010] + out[C_C + K100] * out[C_A + K001] + out[C_C + K010] * out[C_B + K001]);
    /* move the expansion point by the offset (refinement into walls) */
    for (int q = 1; q < 4; ++q) {
        double *a = out + base[q];
        a[K000] = a[K000] + xo * a[K100] + yo * a[K010] + zo * a[K001] + xo * xo * a[K200] + yo * yo * a[K020]
                + zo * zo * a[K002] + xo * yo * a[K110] + xo * zo * a[K101] + yo * zo * a[K011];
        const double g100 = a[K100] + 2.0 * xo * a[K200] + yo * a[K110] + zo * a[K101];
        const double g010 = a[K010] + 2.0 * yo * a[K020] + xo * a[K110] + zo * a[K011];
        const double g001 = a[K001] + 2.0 * zo * a[K002] + xo * a[K101] + yo * a[K011];
        a[K100] = g100;
        a[K010] = g010;
        a[K001] = g001;
    }
    double *d = out + C_D;
    d[0] = d[0] + xo * d[1] + yo * d[2] + zo * d[3] + xo * yo * d[4] + xo * zo * d[5] + yo * zo * d[6];
    const double d100 = d[1] + yo * d[4] + zo * d[5], d010 = d[2] + xo * d[4] + zo * d[6], d001 = d[3] + xo * d[5] + yo * d[6];
    d[1] = d100;
    d[2] = d010;
    d[3] = d001;
}

/* interpolateCF (InterpolationCF.h:57-314) at (x, y, z) and interpolateFC (InterpolationFC.h:56-269)
   at the cell centre: density and velocity from the polynomials, second-order central moments from
   the strain rate scaled by -eps/omega (1 + drho), higher orders at equilibrium, then the backward
   chimera transform to f - w */
void orc_interp_point(const double *c, double omega, double eps, double x, double y, double z, int fc, double out[27])
{
    const double *a = c + C_A, *b = c + C_B, *w = c + C_C, *d = c + C_D;
    double press, u[3], g[3][3]; /* g[i][j] = d u_i / d x_j */
    if (fc) {
        press = d[0] - 2.0 * c[C_LAPLACE] / 8.0;
        u[0] = a[K000];
        u[1] = b[K000];
        u[2] = w[K000];
        const double *p[3] = { a, b, w };
        for (int i = 0; i < 3; ++i) {
            g[i][0] = p[i][K100];
            g[i][1] = p[i][K010];
            g[i][2] = p[i][K001];
        }
    } else {
        press = d[0] + x * d[1] + y * d[2] + z * d[3] + x * y * d[4] + x * z * d[5] + y * z * d[6] + x * y * z * c[C_111 + 3]
              + 3.0 * x * x * c[C_LAPLACE];
        const double *p[3] = { a, b, w };
        for (int i = 0; i < 3; ++i) {
            const double *q = p[i];
            const double q111 = c[C_111 + i];
            u[i] = q[K000] + x * q[K100] + y * q[K010] + z * q[K001] + x * x * q[K200] + y * y * q[K020] + z * z * q[K002]
                 + x * y * q[K110] + x * z * q[K101] + y * z * q[K011] + x * y * z * q111;
            g[i][0] = q[K100] + 2.0 * x * q[K200] + y * q[K110] + z * q[K101] + y * z * q111;
            g[i][1] = q[K010] + 2.0 * y * q[K020] + x * q[K110] + z * q[K011] + x * z * q111;
            g[i][2] = q[K001] + 2.0 * z * q[K002] + x * q[K101] + y * q[K011] + x * y * q111;
        }
    }
    const double s = eps / omega * (1.0 + press);
    double F3[3][3][3];
    memset(F3, 0, sizeof(F3));
#define M(i, j, k) F3[i][j][k]
    const double mxxMyy = -2.0 / 3.0 * (g[0][0] - g[1][1]) * s;
    const double mxxMzz = -2.0 / 3.0 * (g[0][0] - g[2][2]) * s;
    M(0, 1, 1) = -1.0 / 3.0 * (g[1][2] + g[2][1]) * s;
    M(1, 0, 1) = -1.0 / 3.0 * (g[0][2] + g[2][0]) * s;
    M(1, 1, 0) = -1.0 / 3.0 * (g[0][1] + g[1][0]) * s;
    M(0, 0, 0) = press;
    M(2, 0, 0) = (mxxMyy + mxxMzz + press) / 3.0;
    M(0, 2, 0) = (-2.0 * mxxMyy + mxxMzz + press) / 3.0;
    M(0, 0, 2) = (mxxMyy - 2.0 * mxxMzz + press) / 3.0;
    M(0, 2, 2) = M(2, 0, 2) = M(2, 2, 0) = press / 9.0;
    M(2, 2, 2) = press / 27.0;
    const double vx = u[0], vy = u[1], vz = u[2], vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
    static const double kinvZ[3][3] = { { 36, 9, 36 }, { 9, 9.0 / 4.0, 9 }, { 36, 9, 36 } };
    static const double kY[3][2] = { { 1.0 / 6, 1.0 / 18 }, { 2.0 / 3.0, 2.0 / 9.0 }, { 1.0 / 6, 1.0 / 18 } };
    static const double kinvY[3][2] = { { 6, 18 }, { 1.5, 4.5 }, { 6, 18 } };
    for (int jb = 0; jb < 3; ++jb)
        for (int kc = 0; kc < 3; ++kc) {
            if (jb == 0 && kc == 0)
                chim_bwd_k_f64(&M(0, 0, 0), &M(1, 0, 0), &M(2, 0, 0), vx, vx2, 1.0, 1.0);
            else if (jb == 2 && kc == 2)
                chim_bwd_k_f64(&M(0, 2, 2), &M(1, 2, 2), &M(2, 2, 2), vx, vx2, 9.0, 1.0 / 9);
            else if ((jb == 2 && kc == 0) || (jb == 0 && kc == 2))
                chim_bwd_k_f64(&M(0, jb, kc), &M(1, jb, kc), &M(2, jb, kc), vx, vx2, 3.0, 1.0 / 3);
            else
                chim_bwd_f64(&M(0, jb, kc), &M(1, jb, kc), &M(2, jb, kc), vx, vx2);
        }
    for (int ia = 0; ia < 3; ++ia)
        for (int kc = 0; kc < 3; ++kc) {
            if (kc == 1)
                chim_bwd_f64(&M(ia, 0, 1), &M(ia, 1, 1), &M(ia, 2, 1), vy, vy2);
            else
                chim_bwd_k_f64(&M(ia, 0, kc), &M(ia, 1, kc), &M(ia, 2, kc), vy, vy2, kinvY[ia][kc / 2], kY[ia][kc / 2]);
        }
    for (int ia = 0; ia < 3; ++ia)
        for (int jb = 0; jb < 3; ++jb)
            chim_bwd_k_f64(&M(ia, jb, 0), &M(ia, jb, 1), &M(ia, jb, 2), vz, vz2, kinvZ[ia][jb], 1.0 / kinvZ[ia][jb]);
    for (int dd = 0; dd < 27; ++dd)
        out[dd] = F3[ORC_CX[dd] + 1][ORC_CY[dd] + 1][ORC_CZ[dd] + 1];
#undef M
}

/* node of corner (ix, iy, iz) of a cell whose MMM node is `base`, stepping x, then y, then z */
static uint32_t cell_corner(const orc_level *L, uint32_t base, int ix, int iy, int iz)
{
    uint32_t k = base;
    if (ix) k = L->nbx[k];
    if (iy) k = L->nby[k];
    if (iz) k = L->nbz[k];
    return k;
}

static void cell_moments(const orc_level *L, uint32_t base, int is_even, double omega, double mom[72])
{
    for (int c = 0; c < 8; ++c) {
        double f[27];
        orc_read_pre(L, cell_corner(L, base, c & 1, (c >> 1) & 1, (c >> 2) & 1), is_even, f);
        orc_interp_node_moments(f, omega, mom + 9 * c);
    }
}

/* setPreCollisionDistribution of all 27 directions of node k */
static void write_pre_all(orc_level *L, uint32_t k, int is_even, const double f[27])
{
    int map[27];
    orc_pointer_map(is_even, map);
    for (int d = 0; d < 27; ++d)
        write_pre_dir(L, k, map, d, f[d]);
}

/* scaleCoarseToFineCompressible_Device (scaleCoarseToFineCompressible.cu:305-528): moments of the
   coarse cell at the coarse parity, populations of the eight fine nodes at (+-1/4)^3 written at the
   even parity of the fine level, epsilon 1/2 */
void orc_scale_cf(orc_level *coarse, orc_level *fine, const uint32_t *coarse_cells, const uint32_t *fine_cells,
                  uint32_t n_cells, const double *ox, const double *oy, const double *oz, int coarse_is_even,
                  double omega_coarse, double omega_fine)
{
    for (uint32_t i = 0; i < n_cells; ++i) {
        double mom[72], coef[42];
        cell_moments(coarse, coarse_cells[i], coarse_is_even, omega_coarse, mom);
        orc_interp_coefficients(mom, ox[i], oy[i], oz[i], coef);
        for (int c = 0; c < 8; ++c) {
            const int ix = c & 1, iy = (c >> 1) & 1, iz = (c >> 2) & 1;
            double f[27];
            orc_interp_point(coef, omega_fine, 0.5, ix ? 0.25 : -0.25, iy ? 0.25 : -0.25, iz ? 0.25 : -0.25, 0, f);
            write_pre_all(fine, cell_corner(fine, fine_cells[i], ix, iy, iz), 1, f);
        }
    }
}

/* scaleFineToCoarseCompressible_Device (scaleFineToCoarseCompressible.cu:76-124): moments of the fine
   cell at the even parity, populations of the coarse node at the cell centre written at the coarse
   parity, epsilon 2 */
void orc_scale_fc(orc_level *coarse, orc_level *fine, const uint32_t *coarse_cells, const uint32_t *fine_cells,
                  uint32_t n_cells, const double *ox, const double *oy, const double *oz, int coarse_is_even,
                  double omega_coarse, double omega_fine)
{
    for (uint32_t i = 0; i < n_cells; ++i) {
        double mom[72], coef[42], f[27];
        cell_moments(fine, fine_cells[i], 1, omega_fine, mom);
        orc_interp_coefficients(mom, ox[i], oy[i], oz[i], coef);
        orc_interp_point(coef, omega_coarse, 2.0, 0.0, 0.0, 0.0, 1, f);
        write_pre_all(coarse, coarse_cells[i], coarse_is_even, f);
    }
}

/* ---------------- drag and lift (PostProcessor/DragLift.cu, DragLift.cpp) ---------------- */

/* the bracket structure of dragX / dragY / dragZ (DragLift.cu:264-290): per axis four corner pairs,
   four edge pairs and the face pair, each pair (plus direction, minus direction) */
static const int DRAG_PAIRS[3][9][2] = {
    { { D_PMM, D_MPP }, { D_PPM, D_MMP }, { D_PMP, D_MPM }, { D_PPP, D_MMM },
      { D_P0M, D_M0P }, { D_P0P, D_M0M }, { D_PM0, D_MP0 }, { D_PP0, D_MM0 }, { D_P00, D_M00 } },
    { { D_MPP, D_PMM }, { D_PPM, D_MMP }, { D_MPM, D_PMP }, { D_PPP, D_MMM },
      { D_0PM, D_0MP }, { D_0PP, D_0MM }, { D_MP0, D_PM0 }, { D_PP0, D_MM0 }, { D_0P0, D_0M0 } },
    { { D_MPP, D_PMM }, { D_MMP, D_PPM }, { D_PMP, D_MPM }, { D_PPP, D_MMM },
      { D_0MP, D_0PM }, { D_0PP, D_0MM }, { D_M0P, D_P0M }, { D_P0P, D_M0M }, { D_00P, D_00M } }
};

static double drag_axis(const double f[27], const double on[27], int axis)
{
    double t[9];
    for (int i = 0; i < 9; ++i) {
        const int p = DRAG_PAIRS[axis][i][0], m = DRAG_PAIRS[axis][i][1];
        t[i] = (f[p] * on[p]) - (f[m] * on[m]);
    }
    return ((((t[0] + t[1]) + t[2]) + t[3]) + (((t[4] + t[5]) + t[6]) + t[7])) + t[8];
}

/* DragLiftPost27 (DragLift.cu:50-301): after the collision, minus the momentum of the populations
   leaving each geometry node through its cut links (q in [0, 1]) */
void orc_drag_lift_post(const orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                        double *dx, double *dy, double *dz)
{
    for (uint32_t i = 0; i < nbc; ++i) {
        double f[27], on[27];
        read_post(L, (uint32_t)k[i], is_even, f);
        for (int d = 0; d < 27; ++d)
            on[d] = q_active(q27[(uint64_t)d * nbc + i]) ? 1.0 : 0.0;
        dx[i] = -drag_axis(f, on, 0);
        dy[i] = -drag_axis(f, on, 1);
        dz[i] = -drag_axis(f, on, 2);
    }
}

/* DragLiftPre27 (DragLift.cu:304-555): after the parity swap, the populations about to be read by
   each geometry node, weighted by the cut link of the opposite direction */
void orc_drag_lift_pre(const orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                       double *dx, double *dy, double *dz)
{
    for (uint32_t i = 0; i < nbc; ++i) {
        double f[27], on[27];
        orc_read_pre(L, (uint32_t)k[i], is_even, f);
        for (int d = 0; d < 27; ++d)
            on[d] = q_active(q27[(uint64_t)ORC_INV[d] * nbc + i]) ? 1.0 : 0.0;
        dx[i] = -drag_axis(f, on, 0);
        dy[i] = -drag_axis(f, on, 1);
        dz[i] = -drag_axis(f, on, 2);
    }
}

/* calcDragLift (DragLift.cpp:52-73): the force as the node-ordered FP64 sum of pre - post */
void orc_drag_lift_sum(const double *pre_x, const double *pre_y, const double *pre_z, const double *post_x,
                       const double *post_y, const double *post_z, uint32_t nbc, double force[3])
{
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (uint32_t i = 0; i < nbc; ++i) {
        fx += pre_x[i] - post_x[i];
        fy += pre_y[i] - post_y[i];
        fz += pre_z[i] - post_z[i];
    }
    force[0] = fx;
    force[1] = fy;
    force[2] = fz;
}
