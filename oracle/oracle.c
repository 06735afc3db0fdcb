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

/* NoSlipBounceBack_Device (BoundaryConditions/NoSlip/NoSlipBounceBack.cu:44-179) */
void orc_bc_noslip_bounce_back(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even)
{
    int map_next[27];
    orc_pointer_map(!is_even, map_next);
    for (uint32_t i = 0; i < nbc; ++i) {
        const uint32_t node = (uint32_t)k[i];
        double post[27];
        read_post(L, node, is_even, post);
        for (int d = 1; d < 27; ++d)
            if (q_active(q27[(uint64_t)d * nbc + i]))
                write_pre_dir(L, node, map_next, ORC_INV[d], post[d]);
    }
}

/* VelocityBounceBack_Device (BoundaryConditions/Velocity/VelocityBounceBack.cu:44-188):
   f_inv(d) = f_d + 6 w_d (c_inv(d) . u_w) with 6w = 4/9, 1/9, 1/36 */
void orc_bc_velocity_bounce_back(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                                 const double *ux, const double *uy, const double *uz)
{
    int map_next[27];
    orc_pointer_map(!is_even, map_next);
    for (uint32_t i = 0; i < nbc; ++i) {
        const uint32_t node = (uint32_t)k[i];
        double post[27];
        read_post(L, node, is_even, post);
        for (int d = 1; d < 27; ++d) {
            if (!q_active(q27[(uint64_t)d * nbc + i]))
                continue;
            const int e = ORC_INV[d];
            const int nz = (ORC_CX[d] != 0) + (ORC_CY[d] != 0) + (ORC_CZ[d] != 0);
            const double coef = nz == 1 ? 4. / 9. : (nz == 2 ? 1. / 9. : 1. / 36.);
            write_pre_dir(L, node, map_next, e, post[d] + coef * signed_sum(e, ux[i], uy[i], uz[i]));
        }
    }
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
    for (uint32_t i = 0; i < nbc; ++i) {
        const uint32_t node = (uint32_t)k[i];
        double post[27], drho, vx, vy, vz, cu_sq;
        read_post(L, node, is_even, post);
        bc_macros(post, &drho, &vx, &vy, &vz, &cu_sq);
        for (int d = 1; d < 27; ++d) {
            const double q = q27[(uint64_t)d * nbc + i];
            if (!q_active(q))
                continue;
            const double feq = feq_bc(drho, signed_sum(d, vx, vy, vz), cu_sq, ORC_W[d]);
            write_pre_dir(L, node, map_next, ORC_INV[d], interp_noslip(q, post[d], post[ORC_INV[d]], feq, omega));
        }
    }
}

/* VelocityInterpolatedCompressible_Device (Velocity/VelocityInterpolatedCompressible.cu:44-420) */
void orc_bc_velocity_interpolated(orc_level *L, const int32_t *k, const double *q27, uint32_t nbc, int is_even,
                                  double omega, const double *ux, const double *uy, const double *uz)
{
    int map_next[27];
    orc_pointer_map(!is_even, map_next);
    for (uint32_t i = 0; i < nbc; ++i) {
        const uint32_t node = (uint32_t)k[i];
        double post[27], drho, vx, vy, vz, cu_sq;
        read_post(L, node, is_even, post);
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
    for (uint64_t k = 0; k < L->n; ++k) {
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

/* UpdateGrid27::updateGrid for one level (UpdateGrid27.cpp:54-95): collision, post-collision
   velocity then no-slip BCs, parity toggle, pre-collision pressure BCs */
int orc_run(orc_level *L, const uint32_t *fluid, uint32_t n_fluid, int *is_even, double omega, const double lim[3],
            const double forces[3], const orc_velocity *vel, const orc_noslip *ns, const orc_pressure *pr, int n_pr,
            int steps, int n_threads)
{
    for (int t = 0; t < steps; ++t) {
        orc_collision(L, fluid, n_fluid, *is_even, omega, lim, forces, 0, NULL, NULL, NULL, NULL, n_threads);
        if (vel && vel->n) {
            if (vel->kind == 1)
                orc_bc_velocity_bounce_back(L, vel->k, vel->q, vel->n, *is_even, vel->ux, vel->uy, vel->uz);
            else if (vel->kind == 2)
                orc_bc_velocity_interpolated(L, vel->k, vel->q, vel->n, *is_even, omega, vel->ux, vel->uy, vel->uz);
        }
        if (ns && ns->n) {
            if (ns->kind == 1)
                orc_bc_noslip_bounce_back(L, ns->k, ns->q, ns->n, *is_even);
            else if (ns->kind == 2)
                orc_bc_noslip_interpolated(L, ns->k, ns->q, ns->n, *is_even, omega);
        }
        *is_even = !*is_even;
        for (int p = 0; p < n_pr; ++p)
            orc_bc_pressure_neq(L, pr[p].k, pr[p].kN, pr[p].rho, pr[p].n, *is_even, pr[p].direction);
    }
    return 0;
}
