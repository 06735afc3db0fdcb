// Definitions of Launchers<S> for one arithmetic variant (VFB_NS, VFB_EXACT). Included by the
// per-storage translation units, which explicitly instantiate one storage type each.
#pragma once
#include <algorithm>
#include <type_traits>
#include <cstring>

#include "kernels.cuh"
#include "launch.h"

#ifndef VFB_EXACT
#error "VFB_EXACT must be defined"
#endif

namespace vfb {
namespace VFB_NS {

namespace {
inline unsigned grid1d(uint64_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

template <class C>
K17Rates<C> rates_of(double omega, const double lim[3])
{
    return make_k17_rates<C>((C)omega, (C)lim[0], (C)lim[1], (C)lim[2]);
}

// RunCollision.cuh:112-114: forces * c1o2 * forceFactor, forceFactor = 1/2^level (KernelUtilities.h:56)
template <class C>
C force_factor(int level)
{
    C f = C(1);
    for (int i = 1; i <= level; ++i)
        f *= C(2);
    return C(1) / f;
}
} // namespace

template <class S>
cudaError_t Launchers<S>::k17_list(const vfb_level *L, const uint32_t *idx, uint32_t n, int tmpl, cudaStream_t s,
                                   const uint32_t *slots, uint64_t slots_stride)
{
    using C = typename Codec<S>::compute;
    if (n == 0)
        return cudaSuccess;
    ListCollideArgs<C> a;
    a.dist = L->distributions;
    a.n = L->number_of_nodes;
    a.nbx = L->neighbor_x;
    a.nby = L->neighbor_y;
    a.nbz = L->neighbor_z;
    a.idx = idx;
    a.n_idx = n;
    a.slots = slots;
    a.slots_stride = slots_stride;
    a.rates = rates_of<C>(L->omega, L->quadric_limiters);
    const C ff = force_factor<C>(L->level);
    a.fx = (C)L->forces[0] * C(0.5) * ff;
    a.fy = (C)L->forces[1] * C(0.5) * ff;
    a.fz = (C)L->forces[2] * C(0.5) * ff;
    a.force0 = (C)L->forces[0];
    a.force1 = (C)L->forces[1];
    a.force2 = (C)L->forces[2];
    a.force_factor = ff;
    a.bfx = static_cast<C *>(L->body_force_x);
    a.bfy = static_cast<C *>(L->body_force_y);
    a.bfz = static_cast<C *>(L->body_force_z);
    a.rho = static_cast<C *>(L->rho);
    a.vx = static_cast<C *>(L->velocity_x);
    a.vy = static_cast<C *>(L->velocity_y);
    a.vz = static_cast<C *>(L->velocity_z);
    const bool wm = tmpl == VFB_COLLISION_WRITE_MACRO_VARS || tmpl == VFB_COLLISION_ALL_FEATURES || tmpl == VFB_COLLISION_SUBDOMAIN_BORDER;
    const bool bf = tmpl == VFB_COLLISION_APPLY_BODY_FORCE || tmpl == VFB_COLLISION_ALL_FEATURES || tmpl == VFB_COLLISION_SUBDOMAIN_BORDER;
    const unsigned B = 128, G = grid1d(n, B);
    const bool even = L->is_even_timestep != 0;
#define VFB_K17L(E, W, F) k17_list_kernel<S, VFB_EXACT, E, W, F><<<G, B, 0, s>>>(a)
    if (even) {
        if (wm && bf) VFB_K17L(true, true, true);
        else if (wm) VFB_K17L(true, true, false);
        else if (bf) VFB_K17L(true, false, true);
        else VFB_K17L(true, false, false);
    } else {
        if (wm && bf) VFB_K17L(false, true, true);
        else if (wm) VFB_K17L(false, true, false);
        else if (bf) VFB_K17L(false, false, true);
        else VFB_K17L(false, false, false);
    }
#undef VFB_K17L
    return cudaGetLastError();
}

// the default collision template over a staged slot table: persistent warps, as many blocks as
// are resident on the device
template <class S>
cudaError_t Launchers<S>::k17_list_staged(const vfb_level *L, const uint32_t *slots, uint64_t slots_stride, uint32_t n,
                                          int *status, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    if (n == 0)
        return cudaSuccess;
    ListCollideArgs<C> a{};
    a.dist = L->distributions;
    a.n = L->number_of_nodes;
    a.n_idx = n;
    a.slots = slots;
    a.slots_stride = slots_stride;
    a.rates = rates_of<C>(L->omega, L->quadric_limiters);
    const C ff = force_factor<C>(L->level);
    a.fx = (C)L->forces[0] * C(0.5) * ff;
    a.fy = (C)L->forces[1] * C(0.5) * ff;
    a.fz = (C)L->forces[2] * C(0.5) * ff;
    const bool even = L->is_even_timestep != 0;
    const void *fn = even ? reinterpret_cast<const void *>(k17_list_staged_kernel<S, VFB_EXACT, true>)
                          : reinterpret_cast<const void *>(k17_list_staged_kernel<S, VFB_EXACT, false>);
    int dev = 0, sms = 1, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 128, 0);
    if (e != cudaSuccess)
        return e;
    const int64_t tiles = ((int64_t)n + ListTile::N - 1) / ListTile::N;
    const int64_t want = (tiles + ListTile::WARPS - 1) / ListTile::WARPS;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)std::max(occ, 1) * sms));
    if (even) k17_list_staged_kernel<S, VFB_EXACT, true><<<grid, 128, 0, s>>>(a, status);
    else k17_list_staged_kernel<S, VFB_EXACT, false><<<grid, 128, 0, s>>>(a, status);
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::bc(const vfb_level *L, const vfb_bc *bc, int kind, cudaStream_t s, const NodeAddr *box,
                             void *snap, const uint32_t *guard, void *saved)
{
    if (bc->number_of_bc_nodes == 0)
        return cudaSuccess;
    BCArgs a;
    a.dist = L->distributions;
    a.n = L->number_of_nodes;
    a.nbx = box ? nullptr : L->neighbor_x;
    a.nby = box ? nullptr : L->neighbor_y;
    a.nbz = box ? nullptr : L->neighbor_z;
    a.box = box ? *box : NodeAddr{ 0, 0, 0, 0 };
    a.k = bc->k;
    a.q27 = bc->q27;
    a.nbc = bc->number_of_bc_nodes;
    a.ux = bc->vx;
    a.uy = bc->vy;
    a.uz = bc->vz;
    a.omega = L->omega;
    a.snap = nullptr;
    a.guard = nullptr;
    a.saved = nullptr;
    const unsigned B = 128, G = grid1d(a.nbc, B);
    const bool even = L->is_even_timestep != 0;
    using C = typename Codec<S>::compute;
    if (snap) {
        if (even) bc_snapshot_kernel<S, true><<<G, B, 0, s>>>(a, static_cast<C *>(snap));
        else bc_snapshot_kernel<S, false><<<G, B, 0, s>>>(a, static_cast<C *>(snap));
        a.snap = snap;
    } else if (guard) {
        a.guard = guard;
        if (even) bc_guard_kernel<S, true><<<G, B, 0, s>>>(a, static_cast<C *>(saved));
        else bc_guard_kernel<S, false><<<G, B, 0, s>>>(a, static_cast<C *>(saved));
        a.saved = saved;
    }
    switch (kind) {
    case kNoSlipBB:
        if (even) bc_bounce_back_kernel<S, true, false><<<G, B, 0, s>>>(a);
        else bc_bounce_back_kernel<S, false, false><<<G, B, 0, s>>>(a);
        break;
    case kVelocityBB:
        if (even) bc_bounce_back_kernel<S, true, true><<<G, B, 0, s>>>(a);
        else bc_bounce_back_kernel<S, false, true><<<G, B, 0, s>>>(a);
        break;
    case kNoSlipInterp:
        if (even) bc_interpolated_kernel<S, true, false><<<G, B, 0, s>>>(a);
        else bc_interpolated_kernel<S, false, false><<<G, B, 0, s>>>(a);
        break;
    case kVelocityInterp:
        if (even) bc_interpolated_kernel<S, true, true><<<G, B, 0, s>>>(a);
        else bc_interpolated_kernel<S, false, true><<<G, B, 0, s>>>(a);
        break;
    case kNoSlipInterpIncomp:
        if (even) bc_interpolated_kernel<S, true, false, kBCIncompressible><<<G, B, 0, s>>>(a);
        else bc_interpolated_kernel<S, false, false, kBCIncompressible><<<G, B, 0, s>>>(a);
        break;
    case kVelocityInterpIncomp:
        if (even) bc_interpolated_kernel<S, true, true, kBCIncompressible><<<G, B, 0, s>>>(a);
        else bc_interpolated_kernel<S, false, true, kBCIncompressible><<<G, B, 0, s>>>(a);
        break;
    case kVelocityWithPressure:
        if (even) bc_interpolated_kernel<S, true, true, kBCWithPressure><<<G, B, 0, s>>>(a);
        else bc_interpolated_kernel<S, false, true, kBCWithPressure><<<G, B, 0, s>>>(a);
        break;
    case kSlipInterp:
        if (even) bc_interpolated_kernel<S, true, true, kBCSlip><<<G, B, 0, s>>>(a);
        else bc_interpolated_kernel<S, false, true, kBCSlip><<<G, B, 0, s>>>(a);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::pressure(const vfb_level *L, const vfb_directional_bc *bc, cudaStream_t s,
                                   const NodeAddr *box, int kind)
{
    if (bc->number_of_bc_nodes == 0)
        return cudaSuccess;
    PressureArgs a;
    a.dist = L->distributions;
    a.n = L->number_of_nodes;
    a.nbx = box ? nullptr : L->neighbor_x;
    a.nby = box ? nullptr : L->neighbor_y;
    a.nbz = box ? nullptr : L->neighbor_z;
    a.box = box ? *box : NodeAddr{ 0, 0, 0, 0 };
    a.k = bc->k;
    a.kN = bc->k_neighbor;
    a.rho_bc = bc->rho_bc;
    a.nbc = bc->number_of_bc_nodes;
    a.direction = bc->direction;
    const unsigned B = 128, G = grid1d(a.nbc, B);
    const bool even = L->is_even_timestep != 0;
    const double corr = L->outflow_pressure_correction_factor;
    switch (kind) {
    case kPressureNeqComp:
        if (even) bc_pressure_neq_kernel<S, true><<<G, B, 0, s>>>(a);
        else bc_pressure_neq_kernel<S, false><<<G, B, 0, s>>>(a);
        break;
    case kPressureNeqIncomp:
        if (even) bc_pressure_neq_kernel<S, true, true><<<G, B, 0, s>>>(a);
        else bc_pressure_neq_kernel<S, false, true><<<G, B, 0, s>>>(a);
        break;
    case kOutflowNonReflecting:
        if (even) bc_outflow_kernel<S, true, false><<<G, B, 0, s>>>(a, corr);
        else bc_outflow_kernel<S, false, false><<<G, B, 0, s>>>(a, corr);
        break;
    case kOutflowPressureCorrection:
        if (even) bc_outflow_kernel<S, true, true><<<G, B, 0, s>>>(a, corr);
        else bc_outflow_kernel<S, false, true><<<G, B, 0, s>>>(a, corr);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::pool_collide(void *arena, const void *domains, const uint2 *items, const uint32_t *n_items,
                                       int nodes_per_thread, bool even, unsigned grid, unsigned block, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    PoolArgs<C> a;
    a.arena = arena;
    a.domains = static_cast<const PoolDomain<C> *>(domains);
    a.items = items;
    a.n_items = n_items;
    a.nodes_per_thread = nodes_per_thread;
    if (even) k17_pool_kernel<S, VFB_EXACT, true><<<grid, block, 0, s>>>(a);
    else k17_pool_kernel<S, VFB_EXACT, false><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <class S>
const void *Launchers<S>::pool_kernel(bool even)
{
    return even ? reinterpret_cast<const void *>(k17_pool_kernel<S, VFB_EXACT, true>)
                : reinterpret_cast<const void *>(k17_pool_kernel<S, VFB_EXACT, false>);
}

template <class S>
size_t Launchers<S>::pool_domain_bytes()
{
    return sizeof(PoolDomain<typename Codec<S>::compute>);
}

// the domain record in the compute type of S, with the rates and forces rounded as the box path
// rounds them (so a domain in the pool and the same box alone compute the same bits)
template <class S>
void Launchers<S>::pool_domain(void *out, const PoolDomainSpec &spec)
{
    using C = typename Codec<S>::compute;
    PoolDomain<C> d;
    std::memset(&d, 0, sizeof(d));
    d.dist_offset = spec.dist_offset;
    d.pitch = spec.pitch;
    d.mask_offset = spec.mask_offset;
    d.nx = spec.nx;
    d.ny = spec.ny;
    d.nz = spec.nz;
    d.flags = spec.flags;
    d.rates = rates_of<C>(spec.omega, spec.lim);
    d.div_nx = make_fast_div((uint32_t)spec.nx);
    d.div_ny = make_fast_div((uint32_t)spec.ny);
    d.fx = (C)spec.half_force[0];
    d.fy = (C)spec.half_force[1];
    d.fz = (C)spec.half_force[2];
    d.omega = spec.omega;
    d.noslip_offset = spec.noslip_offset;
    d.noslip_cut_offset = spec.noslip_cut_offset;
    d.noslip_q_offset = spec.noslip_q_offset;
    d.noslip_guard_offset = spec.noslip_guard_offset;
    d.noslip_saved_offset = spec.noslip_saved_offset;
    d.pressure_offset = spec.pressure_offset;
    d.pressure_rho_offset = spec.pressure_rho_offset;
    d.n_noslip = spec.n_noslip;
    d.n_guarded = spec.n_guarded;
    d.n_pressure = spec.n_pressure;
    std::memcpy(out, &d, sizeof(d));
}

template <class S>
cudaError_t Launchers<S>::pool_mass(void *arena, const void *domains, const uint2 *items, uint32_t n_items,
                                    int nodes_per_thread, int threads, bool even, double *partials, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    if (n_items == 0)
        return cudaSuccess;
    PoolArgs<C> a;
    a.arena = arena;
    a.domains = static_cast<const PoolDomain<C> *>(domains);
    a.items = items;
    a.n_items = nullptr;
    a.nodes_per_thread = nodes_per_thread;
    if (even) pool_mass_kernel<S, true><<<n_items, threads, 0, s>>>(a, partials);
    else pool_mass_kernel<S, false><<<n_items, threads, 0, s>>>(a, partials);
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::pool_bcs(void *arena, const void *domains, const uint2 *noslip_items,
                                   const uint32_t *n_noslip_items, const uint2 *guard_items,
                                   const uint32_t *n_guard_items, const uint2 *pressure_items,
                                   const uint32_t *n_pressure_items, bool even, unsigned grid, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    PoolBCArgs<C> a;
    a.arena = arena;
    a.domains = static_cast<const PoolDomain<C> *>(domains);
    (void)grid;
    // persistent grids of exactly the resident blocks of each kernel: a grid one block per SM larger
    // than the registers allow runs as a second, mostly empty wave
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto resident = [sms](const void *fn) {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 128, 0) != cudaSuccess || occ < 1)
            occ = 1;
        return (unsigned)(occ * sms);
    };
    if (noslip_items && guard_items) {
        // the guarded values, saved before any no-slip write
        a.items = guard_items;
        a.n_items = n_guard_items;
        const void *g = even ? (const void *)pool_noslip_guard_kernel<S, true>
                             : (const void *)pool_noslip_guard_kernel<S, false>;
        if (even) pool_noslip_guard_kernel<S, true><<<resident(g), 128, 0, s>>>(a);
        else pool_noslip_guard_kernel<S, false><<<resident(g), 128, 0, s>>>(a);
    }
    if (noslip_items) {
        a.items = noslip_items;
        a.n_items = n_noslip_items;
        const void *k = even ? (const void *)pool_noslip_kernel<S, true> : (const void *)pool_noslip_kernel<S, false>;
        if (even) pool_noslip_kernel<S, true><<<resident(k), 128, 0, s>>>(a);
        else pool_noslip_kernel<S, false><<<resident(k), 128, 0, s>>>(a);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            return e;
    }
    if (pressure_items) {
        // after the parity swap
        a.items = pressure_items;
        a.n_items = n_pressure_items;
        const void *k = even ? (const void *)pool_pressure_kernel<S, false> : (const void *)pool_pressure_kernel<S, true>;
        if (even) pool_pressure_kernel<S, false><<<resident(k), 128, 0, s>>>(a);
        else pool_pressure_kernel<S, true><<<resident(k), 128, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::drag_lift(const vfb_level *L, const vfb_bc *bc, bool pre, double *dx, double *dy, double *dz,
                                    cudaStream_t s, const NodeAddr *box)
{
    if (bc->number_of_bc_nodes == 0)
        return cudaSuccess;
    DragArgs a;
    a.dist = L->distributions;
    a.n = L->number_of_nodes;
    a.nbx = box ? nullptr : L->neighbor_x;
    a.nby = box ? nullptr : L->neighbor_y;
    a.nbz = box ? nullptr : L->neighbor_z;
    a.box = box ? *box : NodeAddr{ 0, 0, 0, 0 };
    a.k = bc->k;
    a.q27 = bc->q27;
    a.nbc = bc->number_of_bc_nodes;
    a.dx = dx;
    a.dy = dy;
    a.dz = dz;
    const unsigned B = 128, G = grid1d(a.nbc, B);
    const bool even = L->is_even_timestep != 0;
    if (pre) {
        if (even) drag_lift_kernel<S, true, true><<<G, B, 0, s>>>(a);
        else drag_lift_kernel<S, false, true><<<G, B, 0, s>>>(a);
    } else {
        if (even) drag_lift_kernel<S, true, false><<<G, B, 0, s>>>(a);
        else drag_lift_kernel<S, false, false><<<G, B, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::scale(const vfb_level *coarse, const vfb_level *fine, const vfb_interpolation_cells *cells,
                                const vfb_interpolation_cell_neighbor *offsets, bool fine_to_coarse, cudaStream_t s)
{
    if (cells->number_of_cells == 0)
        return cudaSuccess;
    ScaleArgs a;
    a.dist_coarse = coarse->distributions;
    a.dist_fine = fine->distributions;
    a.n_coarse = coarse->number_of_nodes;
    a.n_fine = fine->number_of_nodes;
    a.nbx_c = coarse->neighbor_x;
    a.nby_c = coarse->neighbor_y;
    a.nbz_c = coarse->neighbor_z;
    a.nbx_f = fine->neighbor_x;
    a.nby_f = fine->neighbor_y;
    a.nbz_f = fine->neighbor_z;
    a.coarse_cells = cells->coarse_cell_indices;
    a.fine_cells = cells->fine_cell_indices;
    a.n_cells = cells->number_of_cells;
    a.ox = offsets->x;
    a.oy = offsets->y;
    a.oz = offsets->z;
    a.omega_coarse = coarse->omega;
    a.omega_fine = fine->omega;
    // eight lanes per cell
    const unsigned B = 128, G = grid1d((uint64_t)a.n_cells * 8u, B);
    const bool even = coarse->is_even_timestep != 0;
    if (fine_to_coarse) {
        if (even) scale_fc_kernel<S, true><<<G, B, 0, s>>>(a);
        else scale_fc_kernel<S, false><<<G, B, 0, s>>>(a);
    } else {
        if (even) scale_cf_kernel<S, true><<<G, B, 0, s>>>(a);
        else scale_cf_kernel<S, false><<<G, B, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::inlet_perturbation(const void *base, void *vel, uint32_t n, uint64_t seed, uint64_t step,
                                             double amplitude, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    if (n == 0)
        return cudaSuccess;
    const C *b = static_cast<const C *>(base);
    C *v = static_cast<C *>(vel);
    inlet_perturbation_kernel<C><<<grid1d(n, 256), 256, 0, s>>>(b, b + n, b + 2 * (uint64_t)n, v, v + n, v + 2 * (uint64_t)n,
                                                                n, seed, step, amplitude);
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::init_list(const vfb_level *L, cudaStream_t s)
{
    const unsigned B = 128, G = grid1d(L->number_of_nodes, B);
    if (L->is_even_timestep)
        init_list_kernel<S, true><<<G, B, 0, s>>>(L->distributions, L->number_of_nodes, L->neighbor_x, L->neighbor_y,
                                                  L->neighbor_z, L->type_of_grid_node, L->rho, L->velocity_x,
                                                  L->velocity_y, L->velocity_z);
    else
        init_list_kernel<S, false><<<G, B, 0, s>>>(L->distributions, L->number_of_nodes, L->neighbor_x, L->neighbor_y,
                                                   L->neighbor_z, L->type_of_grid_node, L->rho, L->velocity_x,
                                                   L->velocity_y, L->velocity_z);
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::init_neq_list(const vfb_level *L, const uint32_t *nb_inverse, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    const unsigned B = 128, G = grid1d(L->number_of_nodes, B);
    const C omega = (C)L->omega;
    if (L->is_even_timestep)
        init_neq_list_kernel<S, true><<<G, B, 0, s>>>(L->distributions, L->number_of_nodes, L->neighbor_x,
                                                      L->neighbor_y, L->neighbor_z, nb_inverse, L->type_of_grid_node,
                                                      L->rho, L->velocity_x, L->velocity_y, L->velocity_z, omega);
    else
        init_neq_list_kernel<S, false><<<G, B, 0, s>>>(L->distributions, L->number_of_nodes, L->neighbor_x,
                                                       L->neighbor_y, L->neighbor_z, nb_inverse, L->type_of_grid_node,
                                                       L->rho, L->velocity_x, L->velocity_y, L->velocity_z, omega);
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::macros_list(const vfb_level *L, cudaStream_t s)
{
    const unsigned B = 128, G = grid1d(L->number_of_nodes, B);
    if (L->is_even_timestep)
        macros_list_kernel<S, true><<<G, B, 0, s>>>(L->distributions, L->number_of_nodes, L->neighbor_x, L->neighbor_y,
                                                    L->neighbor_z, L->type_of_grid_node, L->rho, L->velocity_x,
                                                    L->velocity_y, L->velocity_z, L->pressure);
    else
        macros_list_kernel<S, false><<<G, B, 0, s>>>(L->distributions, L->number_of_nodes, L->neighbor_x, L->neighbor_y,
                                                     L->neighbor_z, L->type_of_grid_node, L->rho, L->velocity_x,
                                                     L->velocity_y, L->velocity_z, L->pressure);
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::energy_list(const vfb_level *L, const uint32_t *idx, uint32_t n, double *partials,
                                      cudaStream_t s)
{
    if (n == 0)
        return cudaSuccess;
    const unsigned B = 256, G = grid1d(n, B);
    if (L->is_even_timestep)
        energy_list_kernel<S, true><<<G, B, 0, s>>>(L->distributions, L->number_of_nodes, L->neighbor_x, L->neighbor_y,
                                                    L->neighbor_z, idx, n, partials);
    else
        energy_list_kernel<S, false><<<G, B, 0, s>>>(L->distributions, L->number_of_nodes, L->neighbor_x, L->neighbor_y,
                                                     L->neighbor_z, idx, n, partials);
    return cudaGetLastError();
}

namespace {
template <class C>
BoxCollideArgs<C> box_args(const BoxState &b)
{
    BoxCollideArgs<C> a;
    a.dist = b.dist;
    a.pitch = b.pitch;
    a.nx = b.nx;
    a.ny = b.ny;
    a.nz = b.nz;
    a.periodic_x = b.periodic_x;
    a.periodic_y = b.periodic_y;
    a.periodic_z = b.periodic_z;
    a.mask = b.mask;
    a.rates = rates_of<C>(b.omega, b.lim);
    a.fx = (C)b.fx;
    a.fy = (C)b.fy;
    a.fz = (C)b.fz;
    a.energy_partials = nullptr;
    a.rho = a.vx = a.vy = a.vz = nullptr;
    a.z_begin = 0;
    return a;
}
inline dim3 box_grid(const BoxState &b)
{
    const int bx = box_block_x(b.nx);
    return dim3((unsigned)((b.nx + bx - 1) / bx), (unsigned)b.ny, (unsigned)b.nz);
}
} // namespace

namespace {
int sm_count()
{
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    }
    return n;
}

// launch one TMA-staged instantiation: persistent grid sized by occupancy
template <class S, bool E, bool M, bool N>
cudaError_t launch_box_tma(const BoxCollideArgs<typename Codec<S>::compute> &a, int *status, uint64_t *n_partials,
                           cudaStream_t s)
{
    auto kern = k17_box_tma_kernel<S, VFB_EXACT, E, M, N>;
    static int blocks_per_sm = -1;
    if (blocks_per_sm < 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TmaTile<S>::SMEM);
        if (e != cudaSuccess)
            return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, 32 * TmaTile<S>::WARPS, TmaTile<S>::SMEM);
        if (e != cudaSuccess)
            return e;
        if (blocks_per_sm < 1)
            blocks_per_sm = 1;
    }
    const int64_t warp_tiles = (int64_t)(a.nx / TmaTile<S>::BX) * a.ny * a.nz;
    const int64_t blocks_needed = (warp_tiles + TmaTile<S>::WARPS - 1) / TmaTile<S>::WARPS;
    const int64_t grid = std::min<int64_t>(blocks_needed, (int64_t)blocks_per_sm * sm_count());
    kern<<<(unsigned)grid, 32 * TmaTile<S>::WARPS, TmaTile<S>::SMEM, s>>>(a, status);
    if (n_partials)
        *n_partials = (uint64_t)grid;
    return cudaGetLastError();
}
// Resident blocks per SM and the shared-memory configuration of the persistent async kernel.
// Every block holds 2 x 27 x 128 populations of staging (55 KB in F64). By default three blocks
// run per SM and the carve-out only hints at the configuration that holds three blocks' staging,
// leaving the rest to L1 (four blocks, possible when the compiler needs no more than 128
// registers, leave almost no L1). With an explicit configuration (smem_kb) each block pads its
// dynamic allocation to a share of it, so no more than the asked number of blocks can be resident
// whatever configuration the driver picks; the box autotuner chooses among such shapes.
constexpr int kAsyncBlocksPerSm = 3;

struct AsyncLaunchShape {
    int target_bps = -1, target_kb = -1;   // the request the cached shape was made for
    int blocks_per_sm = 0;
    int dyn_smem = 0;
};

template <class K>
cudaError_t async_launch_shape(K kern, size_t smem, int bps, int cfg_kb, AsyncLaunchShape &out)
{
    int dev = 0, max_smem = 0, reserved = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int dyn = (int)smem, cfg = bps * ((int)smem + reserved);
    if (cfg_kb > 0) {
        cfg = std::min(cfg_kb * 1024, max_smem);
        dyn = std::max((int)smem, (cfg / bps - reserved) & ~127);
        if (optin > 0)
            dyn = std::min(dyn, optin);
    }
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (e != cudaSuccess)
        return e;
    if (max_smem > 0)
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                             std::min(100, (cfg * 100 + max_smem - 1) / max_smem));
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 128, dyn);
    if (e != cudaSuccess)
        return e;
    out.blocks_per_sm = std::max(1, std::min(occ, bps));
    out.dyn_smem = dyn;
    return cudaSuccess;
}

template <class S, bool E, bool M, bool N>
cudaError_t launch_box_async(const BoxCollideArgs<typename Codec<S>::compute> &a, int bps, int cfg_kb,
                             uint64_t *n_partials, cudaStream_t s)
{
    auto kern = k17_box_async_kernel<S, VFB_EXACT, E, M, N>;
    static AsyncLaunchShape shape;
    if (bps <= 0)
        bps = kAsyncBlocksPerSm;
    if (shape.target_bps != bps || shape.target_kb != cfg_kb) {
        AsyncLaunchShape sh;
        const cudaError_t e = async_launch_shape(kern, AsyncTile<S>::SMEM, bps, cfg_kb, sh);
        if (e != cudaSuccess)
            return e;
        sh.target_bps = bps;
        sh.target_kb = cfg_kb;
        shape = sh;
    }
    const int64_t ntiles = (int64_t)((a.nx + AsyncTile<S>::BX - 1) / AsyncTile<S>::BX) * a.ny * a.nz;
    const int64_t grid = std::min<int64_t>(ntiles, (int64_t)shape.blocks_per_sm * sm_count());
    kern<<<(unsigned)grid, 128, shape.dyn_smem, s>>>(a);
    if (n_partials)
        *n_partials = (uint64_t)grid;
    return cudaGetLastError();
}

// the software-pipelined persistent box kernel: as many blocks as stay resident, each walking
// rows of box_block_x(nx) nodes
template <class S, bool E, bool M, bool N>
cudaError_t launch_box_pipe(const BoxCollideArgs<typename Codec<S>::compute> &a, uint64_t *n_partials, cudaStream_t s)
{
    auto kern = k17_box_pipe_kernel<S, VFB_EXACT, E, M, N>;
    const int B = box_block_x(a.nx);
    static int cached_block = -1, cached_bps = 0;
    if (cached_block != B) {
        int bps = 0;
        const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, B, 0);
        if (e != cudaSuccess)
            return e;
        cached_bps = bps > 0 ? bps : 1;
        cached_block = B;
    }
    const int64_t ntiles = (int64_t)((a.nx + B - 1) / B) * a.ny * a.nz;
    const int64_t grid = std::min<int64_t>(ntiles, (int64_t)cached_bps * sm_count());
    kern<<<(unsigned)grid, (unsigned)B, 0, s>>>(a);
    if (n_partials)
        *n_partials = (uint64_t)grid * (uint64_t)(B / 32);
    return cudaGetLastError();
}
} // namespace

template <class S>
cudaError_t Launchers<S>::box_collide(const BoxState &b, bool even, double *partials, uint64_t *n_partials, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    BoxCollideArgs<C> a = box_args<C>(b);
    a.energy_partials = partials;
    const bool mask = b.mask != nullptr, energy = partials != nullptr;
    if constexpr (sizeof(S) >= 4) {
        if (b.variant == 3) {
#define VFB_K17A(E, M, N) return launch_box_async<S, E, M, N>(a, b.async_blocks_per_sm, b.async_smem_kb, n_partials, s)
        if (even) {
            if (mask && energy) VFB_K17A(true, true, true);
            else if (mask) VFB_K17A(true, true, false);
            else if (energy) VFB_K17A(true, false, true);
            else VFB_K17A(true, false, false);
        } else {
            if (mask && energy) VFB_K17A(false, true, true);
            else if (mask) VFB_K17A(false, true, false);
            else if (energy) VFB_K17A(false, false, true);
            else VFB_K17A(false, false, false);
        }
#undef VFB_K17A
        }
    }
    if (b.variant == 5) {
#define VFB_K17Q(E, M, N) return launch_box_pipe<S, E, M, N>(a, n_partials, s)
        if (even) {
            if (mask && energy) VFB_K17Q(true, true, true);
            else if (mask) VFB_K17Q(true, true, false);
            else if (energy) VFB_K17Q(true, false, true);
            else VFB_K17Q(true, false, false);
        } else {
            if (mask && energy) VFB_K17Q(false, true, true);
            else if (mask) VFB_K17Q(false, true, false);
            else if (energy) VFB_K17Q(false, false, true);
            else VFB_K17Q(false, false, false);
        }
#undef VFB_K17Q
    }
    if constexpr (std::is_same<C, float>::value && !VFB_EXACT) {
        if (b.variant == 4) {
            // two rows per block row of the grid, packed FP32x2 arithmetic
            const int bx = box_block_x(b.nx);
            const dim3 G((unsigned)((b.nx + bx - 1) / bx), (unsigned)((b.ny + 1) / 2), (unsigned)b.nz), B(bx);
            if (n_partials)
                *n_partials = (uint64_t)G.x * G.y * G.z * (B.x / 32);
#define VFB_K17P(E, M, N) k17_box_pair_kernel<S, E, M, N><<<G, B, 0, s>>>(a)
            if (even) {
                if (mask && energy) VFB_K17P(true, true, true);
                else if (mask) VFB_K17P(true, true, false);
                else if (energy) VFB_K17P(true, false, true);
                else VFB_K17P(true, false, false);
            } else {
                if (mask && energy) VFB_K17P(false, true, true);
                else if (mask) VFB_K17P(false, true, false);
                else if (energy) VFB_K17P(false, false, true);
                else VFB_K17P(false, false, false);
            }
#undef VFB_K17P
            return cudaGetLastError();
        }
    }
    const bool tma = b.variant == 2 && (b.nx % TmaTile<S>::BX) == 0 && b.status != nullptr;
    if (tma) {
#define VFB_K17T(E, M, N) return launch_box_tma<S, E, M, N>(a, b.status, n_partials, s)
        if (even) {
            if (mask && energy) VFB_K17T(true, true, true);
            else if (mask) VFB_K17T(true, true, false);
            else if (energy) VFB_K17T(true, false, true);
            else VFB_K17T(true, false, false);
        } else {
            if (mask && energy) VFB_K17T(false, true, true);
            else if (mask) VFB_K17T(false, true, false);
            else if (energy) VFB_K17T(false, false, true);
            else VFB_K17T(false, false, false);
        }
#undef VFB_K17T
    }
    const dim3 G = box_grid(b), B(box_block_x(b.nx));
    if (n_partials)
        *n_partials = (uint64_t)G.x * G.y * G.z * (B.x / 32);
#define VFB_K17B(E, M, N) k17_box_kernel<S, VFB_EXACT, E, M, N, false><<<G, B, 0, s>>>(a)
    if (even) {
        if (mask && energy) VFB_K17B(true, true, true);
        else if (mask) VFB_K17B(true, true, false);
        else if (energy) VFB_K17B(true, false, true);
        else VFB_K17B(true, false, false);
    } else {
        if (mask && energy) VFB_K17B(false, true, true);
        else if (mask) VFB_K17B(false, true, false);
        else if (energy) VFB_K17B(false, false, true);
        else VFB_K17B(false, false, false);
    }
#undef VFB_K17B
    return cudaGetLastError();
}

// the bounds record of this translation unit's kernels (bounds-checked build), read and cleared;
// 0 in the default build
template <class S>
cudaError_t Launchers<S>::bounds_error(uint64_t *record)
{
#ifdef VFB_BOUNDS_CHECK
    unsigned long long v = 0, zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_bounds_error, sizeof(v));
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbol(g_bounds_error, &zero, sizeof(zero));
    *record = v;
    return e;
#else
    *record = 0;
    return cudaSuccess;
#endif
}

// the direct collision kernel over the planes [z0, z1) only (no energy, no macroscopic output): a
// time step split into parts, e.g. the border planes of a slab before its interior
template <class S>
cudaError_t Launchers<S>::box_collide_planes(const BoxState &b, bool even, int z0, int z1, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    if (z1 <= z0)
        return cudaSuccess;
    BoxCollideArgs<C> a = box_args<C>(b);
    a.z_begin = z0;
    dim3 G = box_grid(b);
    G.z = (unsigned)(z1 - z0);
    const dim3 B(box_block_x(b.nx));
    const bool mask = b.mask != nullptr;
    if (even) {
        if (mask) k17_box_kernel<S, VFB_EXACT, true, true, false, false><<<G, B, 0, s>>>(a);
        else k17_box_kernel<S, VFB_EXACT, true, false, false, false><<<G, B, 0, s>>>(a);
    } else {
        if (mask) k17_box_kernel<S, VFB_EXACT, false, true, false, false><<<G, B, 0, s>>>(a);
        else k17_box_kernel<S, VFB_EXACT, false, false, false, false><<<G, B, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::box_collide_border(const BoxState &b, bool even, int z, void *up, void *down, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    BoxCollideArgs<C> a = box_args<C>(b);
    dim3 G = box_grid(b);
    G.z = 1;
    const dim3 B(box_block_x(b.nx));
    S *u = static_cast<S *>(up), *d = static_cast<S *>(down);
    const bool mask = b.mask != nullptr;
    if (even) {
        if (mask) k17_box_border_kernel<S, VFB_EXACT, true, true><<<G, B, 0, s>>>(a, z, u, d);
        else k17_box_border_kernel<S, VFB_EXACT, true, false><<<G, B, 0, s>>>(a, z, u, d);
    } else {
        if (mask) k17_box_border_kernel<S, VFB_EXACT, false, true><<<G, B, 0, s>>>(a, z, u, d);
        else k17_box_border_kernel<S, VFB_EXACT, false, false><<<G, B, 0, s>>>(a, z, u, d);
    }
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::box_init(const BoxState &b, bool even, const void *rho, const void *ux, const void *uy,
                                   const void *uz, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    BoxCollideArgs<C> a = box_args<C>(b);
    const dim3 G = box_grid(b), B(box_block_x(b.nx));
    if (even) init_box_kernel<S, true><<<G, B, 0, s>>>(a, rho, ux, uy, uz);
    else init_box_kernel<S, false><<<G, B, 0, s>>>(a, rho, ux, uy, uz);
    return cudaGetLastError();
}

template <class S>
cudaError_t Launchers<S>::box_macros(const BoxState &b, bool even, void *rho, void *ux, void *uy, void *uz, cudaStream_t s)
{
    using C = typename Codec<S>::compute;
    BoxCollideArgs<C> a = box_args<C>(b);
    a.rho = static_cast<C *>(rho);
    a.vx = static_cast<C *>(ux);
    a.vy = static_cast<C *>(uy);
    a.vz = static_cast<C *>(uz);
    const dim3 G = box_grid(b), B(box_block_x(b.nx));
    if (even) macros_box_kernel<S, true><<<G, B, 0, s>>>(a);
    else macros_box_kernel<S, false><<<G, B, 0, s>>>(a);
    return cudaGetLastError();
}

} // namespace VFB_NS
} // namespace vfb
