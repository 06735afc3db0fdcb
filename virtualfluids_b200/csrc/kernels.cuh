// Device kernels of the time step, templated over storage type, parity and features.
//
// This header is compiled twice into the library: once with contraction off (-fmad=false,
// namespace vfb::exact) and once with the default FMA contraction (namespace vfb::fast). The
// first reproduces the reference's operation-by-operation rounding; the second is the default.
//
// Every direction loop is fully unrolled, so direction-dependent constants (plane, shift class,
// weight, inverse) fold and the 27 populations stay in registers.
#pragma once
#include <cstdint>

#include "addr.h"
#include "interp.cuh"
#include "k17.cuh"
#include "packed.cuh"
#include "storage.cuh"
#include "tma.cuh"

#ifndef VFB_NS
#error "VFB_NS must name the compilation variant"
#endif

namespace vfb {
namespace VFB_NS {

// ---------------------------------------------------------------------------------------------
// Bounds-checked build (-DVFB_BOUNDS_CHECK, libvfb_checked.so): every node index a kernel takes
// from a caller's array (fluid-node lists, neighbour lists, BC node lists, interpolation cells,
// slot tables) is compared with the node count of its level before it is used. An index out of
// range is recorded -- the first one since the last read, as (bound << 32) | (index + 1) -- and
// replaced by the dummy node 0, so no access leaves the arrays; the host reads the record with
// vfb_bounds_check_status. In the default build VFB_NODE is the index itself.
// ---------------------------------------------------------------------------------------------
#ifdef VFB_BOUNDS_CHECK
static __device__ unsigned long long g_bounds_error;
__device__ __forceinline__ uint32_t checked_node(uint32_t v, uint64_t n)
{
    if ((uint64_t)v < n)
        return v;
    atomicCAS(&g_bounds_error, 0ull, ((unsigned long long)(n & 0xffffffffull) << 32) | ((unsigned long long)v + 1ull));
    return 0u;
}
#define VFB_NODE(v, n) checked_node((v), (n))
#else
#define VFB_NODE(v, n) (v)
#endif

// ---------------------------------------------------------------------------------------------
// argument packs
// ---------------------------------------------------------------------------------------------
template <class C>
struct ListCollideArgs {
    void *dist;                 // distributions.f[0]
    uint64_t n;                 // numberOfNodes (plane stride)
    const uint32_t *nbx, *nby, *nbz;
    const uint32_t *idx;        // fluid node indices
    uint32_t n_idx;
    const uint32_t *slots;      // optional slot table: node j (0 = idx[i], then the seven +1
    uint64_t slots_stride;      //   neighbours) of entry i at slots[j * slots_stride + i]
    K17Rates<C> rates;
    C fx, fy, fz;               // forces * 1/2 * 2^-level (RunCollision.cuh:112-114)
    C force0, force1, force2;   // forces, for the body-force variant
    C force_factor;             // 2^-level
    C *bfx, *bfy, *bfz;         // per-node body force (reset after use)
    C *rho, *vx, *vy, *vz;      // macroscopic outputs
};

template <class C>
struct BoxCollideArgs {
    void *dist;                 // 27 planes of `pitch` elements, node k = x + nx (y + ny z)
    uint64_t pitch;
    int nx, ny, nz;
    int periodic_x, periodic_y, periodic_z;
    const uint8_t *mask;        // optional: nonzero = collide (fluid); nullptr = every node
    K17Rates<C> rates;
    C fx, fy, fz;
    double *energy_partials;    // optional: per block {sum(1+drho), sum(0.5 (1+drho) u^2)}
    C *rho, *vx, *vy, *vz;      // optional macroscopic outputs
    int z_begin;                // the direct kernel collides planes z_begin + blockIdx.z (0: the whole box)
};

// where a node's eight slot nodes are: from the neighbour lists (reference layout), or, when
// nbx is null, by index arithmetic on the structured box `box`

struct BCArgs {
    void *dist;
    uint64_t n;                 // plane stride
    const uint32_t *nbx, *nby, *nbz;
    NodeAddr box;
    const int32_t *k;           // BC node indices
    const void *q27;            // q27[dir * nbc + i], compute type
    uint32_t nbc;
    const void *ux, *uy, *uz;   // wall / inlet velocity per BC node, compute type
    double omega;
    const void *snap;           // optional: the list's post-collision populations taken before any BC
                                // write, snap[d * nbc + i] (compute type); read instead of the slots
    const uint32_t *guard;      // optional guard table (guards.h): mask[i], then first[nbc + i]
    const void *saved;          // the guarded values, saved before the list's writes (compute type)
};

struct PressureArgs {
    void *dist;
    uint64_t n;
    const uint32_t *nbx, *nby, *nbz;
    NodeAddr box;
    const int32_t *k, *kN;
    const void *rho_bc;
    uint32_t nbc;
    int direction;
};

// ---------------------------------------------------------------------------------------------
// addressing
// ---------------------------------------------------------------------------------------------

// ListIndices (KernelUtilities.h:221-250) by shift class: bit0 x+1, bit1 y+1, bit2 z+1
// (n: node count of the level, the bound of the bounds-checked build)
__device__ __forceinline__ void list_nodes(uint32_t k, const uint32_t *__restrict__ nbx, const uint32_t *__restrict__ nby,
                                           const uint32_t *__restrict__ nbz, uint64_t n, uint32_t (&nodes)[8])
{
    (void)n;
    k = VFB_NODE(k, n);
    const uint32_t kx = VFB_NODE(__ldg(nbx + k), n), ky = VFB_NODE(__ldg(nby + k), n), kz = VFB_NODE(__ldg(nbz + k), n);
    const uint32_t kxy = VFB_NODE(__ldg(nby + kx), n);
    nodes[0] = k;
    nodes[1] = kx;
    nodes[2] = ky;
    nodes[3] = kxy;
    nodes[4] = kz;
    nodes[5] = VFB_NODE(__ldg(nbz + kx), n);
    nodes[6] = VFB_NODE(__ldg(nbz + ky), n);
    nodes[7] = VFB_NODE(__ldg(nbz + kxy), n);
}

// the eight slot nodes of a node on a structured box
__device__ __forceinline__ void box_nodes_at(uint32_t k, uint32_t x, uint32_t y, uint32_t z, const NodeAddr &b,
                                             uint32_t (&nodes)[8])
{
    const int xp = ((int)x + 1 < b.nx) ? (int)x + 1 : ((b.periodic & 1) ? 0 : (int)x);
    const int yp = ((int)y + 1 < b.ny) ? (int)y + 1 : ((b.periodic & 2) ? 0 : (int)y);
    const int zp = ((int)z + 1 < b.nz) ? (int)z + 1 : ((b.periodic & 4) ? 0 : (int)z);
    const uint32_t sx = (uint32_t)(xp - (int)x);
    const uint32_t sy = (uint32_t)((yp - (int)y) * b.nx);
    const uint32_t sz = (uint32_t)((int64_t)(zp - (int)z) * b.nx * b.ny);
    nodes[0] = k;
    nodes[1] = k + sx;
    nodes[2] = k + sy;
    nodes[3] = k + sx + sy;
    nodes[4] = k + sz;
    nodes[5] = k + sx + sz;
    nodes[6] = k + sy + sz;
    nodes[7] = k + sx + sy + sz;
}

__device__ __forceinline__ void box_nodes(uint32_t k, const NodeAddr &b, uint32_t (&nodes)[8])
{
    k = VFB_NODE(k, (uint64_t)b.nx * (uint64_t)b.ny * (uint64_t)b.nz);
    const uint32_t x = k % (uint32_t)b.nx, yz = k / (uint32_t)b.nx;
    const uint32_t y = yz % (uint32_t)b.ny, z = yz / (uint32_t)b.ny;
    box_nodes_at(k, x, y, z, b, nodes);
}

// the same with the divisions by nx and ny as multiply-shifts (k < 2^31)
__device__ __forceinline__ void box_nodes(uint32_t k, const NodeAddr &b, FastDiv div_nx, FastDiv div_ny,
                                          uint32_t (&nodes)[8])
{
    k = VFB_NODE(k, (uint64_t)b.nx * (uint64_t)b.ny * (uint64_t)b.nz);
    const uint32_t yz = fast_div(k, div_nx), x = k - yz * (uint32_t)b.nx;
    const uint32_t z = fast_div(yz, div_ny), y = yz - z * (uint32_t)b.ny;
    box_nodes_at(k, x, y, z, b, nodes);
}

__device__ __forceinline__ void node_slots(uint32_t k, const uint32_t *nbx, const uint32_t *nby, const uint32_t *nbz,
                                           uint64_t n, const NodeAddr &b, uint32_t (&nodes)[8])
{
    if (nbx)
        list_nodes(k, nbx, nby, nbz, n, nodes);
    else
        box_nodes(k, b, nodes);
}

template <class S, bool EVEN>
__device__ __forceinline__ void gather_pre(const S *__restrict__ base, uint64_t n, const uint32_t (&nodes)[8],
                                           typename Codec<S>::compute (&f)[27])
{
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = Codec<S>::load(base + (uint64_t)plane<EVEN>(d) * n + nodes[shift_class(d)], d);
}

// setPostCollisionDistribution (KernelUtilities.h:350): the slot of d receives f[inv d]
template <class S, bool EVEN>
__device__ __forceinline__ void scatter_post(S *__restrict__ base, uint64_t n, const uint32_t (&nodes)[8],
                                             const typename Codec<S>::compute (&f)[27])
{
    if constexpr (Codec<S>::kPairs) {
        // 16-bit storage: two directions share one stochastic-rounding conversion
#pragma unroll
        for (int d = 0; d + 1 < 27; d += 2)
            Codec<S>::store_pair_at(base, (uint64_t)plane<EVEN>(d) * n + nodes[shift_class(d)], f[inv(d)], d,
                                    (uint64_t)plane<EVEN>(d + 1) * n + nodes[shift_class(d + 1)], f[inv(d + 1)], d + 1);
        Codec<S>::store_at(base, (uint64_t)plane<EVEN>(26) * n + nodes[shift_class(26)], f[inv(26)], 26);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d)
            Codec<S>::store_at(base, (uint64_t)plane<EVEN>(d) * n + nodes[shift_class(d)], f[inv(d)], d);
    }
}

// getPostCollisionDistribution (KernelUtilities.h:283): post[d] leaves the node along d
template <class S, bool EVEN>
__device__ __forceinline__ void gather_post(const S *base, uint64_t n, const uint32_t (&nodes)[8],
                                            typename Codec<S>::compute (&post)[27])
{
#pragma unroll
    for (int d = 0; d < 27; ++d)
        post[d] = Codec<S>::load(base + (uint64_t)plane<EVEN>(inv(d)) * n + nodes[shift_class(inv(d))], d);
}

// ---------------------------------------------------------------------------------------------
// collision + streaming, reference layout (RunCollision.cuh:75-143)
// ---------------------------------------------------------------------------------------------
template <class S, bool EXACT, bool EVEN, bool WRITE_MACRO, bool BODY_FORCE>
__global__ void __launch_bounds__(128) k17_list_kernel(ListCollideArgs<typename Codec<S>::compute> a)
{
    using C = typename Codec<S>::compute;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_idx)
        return;
    const uint32_t k = VFB_NODE(__ldg(a.idx + i), a.n);
    C fx = a.fx, fy = a.fy, fz = a.fz;
    if (BODY_FORCE) {
        fx = (a.force0 + a.bfx[k]) * C(0.5) * a.force_factor;
        fy = (a.force1 + a.bfy[k]) * C(0.5) * a.force_factor;
        fz = (a.force2 + a.bfz[k]) * C(0.5) * a.force_factor;
        a.bfx[k] = C(0);
        a.bfy[k] = C(0);
        a.bfz[k] = C(0);
    }
    uint32_t nodes[8];
    if (a.slots) {
        // slot table built once per level: one coalesced load per slot, no dependent chain
        nodes[0] = k;
#pragma unroll
        for (int j = 1; j < 8; ++j)
            nodes[j] = VFB_NODE(__ldg(a.slots + (size_t)j * a.slots_stride + i), a.n);
    } else {
        list_nodes(k, a.nbx, a.nby, a.nbz, a.n, nodes);
    }
    S *base = static_cast<S *>(a.dist);
    C f[27];
    gather_pre<S, EVEN>(base, a.n, nodes, f);
    C drho, vx, vy, vz;
    collide<C, EXACT>(f, a.rates, fx, fy, fz, drho, vx, vy, vz);
    if (WRITE_MACRO) {
        a.vx[k] = vx;
        a.vy[k] = vy;
        a.vz[k] = vz;
        a.rho[k] = drho;
    }
    scatter_post<S, EVEN>(base, a.n, nodes, f);
}

// ---------------------------------------------------------------------------------------------
// The same collision over the reference layout with the slot table staged in shared memory: every
// warp walks tiles of 32 list entries and keeps the eight node indices of its next two tiles in
// flight as bulk asynchronous copies (TMA, one 128-byte copy per slot array, counted on a per-warp
// mbarrier), so the population loads of a tile never wait for its indices. The table's arrays
// have a stride that is a multiple of 32 entries (16-byte aligned tiles); entries past n_idx are
// read but not computed. Waits are bounded: a copy that never lands sets *status and ends the warp.
// ---------------------------------------------------------------------------------------------
struct ListTile {
    static constexpr int N = 32;                  // entries per warp tile
    static constexpr int WARPS = 4;
    static constexpr int STAGES = 2;
    static constexpr uint32_t STAGE_WORDS = 8u * N;
    static constexpr size_t SMEM = WARPS * (STAGES * STAGE_WORDS * sizeof(uint32_t) + STAGES * sizeof(uint64_t));
};

__device__ __forceinline__ void list_issue_tile(const uint32_t *slots, uint64_t stride, int64_t t, uint32_t *stage,
                                                uint64_t *bar, int lane)
{
    if (lane == 0)
        mbar_arrive_expect_tx(bar, 8u * ListTile::N * (uint32_t)sizeof(uint32_t));
    __syncwarp();
    if (lane < 8)
        bulk_copy_g2s(stage + lane * ListTile::N, slots + (uint64_t)lane * stride + (uint64_t)t * ListTile::N,
                      ListTile::N * (uint32_t)sizeof(uint32_t), bar);
}

template <class S, bool EXACT, bool EVEN>
__global__ void __launch_bounds__(128) k17_list_staged_kernel(ListCollideArgs<typename Codec<S>::compute> a, int *status)
{
    using C = typename Codec<S>::compute;
    using T = ListTile;
    __shared__ __align__(128) uint32_t tiles[T::WARPS][T::STAGES][T::STAGE_WORDS];
    __shared__ __align__(8) uint64_t bars[T::WARPS][T::STAGES];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t *bar = bars[warp];
    const int64_t ntiles = ((int64_t)a.n_idx + T::N - 1) / T::N;
    const int64_t first = (int64_t)blockIdx.x * T::WARPS + warp;
    const int64_t stride = (int64_t)gridDim.x * T::WARPS;
    if (lane == 0) {
        for (int s = 0; s < T::STAGES; ++s)
            mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncwarp();
    for (int s = 0; s < T::STAGES; ++s) {
        const int64_t t = first + s * stride;
        if (t < ntiles)
            list_issue_tile(a.slots, a.slots_stride, t, tiles[warp][s], &bar[s], lane);
    }
    S *base = static_cast<S *>(a.dist);
    uint32_t parity = 0;
    bool failed = false;
    int it = 0;
    for (int64_t t = first; t < ntiles; t += stride, ++it) {
        const int s = it & 1;
        const bool ok = mbar_wait(&bar[s], (parity >> s) & 1u);
        if (__any_sync(0xffffffffu, !ok)) {
            failed = true;
            break;
        }
        parity ^= 1u << s;
        const uint32_t *tile = tiles[warp][s];
        uint32_t nodes[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            nodes[j] = tile[j * T::N + lane];
        // the warp is done reading the stage: order the reads before the next copies into it
        fence_proxy_async_smem();
        __syncwarp();
        const int64_t tn = t + (int64_t)T::STAGES * stride;
        if (tn < ntiles)
            list_issue_tile(a.slots, a.slots_stride, tn, tiles[warp][s], &bar[s], lane);
        if ((uint64_t)t * T::N + lane < a.n_idx) {
            C f[27];
            gather_pre<S, EVEN>(base, a.n, nodes, f);
            C drho, vx, vy, vz;
            collide<C, EXACT>(f, a.rates, a.fx, a.fy, a.fz, drho, vx, vy, vz);
            scatter_post<S, EVEN>(base, a.n, nodes, f);
        }
    }
    if (failed) {
        if (lane == 0) {
            atomicExch(status, (int)kDevWaitTimeout);
            // let copies still in flight land before the block's shared memory is released
            for (int s = 0; s < T::STAGES; ++s)
                mbar_wait(&bar[s], (parity >> s) & 1u, 1u << 16);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------------
// collision + streaming on a structured box: neighbours by index arithmetic, one node per
// thread, x fastest so every direction plane is read and written by whole warps in order.
// ---------------------------------------------------------------------------------------------
// resident blocks per SM the register budget must allow: three for FP64 arithmetic (at most 168
// registers; an unbounded build of the exact energy variant takes 170, which rounds to 176 and
// leaves two), four for FP32 arithmetic (at most 128)
template <class S>
constexpr int box_min_blocks() { return sizeof(typename Codec<S>::compute) == 8 ? 3 : 4; }

template <class S, bool EXACT, bool EVEN, bool MASK, bool ENERGY, bool WRITE_MACRO>
__global__ void __launch_bounds__(128, box_min_blocks<S>()) k17_box_kernel(BoxCollideArgs<typename Codec<S>::compute> a)
{
    using C = typename Codec<S>::compute;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z + a.z_begin;
    const bool active_x = x < a.nx;
    const uint64_t row = (uint64_t)a.nx * ((uint64_t)y + (uint64_t)a.ny * (uint64_t)z);
    const uint32_t k = (uint32_t)(row + (uint64_t)x);
    bool active = active_x;
    if (MASK && active)
        active = __ldg(a.mask + k) != 0;

    C drho = C(0), vx = C(0), vy = C(0), vz = C(0);
    if (active) {
        // +1 neighbours, wrapping on periodic axes (the mask keeps walled boxes inside)
        const int xp = (x + 1 < a.nx) ? x + 1 : (a.periodic_x ? 0 : x);
        const int yp = (y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y);
        const int zp = (z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z);
        const uint32_t sx = (uint32_t)(xp - x);
        const uint32_t sy = (uint32_t)((yp - y) * a.nx);
        const uint32_t sz = (uint32_t)((int64_t)(zp - z) * a.nx * a.ny);
        uint32_t nodes[8];
        nodes[0] = k;
        nodes[1] = k + sx;
        nodes[2] = k + sy;
        nodes[3] = k + sx + sy;
        nodes[4] = k + sz;
        nodes[5] = k + sx + sz;
        nodes[6] = k + sy + sz;
        nodes[7] = k + sx + sy + sz;
        S *base = static_cast<S *>(a.dist);
        C f[27];
        gather_pre<S, EVEN>(base, a.pitch, nodes, f);
        collide<C, EXACT>(f, a.rates, a.fx, a.fy, a.fz, drho, vx, vy, vz);
        if (WRITE_MACRO) {
            a.rho[k] = drho;
            a.vx[k] = vx;
            a.vy[k] = vy;
            a.vz[k] = vz;
        }
        scatter_post<S, EVEN>(base, a.pitch, nodes, f);
    }

    if (ENERGY) {
        // FP64 partials of mass and kinetic energy per warp (fixed reduction order, no block barrier,
        // so the warps of a block retire independently)
        double m = active ? 1.0 + (double)drho : 0.0;
        double e = active ? 0.5 * (1.0 + (double)drho) * ((double)vx * vx + (double)vy * vy + (double)vz * vz) : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m += __shfl_down_sync(0xffffffffu, m, o);
            e += __shfl_down_sync(0xffffffffu, e, o);
        }
        if ((threadIdx.x & 31) == 0) {
            const uint64_t b = blockIdx.x + (uint64_t)gridDim.x * (blockIdx.y + (uint64_t)gridDim.y * blockIdx.z);
            const uint64_t w = b * (blockDim.x >> 5) + (threadIdx.x >> 5);
            a.energy_partials[2 * w] = m;
            a.energy_partials[2 * w + 1] = e;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// One z plane of a box that is a slab of a larger domain, whose neighbouring slabs live in other
// population arrays of the same shape (on this GPU, or on another through a peer mapping): the
// collision of k17_box_kernel, with the stores that belong to a neighbour made straight into the
// neighbour's array, so that no exchange step follows.
//   up   : the slots this plane writes in plane z + 1 (directions with a negative z component at
//          this parity) go to plane 0 of `up` (the slab above, whose bottom layer reads them);
//   down : the slots this plane writes in its own plane for directions with a positive z
//          component go to the last plane of `down` (the slab below's ghost plane, read by its top
//          layer).
// Either may be null (the store stays local). In the esoteric twist no node of the receiving slab
// touches those slots in the same step, so the stores need no ordering against the neighbour's
// kernels of that step; the caller orders the steps (a barrier between them).
// ---------------------------------------------------------------------------------------------
template <class S, bool EXACT, bool EVEN, bool MASK>
__global__ void __launch_bounds__(128, box_min_blocks<S>())
    k17_box_border_kernel(BoxCollideArgs<typename Codec<S>::compute> a, int z, S *up, S *down)
{
    using C = typename Codec<S>::compute;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= a.nx)
        return;
    const uint64_t plane_nodes = (uint64_t)a.nx * (uint64_t)a.ny;
    const uint32_t k = (uint32_t)(plane_nodes * (uint64_t)z + (uint64_t)a.nx * (uint64_t)y + (uint64_t)x);
    if (MASK && __ldg(a.mask + k) == 0)
        return;
    const int xp = (x + 1 < a.nx) ? x + 1 : (a.periodic_x ? 0 : x);
    const int yp = (y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y);
    const int zp = (z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z);
    const uint32_t sx = (uint32_t)(xp - x);
    const uint32_t sy = (uint32_t)((yp - y) * a.nx);
    const uint32_t sz = (uint32_t)((int64_t)(zp - z) * a.nx * a.ny);
    uint32_t nodes[8];
    nodes[0] = k;
    nodes[1] = k + sx;
    nodes[2] = k + sy;
    nodes[3] = k + sx + sy;
    nodes[4] = k + sz;
    nodes[5] = k + sx + sz;
    nodes[6] = k + sy + sz;
    nodes[7] = k + sx + sy + sz;
    S *base = static_cast<S *>(a.dist);
    C f[27];
    gather_pre<S, EVEN>(base, a.pitch, nodes, f);
    C drho, vx, vy, vz;
    collide<C, EXACT>(f, a.rates, a.fx, a.fy, a.fz, drho, vx, vy, vz);
    const uint64_t up_shift = plane_nodes * (uint64_t)(z + 1);                 // plane z + 1 -> plane 0
    const uint64_t down_shift = plane_nodes * (uint64_t)(a.nz - 1 - z);        // plane z -> last plane
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const uint64_t off = (uint64_t)plane<EVEN>(d) * a.pitch + nodes[shift_class(d)];
        if (cz(d) < 0 && up != nullptr)
            Codec<S>::store_at(up, off - up_shift, f[inv(d)], d);
        else if (cz(d) > 0 && down != nullptr)
            Codec<S>::store_at(down, off + down_shift, f[inv(d)], d);
        else
            Codec<S>::store_at(base, off, f[inv(d)], d);
    }
    // stores into another GPU's memory are made visible at system scope before the kernel ends, so
    // the barrier that follows (an NCCL all-reduce) orders them for the neighbour
    if (up != nullptr || down != nullptr)
        __threadfence_system();
}

// ---------------------------------------------------------------------------------------------
// The box collision as a persistent, software-pipelined loop. A block walks rows of blockDim.x
// nodes along x (tile t = (x tile, y, z)); before a thread collides and stores its node of the
// current tile it issues the 27 loads of its node in the next tile into registers, so the loads of
// one tile are in flight while the arithmetic of the one before runs. Reading the next tile's slots
// before the current tile's stores is safe: in esoteric-twist streaming every slot is read and
// written by exactly one node per step. The energy partials are per warp over all of its tiles (a
// fixed order for a fixed grid).
// ---------------------------------------------------------------------------------------------
template <class S>
constexpr int pipe_min_blocks() { return sizeof(typename Codec<S>::compute) == 8 ? 2 : 3; }

template <class C>
__device__ __forceinline__ bool pipe_node(const BoxCollideArgs<C> &a, uint32_t tiles_x, int64_t t, uint32_t (&nodes)[8])
{
    const uint32_t tt = (uint32_t)t;
    const uint32_t row = tt / tiles_x;
    const int x = (int)((tt - row * tiles_x) * blockDim.x + threadIdx.x);
    const int y = (int)(row % (uint32_t)a.ny), z = (int)(row / (uint32_t)a.ny);
    if (x >= a.nx)
        return false;
    const int xp = (x + 1 < a.nx) ? x + 1 : (a.periodic_x ? 0 : x);
    const int yp = (y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y);
    const int zp = (z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z);
    const uint32_t k = (uint32_t)((uint64_t)a.nx * ((uint64_t)y + (uint64_t)a.ny * (uint64_t)z) + (uint64_t)x);
    const uint32_t sx = (uint32_t)(xp - x);
    const uint32_t sy = (uint32_t)((yp - y) * a.nx);
    const uint32_t sz = (uint32_t)((int64_t)(zp - z) * a.nx * a.ny);
    nodes[0] = k;
    nodes[1] = k + sx;
    nodes[2] = k + sy;
    nodes[3] = k + sx + sy;
    nodes[4] = k + sz;
    nodes[5] = k + sx + sz;
    nodes[6] = k + sy + sz;
    nodes[7] = k + sx + sy + sz;
    return true;
}

template <class S, bool EXACT, bool EVEN, bool MASK, bool ENERGY>
__global__ void __launch_bounds__(128, pipe_min_blocks<S>()) k17_box_pipe_kernel(BoxCollideArgs<typename Codec<S>::compute> a)
{
    using C = typename Codec<S>::compute;
    const uint32_t tiles_x = ((uint32_t)a.nx + blockDim.x - 1) / blockDim.x;
    const int64_t ntiles = (int64_t)tiles_x * a.ny * a.nz;
    S *base = static_cast<S *>(a.dist);
    double m_acc = 0.0, e_acc = 0.0;

    C fn[27];
    uint32_t nn[8];
    int64_t t = blockIdx.x;
    bool an = t < ntiles && pipe_node(a, tiles_x, t, nn);
    if (MASK && an)
        an = __ldg(a.mask + nn[0]) != 0;
    if (an)
        gather_pre<S, EVEN>(base, a.pitch, nn, fn);
    for (; t < ntiles; t += gridDim.x) {
        C f[27];
        uint32_t nodes[8];
        const bool act = an;
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = fn[d];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            nodes[j] = nn[j];
        // the next tile's loads go out before this tile's arithmetic
        const int64_t tn = t + gridDim.x;
        an = tn < ntiles && pipe_node(a, tiles_x, tn, nn);
        if (MASK && an)
            an = __ldg(a.mask + nn[0]) != 0;
        if (an)
            gather_pre<S, EVEN>(base, a.pitch, nn, fn);
        if (act) {
            C drho, vx, vy, vz;
            collide<C, EXACT>(f, a.rates, a.fx, a.fy, a.fz, drho, vx, vy, vz);
            scatter_post<S, EVEN>(base, a.pitch, nodes, f);
            if (ENERGY) {
                m_acc += 1.0 + (double)drho;
                e_acc += 0.5 * (1.0 + (double)drho) * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
            }
        }
    }
    if (ENERGY) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m_acc += __shfl_down_sync(0xffffffffu, m_acc, o);
            e_acc += __shfl_down_sync(0xffffffffu, e_acc, o);
        }
        if ((threadIdx.x & 31) == 0) {
            const uint64_t w = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
            a.energy_partials[2 * w] = m_acc;
            a.energy_partials[2 * w + 1] = e_acc;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// The box collision for the FP32-arithmetic forms with two nodes per thread, (x, y) and (x, y + 1),
// collided together in packed FP32x2 arithmetic (packed.cuh): the arithmetic issues about half the
// instructions, the loads and stores stay coalesced per row. FMA arithmetic only.
// ---------------------------------------------------------------------------------------------
template <class S, bool EVEN, bool MASK, bool ENERGY>
__global__ void __launch_bounds__(128) k17_box_pair_kernel(BoxCollideArgs<float> a)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.z;
    const int y0 = 2 * (int)blockIdx.y;
    bool act[2];
    uint32_t nodes[2][8];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const int y = y0 + p;
        const uint32_t k = (uint32_t)((uint64_t)a.nx * ((uint64_t)y + (uint64_t)a.ny * (uint64_t)z) + (uint64_t)x);
        act[p] = x < a.nx && y < a.ny;
        if (MASK && act[p])
            act[p] = __ldg(a.mask + k) != 0;
        const int xp = (x + 1 < a.nx) ? x + 1 : (a.periodic_x ? 0 : x);
        const int yp = (y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y);
        const int zp = (z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z);
        const uint32_t sx = (uint32_t)(xp - x);
        const uint32_t sy = (uint32_t)((yp - y) * a.nx);
        const uint32_t sz = (uint32_t)((int64_t)(zp - z) * a.nx * a.ny);
        nodes[p][0] = k;
        nodes[p][1] = k + sx;
        nodes[p][2] = k + sy;
        nodes[p][3] = k + sx + sy;
        nodes[p][4] = k + sz;
        nodes[p][5] = k + sx + sz;
        nodes[p][6] = k + sy + sz;
        nodes[p][7] = k + sx + sy + sz;
    }
    float mac[2][4] = { { 0.f, 0.f, 0.f, 0.f }, { 0.f, 0.f, 0.f, 0.f } };
    if (act[0] || act[1]) {
        S *base = static_cast<S *>(a.dist);
        float fa[27], fb[27];
        // an inactive partner collides a rest state (drho = 0, u = 0): finite, never stored
        if (act[0]) gather_pre<S, EVEN>(base, a.pitch, nodes[0], fa);
        else
#pragma unroll
            for (int d = 0; d < 27; ++d) fa[d] = 0.f;
        if (act[1]) gather_pre<S, EVEN>(base, a.pitch, nodes[1], fb);
        else
#pragma unroll
            for (int d = 0; d < 27; ++d) fb[d] = 0.f;
        collide_pair(fa, fb, a.rates, a.fx, a.fy, a.fz, mac[0], mac[1]);
        if (act[0])
            scatter_post<S, EVEN>(base, a.pitch, nodes[0], fa);
        if (act[1])
            scatter_post<S, EVEN>(base, a.pitch, nodes[1], fb);
    }
    if (ENERGY) {
        double m = 0.0, e = 0.0;
#pragma unroll
        for (int p = 0; p < 2; ++p)
            if (act[p]) {
                const double r = 1.0 + (double)mac[p][0];
                m += r;
                e += 0.5 * r * ((double)mac[p][1] * mac[p][1] + (double)mac[p][2] * mac[p][2] + (double)mac[p][3] * mac[p][3]);
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m += __shfl_down_sync(0xffffffffu, m, o);
            e += __shfl_down_sync(0xffffffffu, e, o);
        }
        if ((threadIdx.x & 31) == 0) {
            const uint64_t b = blockIdx.x + (uint64_t)gridDim.x * (blockIdx.y + (uint64_t)gridDim.y * blockIdx.z);
            const uint64_t w = b * (blockDim.x >> 5) + (threadIdx.x >> 5);
            a.energy_partials[2 * w] = m;
            a.energy_partials[2 * w + 1] = e;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// The same collision + streaming with the populations of the next tile staged in shared memory by
// bulk asynchronous copies (TMA) while the current tile computes.
//
// Every warp runs its own pipeline: it walks warp tiles (32 consecutive nodes of one x-row) of
// the box, and for each tile 27 lanes issue one 1-D bulk copy each (one per direction plane) of
// the row segment the tile reads, shifted by one node in x, y or z for directions with negative
// components (the x-shifted ones copy 16 extra bytes). A per-warp mbarrier counts the bytes in.
// With two stages the copies of tile i+1 are in flight while tile i computes, so memory latency
// overlaps the arithmetic, and no warp ever waits for another (no block-wide barrier in the
// loop). Results go straight to global memory: in the esoteric twist each node writes exactly
// the slots it read, so the stores of one tile never touch slots another tile still has to load.
// Requires nx % 32 == 0 (rows split into whole warp tiles, 16-byte aligned rows).
// ---------------------------------------------------------------------------------------------
template <class S>
struct TmaTile {
    static constexpr int BX = 32;                        // nodes per warp tile
    static constexpr int WARPS = 4;                      // warps per block
    static constexpr int EXTRA = 16 / (int)sizeof(S);    // 16 bytes of elements
    static constexpr int ROW = BX + EXTRA;
    static constexpr int STAGES = 2;
    static constexpr uint32_t STAGE_ELEMS = 27u * ROW;
    static constexpr uint32_t WARP_ELEMS = STAGES * STAGE_ELEMS;
    static constexpr size_t SMEM = WARPS * (WARP_ELEMS * sizeof(S) + STAGES * sizeof(uint64_t));
};

// issue the copies of tile t into one stage: lane 0 announces the bytes, lanes 0..26 copy one
// direction each (the announcement precedes the copies in program order of lane 0 and the
// warp-synchronous __syncwarp orders the other lanes after it)
template <class S, bool EVEN, class A>
__device__ __forceinline__ void tma_issue_tile(const A &a, int64_t t, S *stage, uint64_t *bar, int lane)
{
    using T = TmaTile<S>;
    const int tiles_x = a.nx / T::BX;
    const int xt = (int)(t % tiles_x);
    const int64_t r = t / tiles_x;
    const int y = (int)(r % a.ny), z = (int)(r / a.ny);
    const int x0 = xt * T::BX;
    const bool row_end = x0 + T::BX == a.nx;
    if (lane == 0) {
        // 9 directions point negative in x: they copy 16 more bytes (the wrap copy at a row end)
        const uint32_t extra = (!row_end || a.periodic_x) ? 16u : 0u;
        mbar_arrive_expect_tx(bar, 27u * T::BX * (uint32_t)sizeof(S) + 9u * extra);
    }
    __syncwarp();
    if (lane < 27) {
        const int d = lane;
        const int ddx = cx(d), ddy = cy(d), ddz = cz(d);
        const int yy = ddy < 0 ? ((y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y)) : y;
        const int zz = ddz < 0 ? ((z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z)) : z;
        const int pl = EVEN ? d : inv(d);
        const S *row = static_cast<const S *>(a.dist) + (uint64_t)pl * a.pitch
                     + (uint64_t)a.nx * ((uint64_t)yy + (uint64_t)a.ny * zz);
        S *dst = stage + d * T::ROW;
        if (ddx < 0 && !row_end) {
            bulk_copy_g2s(dst, row + x0, (T::BX + T::EXTRA) * (uint32_t)sizeof(S), bar);
        } else {
            bulk_copy_g2s(dst, row + x0, T::BX * (uint32_t)sizeof(S), bar);
            if (ddx < 0 && a.periodic_x) // x + 1 of the last node wraps to x = 0 of the same row
                bulk_copy_g2s(dst + T::BX, row, 16u, bar);
        }
    }
}

template <class S, bool EXACT, bool EVEN, bool MASK, bool ENERGY>
__global__ void __launch_bounds__(128) k17_box_tma_kernel(BoxCollideArgs<typename Codec<S>::compute> a, int *status)
{
    using C = typename Codec<S>::compute;
    using T = TmaTile<S>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    S *buf = reinterpret_cast<S *>(smem_raw) + warp * T::WARP_ELEMS;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + T::WARPS * T::WARP_ELEMS * sizeof(S)) + warp * T::STAGES;
    const int tiles_x = a.nx / T::BX;
    const int64_t ntiles = (int64_t)tiles_x * a.ny * a.nz;
    const int64_t first = (int64_t)blockIdx.x * T::WARPS + warp;
    const int64_t stride = (int64_t)gridDim.x * T::WARPS;

    if (lane == 0) {
        for (int s = 0; s < T::STAGES; ++s)
            mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncwarp();
    for (int s = 0; s < T::STAGES; ++s) {
        const int64_t t = first + s * stride;
        if (t < ntiles)
            tma_issue_tile<S, EVEN>(a, t, buf + s * T::STAGE_ELEMS, &bar[s], lane);
    }

    double m_acc = 0.0, e_acc = 0.0;
    uint32_t parity = 0; // bit s: parity of the next phase of stage s
    bool failed = false;
    int i = 0;
    for (int64_t t = first; t < ntiles; t += stride, ++i) {
        const int s = i & 1;
        const bool ok = mbar_wait(&bar[s], (parity >> s) & 1u);
        if (__any_sync(0xffffffffu, !ok)) {
            failed = true;
            break;
        }
        parity ^= 1u << s;

        const int xt = (int)(t % tiles_x);
        const int64_t r = t / tiles_x;
        const int y = (int)(r % a.ny), z = (int)(r / a.ny);
        const int x = xt * T::BX + lane;
        const uint32_t k = (uint32_t)((uint64_t)a.nx * ((uint64_t)y + (uint64_t)a.ny * z) + x);
        const bool active = !MASK || __ldg(a.mask + k) != 0;
        if (active) {
            const S *sb = buf + s * T::STAGE_ELEMS;
            C f[27];
#pragma unroll
            for (int d = 0; d < 27; ++d)
                f[d] = Codec<S>::load(sb + d * T::ROW + lane + (cx(d) < 0 ? 1 : 0), d);
            C drho, vx, vy, vz;
            collide<C, EXACT>(f, a.rates, a.fx, a.fy, a.fz, drho, vx, vy, vz);
            const int xp = (x + 1 < a.nx) ? x + 1 : (a.periodic_x ? 0 : x);
            const int yp = (y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y);
            const int zp = (z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z);
            const uint32_t sx = (uint32_t)(xp - x);
            const uint32_t sy = (uint32_t)((yp - y) * a.nx);
            const uint32_t sz = (uint32_t)((int64_t)(zp - z) * a.nx * a.ny);
            const uint32_t nodes[8] = { k, k + sx, k + sy, k + sx + sy, k + sz, k + sx + sz, k + sy + sz, k + sx + sy + sz };
            scatter_post<S, EVEN>(static_cast<S *>(a.dist), a.pitch, nodes, f);
            if (ENERGY) {
                m_acc += 1.0 + (double)drho;
                e_acc += 0.5 * (1.0 + (double)drho) * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
            }
        }
        // the warp is done reading stage s: order those generic-proxy reads before the async-proxy
        // writes of the next copies into it
        fence_proxy_async_smem();
        __syncwarp();
        const int64_t tn = t + (int64_t)T::STAGES * stride;
        if (tn < ntiles)
            tma_issue_tile<S, EVEN>(a, tn, buf + s * T::STAGE_ELEMS, &bar[s], lane);
    }

    if (failed) {
        if (lane == 0) {
            atomicExch(status, (int)kDevWaitTimeout);
            // let copies still in flight land before the block's shared memory is released
            for (int s = 0; s < T::STAGES; ++s)
                mbar_wait(&bar[s], (parity >> s) & 1u, 1u << 16);
        }
        __syncwarp();
    }

    if (ENERGY) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m_acc += __shfl_down_sync(0xffffffffu, m_acc, o);
            e_acc += __shfl_down_sync(0xffffffffu, e_acc, o);
        }
        __shared__ double red[2][T::WARPS];
        if (lane == 0) {
            red[0][warp] = m_acc;
            red[1][warp] = e_acc;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double mm = 0.0, ee = 0.0;
            for (int w = 0; w < T::WARPS; ++w) {
                mm += red[0][w];
                ee += red[1][w];
            }
            a.energy_partials[2 * blockIdx.x] = mm;
            a.energy_partials[2 * blockIdx.x + 1] = ee;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Collision + streaming with a per-thread software pipeline through shared memory: while a thread
// computes its node of tile i, cp.async copies of the 27 populations of its node of tile i+1 are
// in flight into slots of shared memory only this thread uses. Memory latency overlaps the
// arithmetic without extra registers and without any synchronisation between threads.
// Persistent blocks of 128 threads walk tiles of 128 nodes of an x-row. F64 and F32 storage
// (cp.async moves 4 or 8 bytes per copy).
// ---------------------------------------------------------------------------------------------
template <class S>
struct AsyncTile {
    static constexpr int BX = 128;
    static constexpr size_t SMEM = 2 * 27 * BX * sizeof(S);
};

template <class S, bool EVEN, class A>
__device__ __forceinline__ void async_issue_node(const A &a, int64_t t, int tid, S *stage, uint32_t &k_out, bool &active)
{
    const int tiles_x = (a.nx + AsyncTile<S>::BX - 1) / AsyncTile<S>::BX;
    const int xt = (int)(t % tiles_x);
    const int64_t r = t / tiles_x;
    const int y = (int)(r % a.ny), z = (int)(r / a.ny);
    const int x = xt * AsyncTile<S>::BX + tid;
    active = x < a.nx;
    const uint32_t k = (uint32_t)((uint64_t)a.nx * ((uint64_t)y + (uint64_t)a.ny * z) + (active ? x : 0));
    k_out = k;
    if (!active)
        return;
    const int xp = (x + 1 < a.nx) ? x + 1 : (a.periodic_x ? 0 : x);
    const int yp = (y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y);
    const int zp = (z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z);
    const uint32_t sx = (uint32_t)(xp - x), sy = (uint32_t)((yp - y) * a.nx), sz = (uint32_t)((int64_t)(zp - z) * a.nx * a.ny);
    const uint32_t nodes[8] = { k, k + sx, k + sy, k + sx + sy, k + sz, k + sx + sz, k + sy + sz, k + sx + sy + sz };
    const S *base = static_cast<const S *>(a.dist);
#pragma unroll
    for (int d = 0; d < 27; ++d)
        cp_async<(int)sizeof(S)>(stage + d * AsyncTile<S>::BX + tid,
                                 base + (uint64_t)plane<EVEN>(d) * a.pitch + nodes[shift_class(d)]);
}

template <class S, bool EXACT, bool EVEN, bool MASK, bool ENERGY>
__global__ void __launch_bounds__(128) k17_box_async_kernel(BoxCollideArgs<typename Codec<S>::compute> a)
{
    using C = typename Codec<S>::compute;
    constexpr int BX = AsyncTile<S>::BX;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    S *buf = reinterpret_cast<S *>(smem_raw);
    const int tid = threadIdx.x;
    const int tiles_x = (a.nx + BX - 1) / BX;
    const int64_t ntiles = (int64_t)tiles_x * a.ny * a.nz;

    double m_acc = 0.0, e_acc = 0.0;
    uint32_t k_cur = 0, k_next = 0;
    bool act_cur = false, act_next = false;
    int64_t t = blockIdx.x;
    if (t < ntiles)
        async_issue_node<S, EVEN>(a, t, tid, buf, k_cur, act_cur);
    cp_async_commit();
    for (int i = 0; t < ntiles; t += gridDim.x, ++i) {
        const int s = i & 1;
        const int64_t tn = t + gridDim.x;
        if (tn < ntiles)
            async_issue_node<S, EVEN>(a, tn, tid, buf + (s ^ 1) * 27 * BX, k_next, act_next);
        cp_async_commit();
        cp_async_wait<1>(); // this thread's copies of tile t have landed
        bool active = act_cur;
        if (MASK && active)
            active = __ldg(a.mask + k_cur) != 0;
        if (active) {
            const S *sb = buf + s * 27 * BX;
            C f[27];
#pragma unroll
            for (int d = 0; d < 27; ++d)
                f[d] = Codec<S>::load(sb + d * BX + tid, d);
            C drho, vx, vy, vz;
            collide<C, EXACT>(f, a.rates, a.fx, a.fy, a.fz, drho, vx, vy, vz);
            const uint32_t k = k_cur;
            const int x = (int)(k % (uint32_t)a.nx);
            const int y = (int)((k / (uint32_t)a.nx) % (uint32_t)a.ny);
            const int z = (int)(k / ((uint32_t)a.nx * (uint32_t)a.ny));
            const int xp = (x + 1 < a.nx) ? x + 1 : (a.periodic_x ? 0 : x);
            const int yp = (y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y);
            const int zp = (z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z);
            const uint32_t sx = (uint32_t)(xp - x), sy = (uint32_t)((yp - y) * a.nx), sz = (uint32_t)((int64_t)(zp - z) * a.nx * a.ny);
            const uint32_t nodes[8] = { k, k + sx, k + sy, k + sx + sy, k + sz, k + sx + sz, k + sy + sz, k + sx + sy + sz };
            scatter_post<S, EVEN>(static_cast<S *>(a.dist), a.pitch, nodes, f);
            if (ENERGY) {
                m_acc += 1.0 + (double)drho;
                e_acc += 0.5 * (1.0 + (double)drho) * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
            }
        }
        k_cur = k_next;
        act_cur = act_next;
    }
    cp_async_wait<0>();

    if (ENERGY) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m_acc += __shfl_down_sync(0xffffffffu, m_acc, o);
            e_acc += __shfl_down_sync(0xffffffffu, e_acc, o);
        }
        __shared__ double red[2][4];
        const int warp = tid >> 5, lane = tid & 31;
        if (lane == 0) {
            red[0][warp] = m_acc;
            red[1][warp] = e_acc;
        }
        __syncthreads();
        if (tid == 0) {
            double mm = 0.0, ee = 0.0;
            for (int w = 0; w < 4; ++w) {
                mm += red[0][w];
                ee += red[1][w];
            }
            a.energy_partials[2 * blockIdx.x] = mm;
            a.energy_partials[2 * blockIdx.x + 1] = ee;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// boundary conditions (one thread per BC node)
// ---------------------------------------------------------------------------------------------
template <class C>
__device__ __forceinline__ bool q_active(C q)
{
    return q >= C(0) && q <= C(1);
}

// NoSlipBounceBack_Device (NoSlip/NoSlipBounceBack.cu:44-179) and VelocityBounceBack_Device
// (Velocity/VelocityBounceBack.cu:44-188): for every link with q in [0,1] the population leaving
// along d comes back as inv(d) into the slot the node reads on the next step; the velocity
// variant adds 6 w (c_inv(d) . u_w) (coefficients 4/9, 1/9, 1/36).
template <class S, bool EVEN, bool VELOCITY>
__global__ void __launch_bounds__(128) bc_bounce_back_kernel(BCArgs a)
{
    using C = typename Codec<S>::compute;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nbc)
        return;
    const uint32_t node = (uint32_t)a.k[i];
    uint32_t nodes[8];
    node_slots(node, a.nbx, a.nby, a.nbz, a.n, a.box, nodes);
    S *base = static_cast<S *>(a.dist);
    C post[27];
    if (a.snap) {
#pragma unroll
        for (int d = 0; d < 27; ++d)
            post[d] = static_cast<const C *>(a.snap)[(uint64_t)d * a.nbc + i];
    } else {
        gather_post<S, EVEN>(base, a.n, nodes, post);
        const uint32_t mask = a.guard ? a.guard[i] : 0u;
        if (mask) {
            const C *saved = static_cast<const C *>(a.saved) + a.guard[a.nbc + i];
            int r = 0;
#pragma unroll
            for (int d = 1; d < 27; ++d)
                if ((mask >> d) & 1u)
                    post[d] = saved[r++];
        }
    }
    const C *q27 = static_cast<const C *>(a.q27);
    C ux = C(0), uy = C(0), uz = C(0);
    if (VELOCITY) {
        ux = static_cast<const C *>(a.ux)[i];
        uy = static_cast<const C *>(a.uy)[i];
        uz = static_cast<const C *>(a.uz)[i];
    }
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        const C q = q27[(uint64_t)d * a.nbc + i];
        if (q_active(q)) {
            const int e = inv(d);
            C v = post[d];
            if (VELOCITY) {
                const C coef = order(d) == 1 ? C(4) / C(9) : order(d) == 2 ? C(1) / C(9) : C(1) / C(36);
                C cu = C(0);
                // c_e . u spelled as the reference: signed sum x, y, z
                {
                    bool first = true;
                    if (cx(e) != 0) { cu = cx(e) > 0 ? ux : -ux; first = false; }
                    if (cy(e) != 0) { cu = first ? (cy(e) > 0 ? uy : -uy) : (cy(e) > 0 ? cu + uy : cu - uy); first = false; }
                    if (cz(e) != 0) { cu = first ? (cz(e) > 0 ? uz : -uz) : (cz(e) > 0 ? cu + uz : cu - uz); }
                }
                v = v + coef * cu;
            }
            // next parity: slot of direction e at its own read node
            Codec<S>::store_at(base, (uint64_t)plane<!EVEN>(e) * a.n + nodes[shift_class(e)], v, e);
        }
    }
}

template <int D, class C>
__device__ __forceinline__ C cdot(C ux, C uy, C uz)
{
    C s = C(0);
    bool first = true;
    if (cx(D) != 0) { s = cx(D) > 0 ? ux : -ux; first = false; }
    if (cy(D) != 0) { s = first ? (cy(D) > 0 ? uy : -uy) : (cy(D) > 0 ? s + uy : s - uy); first = false; }
    if (cz(D) != 0) { s = first ? (cz(D) > 0 ? uz : -uz) : (cz(D) > 0 ? s + uz : s - uz); }
    return s;
}

__device__ __forceinline__ int dir_sum_term(int d, int axis) { return axis == 0 ? cx(d) : axis == 1 ? cy(d) : cz(d); }

// signed sum c_d . u with a runtime-unrolled d
template <class C>
__device__ __forceinline__ C cdot_rt(int d, C ux, C uy, C uz)
{
    C s = C(0);
    bool first = true;
    if (cx(d) != 0) { s = cx(d) > 0 ? ux : -ux; first = false; }
    if (cy(d) != 0) { s = first ? (cy(d) > 0 ? uy : -uy) : (cy(d) > 0 ? s + uy : s - uy); first = false; }
    if (cz(d) != 0) { s = first ? (cz(d) > 0 ? uz : -uz) : (cz(d) > 0 ? s + uz : s - uz); }
    return s;
}

// NoSlipInterpolatedCompressible_Device (NoSlip/NoSlipInterpolatedCompressible.cu:44-381) and
// VelocityInterpolatedCompressible_Device (Velocity/VelocityInterpolatedCompressible.cu:44-420),
// with the helper formulas of KernelUtilities.h:171-210. FORM selects the variant:
//   kBCCompressible  — the two kernels above;
//   kBCIncompressible — NoSlipInterpolatedIncompressible.cu:44-387 / VelocityInterpolatedIncompressible.cu:44-497:
//                       the momenta are not divided by rho and cu_sq does not carry (1 + drho); feq drops
//                       (1 + drho) in the velocity kernel only (the no-slip one calls getEquilibriumForBC);
//   kBCWithPressure  — VelocityWithPressureInterpolatedCompressible.cu:44-422: the compressible
//                       form minus w drho (getInterpolatedDistributionForVeloWithPressureBC);
//   kBCSlip          — SlipCompressible_Device (Slip/SlipCompressible.cu:44-550): the compressible
//                       velocity form whose wall velocity is the node's own velocity (slip length
//                       1), with the component along an axis zeroed when either of that axis's two
//                       links is cut.
enum : int { kBCCompressible = 0, kBCIncompressible = 1, kBCWithPressure = 2, kBCSlip = 3 };

// density, velocity and c_s^2-scaled u^2 of a BC node's post-collision populations
// (NoSlipInterpolatedCompressible.cu:134-153: plain-sum density, grouped momenta)
template <class C>
struct BCMoments {
    C drho, ux, uy, uz, cu_sq;
};

template <class C, int FORM>
__device__ __forceinline__ BCMoments<C> bc_moments(const C (&p)[27])
{
    BCMoments<C> m;
    m.drho = p[21] + p[20] + p[19] + p[22] + p[25] + p[24] + p[23] + p[26] + p[17] + p[18] + p[15] + p[16] + p[13]
           + p[14] + p[11] + p[12] + p[9] + p[10] + p[7] + p[8] + p[5] + p[6] + p[3] + p[4] + p[1] + p[2] + p[0];
    const C r = C(1) + m.drho;
    const C vx = (((((p[21] - p[24]) - (p[20] - p[25])) + ((p[19] - p[26]) - (p[22] - p[23]))) + ((p[13] - p[14]) + (p[11] - p[12])))
                  + ((p[9] - p[10]) + (p[7] - p[8]))) + (p[1] - p[2]);
    const C vy = (((((-(p[21] - p[24])) + (p[20] - p[25])) + ((p[19] - p[26]) - (p[22] - p[23]))) + ((p[17] - p[18]) + (p[15] - p[16])))
                  + ((-(p[9] - p[10])) + (p[7] - p[8]))) + (p[3] - p[4]);
    const C vz = (((((p[21] - p[24]) + (p[20] - p[25])) + ((p[19] - p[26]) + (p[22] - p[23]))) + ((-(p[17] - p[18])) + (p[15] - p[16])))
                  + ((p[11] - p[12]) - (p[13] - p[14]))) + (p[5] - p[6]);
    m.ux = FORM == kBCIncompressible ? vx : vx / r;
    m.uy = FORM == kBCIncompressible ? vy : vy / r;
    m.uz = FORM == kBCIncompressible ? vz : vz / r;
    m.cu_sq = FORM == kBCIncompressible ? C(1.5) * (m.ux * m.ux + m.uy * m.uy + m.uz * m.uz)
                                        : C(1.5) * (m.ux * m.ux + m.uy * m.uy + m.uz * m.uz) * (C(1) + m.drho);
    return m;
}

// the value written for one cut link: f = p[d], fi = p[inv d], w and vel = c_d . u of direction d,
// vbc = c_d . u_wall (velocity kernels)
template <class C, bool VELOCITY, int FORM>
__device__ __forceinline__ C bc_link_value(C f, C fi, C q, C w, C vel, C vbc, const BCMoments<C> &m, C omega)
{
    // the incompressible velocity kernel writes feq inline without (1 + drho); the incompressible
    // no-slip kernel keeps getEquilibriumForBC, which carries it
    const C feq = (FORM == kBCIncompressible && VELOCITY) ? w * (m.drho + C(4.5) * vel * vel - m.cu_sq)
                                                          : w * (m.drho + C(4.5) * vel * vel * (C(1) + m.drho) - m.cu_sq);
    C v;
    if (VELOCITY) {
        v = (C(1) - q) / (C(1) + q) * (f - fi + (f + fi - C(2) * feq * omega) / (C(1) - omega)) * C(0.5)
          + (q * (f + fi) - C(6) * w * vbc) / (C(1) + q);
        if (FORM == kBCWithPressure)
            v = v - w * m.drho;
    } else {
        v = (C(1) - q) / (C(1) + q) * (f - fi + (f + fi - C(2) * feq * omega) / (C(1) - omega)) * C(0.5)
          + (q * (f + fi)) / (C(1) + q);
    }
    return v;
}

// one BC node: its slot nodes, its q of every direction at q27[d * q_stride], the wall velocity
template <class S, bool EVEN, bool VELOCITY, int FORM>
__device__ __forceinline__ void bc_interpolated_node(S *base, uint64_t n, const uint32_t (&nodes)[8],
                                                     const typename Codec<S>::compute *q27, uint64_t q_stride,
                                                     double omega_real, typename Codec<S>::compute bx,
                                                     typename Codec<S>::compute by, typename Codec<S>::compute bz,
                                                     const typename Codec<S>::compute *snap = nullptr,
                                                     uint64_t snap_stride = 0, uint32_t guard_mask = 0,
                                                     const typename Codec<S>::compute *guard = nullptr)
{
    using C = typename Codec<S>::compute;
    C p[27];
    if (snap) {
#pragma unroll
        for (int d = 0; d < 27; ++d)
            p[d] = snap[(uint64_t)d * snap_stride];
    } else {
        gather_post<S, EVEN>(base, n, nodes, p);
        // directions whose slot another node of the list overwrites: the value saved before
        if (guard_mask) {
            int r = 0;
#pragma unroll
            for (int d = 1; d < 27; ++d)
                if ((guard_mask >> d) & 1u)
                    p[d] = guard[r++];
        }
    }
    const BCMoments<C> m = bc_moments<C, FORM>(p);
    const C omega = (C)omega_real;
    if (FORM == kBCSlip) {
        // the reference zeroes VeloX when the link P00 or M00 is cut, and so on; the links along the
        // axes come first there, so every diagonal link sees the zeroing of all three axes
        const bool cut_x = q_active(q27[1 * q_stride]) || q_active(q27[2 * q_stride]);
        const bool cut_y = q_active(q27[3 * q_stride]) || q_active(q27[4 * q_stride]);
        const bool cut_z = q_active(q27[5 * q_stride]) || q_active(q27[6 * q_stride]);
        bx = cut_x ? C(0) : m.ux;
        by = cut_y ? C(0) : m.uy;
        bz = cut_z ? C(0) : m.uz;
    }
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        const C q = q27[(uint64_t)d * q_stride];
        if (q_active(q)) {
            const C v = bc_link_value<C, VELOCITY, FORM>(p[d], p[inv(d)], q, weight_t<C>(d), cdot_rt<C>(d, m.ux, m.uy, m.uz),
                                                         VELOCITY ? cdot_rt<C>(d, bx, by, bz) : C(0), m, omega);
            const int e = inv(d);
            Codec<S>::store_at(base, (uint64_t)plane<!EVEN>(e) * n + nodes[shift_class(e)], v, e);
        }
    }
}

template <class S, bool EVEN, bool VELOCITY, int FORM = kBCCompressible>
__global__ void __launch_bounds__(128) bc_interpolated_kernel(BCArgs a)
{
    using C = typename Codec<S>::compute;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nbc)
        return;
    uint32_t nodes[8];
    node_slots((uint32_t)a.k[i], a.nbx, a.nby, a.nbz, a.n, a.box, nodes);
    C bx = C(0), by = C(0), bz = C(0);
    if (VELOCITY && FORM != kBCSlip) {
        bx = static_cast<const C *>(a.ux)[i];
        by = static_cast<const C *>(a.uy)[i];
        bz = static_cast<const C *>(a.uz)[i];
    }
    const C *snap = a.snap ? static_cast<const C *>(a.snap) + i : nullptr;
    const uint32_t mask = a.guard ? a.guard[i] : 0u;
    const C *saved = mask ? static_cast<const C *>(a.saved) + a.guard[a.nbc + i] : nullptr;
    bc_interpolated_node<S, EVEN, VELOCITY, FORM>(static_cast<S *>(a.dist), a.n, nodes,
                                                  static_cast<const C *>(a.q27) + i, a.nbc, a.omega, bx, by, bz,
                                                  snap, a.nbc, mask, saved);
}

// the guarded post-collision values of a list (guards.h), saved before the list's BC kernel writes
template <class S, bool EVEN>
__global__ void __launch_bounds__(128) bc_guard_kernel(BCArgs a, typename Codec<S>::compute *saved)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nbc)
        return;
    const uint32_t mask = a.guard[i];
    if (!mask)
        return;
    uint32_t nodes[8];
    node_slots((uint32_t)a.k[i], a.nbx, a.nby, a.nbz, a.n, a.box, nodes);
    const S *base = static_cast<const S *>(a.dist);
    typename Codec<S>::compute *out = saved + a.guard[a.nbc + i];
    int r = 0;
#pragma unroll
    for (int d = 1; d < 27; ++d)
        if ((mask >> d) & 1u)
            out[r++] = Codec<S>::load(base + (uint64_t)plane<EVEN>(inv(d)) * a.n + nodes[shift_class(inv(d))], d);
}

// The post-collision populations of every node of a BC list into snap[d * nbc + i], taken before
// the list's BC kernel writes anything: where two BC nodes of one list are joined by a link cut
// from both ends, each node's write lands in a slot the other reads, so reading the snapshot
// makes the result independent of thread order (every node sees the collision's values).
template <class S, bool EVEN>
__global__ void __launch_bounds__(128) bc_snapshot_kernel(BCArgs a, typename Codec<S>::compute *snap)
{
    using C = typename Codec<S>::compute;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nbc)
        return;
    uint32_t nodes[8];
    node_slots((uint32_t)a.k[i], a.nbx, a.nby, a.nbz, a.n, a.box, nodes);
    C p[27];
    gather_post<S, EVEN>(static_cast<const S *>(a.dist), a.n, nodes, p);
#pragma unroll
    for (int d = 0; d < 27; ++d)
        snap[(uint64_t)d * a.nbc + i] = p[d];
}

// feq - w of one direction in the form of the init and pressure kernels
template <class C>
__device__ __forceinline__ C feq_shifted(int d, C drho, C ux, C uy, C uz, C cusq)
{
    if (d == 0)
        return weight_t<C>(0) * (drho - (drho + C(1)) * cusq);
    const C cu = cdot_rt<C>(d, ux, uy, uz);
    return weight_t<C>(d) * (drho + (drho + C(1)) * (C(3) * cu + C(4.5) * cu * cu - cusq));
}

// PressureNonEquilibriumCompressible_Device (Pressure/PressureNonEquilibriumCompressible.cu:45-314).
// The reference's __syncthreads() between the neighbour reads and the writes (:174) sits in
// divergent code and orders nothing that needs ordering (no thread writes a slot another thread
// of the launch reads), so it has no counterpart here.
// INCOMP: PressureNonEquilibriumIncompressible_Device (Pressure/PressureNonEquilibriumIncompressible.cu:45-314),
// the same with getIncompressibleMacroscopicValues (u = momentum, not divided by rho)
// one BC node: the slot nodes of the node (nk) and of its inward neighbour (nn)
template <class S, bool EVEN, bool INCOMP>
__device__ __forceinline__ void bc_pressure_neq_node(S *base, uint64_t n, const uint32_t (&nk)[8],
                                                     const uint32_t (&nn)[8], typename Codec<S>::compute rbc,
                                                     int direction)
{
    using C = typename Codec<S>::compute;
    C f[27];
    gather_pre<S, EVEN>(base, n, nn, f);
    const C drho1 = density_pyramid(f);
    C vx, vy, vz;
    if (INCOMP) {
        vx = momentum_x(f);
        vy = momentum_y(f);
        vz = momentum_z(f);
    } else {
        const C inv_rho = C(1) / (drho1 + C(1));
        vx = momentum_x(f) * inv_rho;
        vy = momentum_y(f) * inv_rho;
        vz = momentum_z(f) * inv_rho;
    }
    const C cusq = C(1.5) * (vx * vx + vy * vy + vz * vz);
    const int axis = cx(direction) != 0 ? 0 : (cy(direction) != 0 ? 1 : 2);
    const int sgn = axis == 0 ? cx(direction) : (axis == 1 ? cy(direction) : cz(direction));
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        C v = f[d] - feq_shifted<C>(d, drho1, vx, vy, vz, cusq);
        v = v + feq_shifted<C>(d, rbc, vx, vy, vz, cusq);
        const int c = axis == 0 ? cx(d) : (axis == 1 ? cy(d) : cz(d));
        if (c != sgn)
            Codec<S>::store_at(base, (uint64_t)plane<EVEN>(d) * n + nk[shift_class(d)], v, d);
    }
}

template <class S, bool EVEN, bool INCOMP = false>
__global__ void __launch_bounds__(128) bc_pressure_neq_kernel(PressureArgs a)
{
    using C = typename Codec<S>::compute;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nbc)
        return;
    uint32_t nn[8], nk[8];
    node_slots((uint32_t)a.kN[i], a.nbx, a.nby, a.nbz, a.n, a.box, nn);
    node_slots((uint32_t)a.k[i], a.nbx, a.nby, a.nbz, a.n, a.box, nk);
    bc_pressure_neq_node<S, EVEN, INCOMP>(static_cast<S *>(a.dist), a.n, nk, nn, static_cast<const C *>(a.rho_bc)[i],
                                          a.direction);
}

// OutflowNonReflecting_Device (Outflow/OutflowNonReflecting.cu:50-276) and, with CORRECTION,
// OutflowNonReflectingPressureCorrection_Device (OutflowNonReflectingPressureCorrection.cu:53-241).
// Reads the node's and the inward neighbour's populations at the current parity and writes the
// nine directions pointing away from the outlet normal into the other parity:
//   f_d <- fN_d cs + (1 - cs) f_d  [- w_d c drho(f)],  cs = 1 / sqrtf(3).
// The corrected form reads fN with the neighbour index only for the unshifted slots and the node's
// own shifted slots otherwise (OutflowNonReflectingPressureCorrection.cu:75-81 take the shifted
// neighbours of k, not of kN); the same slots are read here.
template <class S, bool EVEN, bool CORRECTION>
__global__ void __launch_bounds__(128) bc_outflow_kernel(PressureArgs a, double correction)
{
    using C = typename Codec<S>::compute;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nbc)
        return;
    uint32_t nk[8], nn[8];
    node_slots((uint32_t)a.k[i], a.nbx, a.nby, a.nbz, a.n, a.box, nk);
    if (CORRECTION) {
#pragma unroll
        for (int c = 0; c < 8; ++c)
            nn[c] = nk[c];
        nn[0] = (uint32_t)a.kN[i];
    } else {
        node_slots((uint32_t)a.kN[i], a.nbx, a.nby, a.nbz, a.n, a.box, nn);
    }
    S *base = static_cast<S *>(a.dist);
    C f[27], fn[27];
    gather_pre<S, EVEN>(base, a.n, nk, f);
    gather_pre<S, EVEN>(base, a.n, nn, fn);
    const C cs = C(1) / (C)sqrtf(3.0f);
    C rho_corr = C(0);
    if (CORRECTION)
        rho_corr = (C)correction * density_pyramid(f);
    const int axis = cx(a.direction) != 0 ? 0 : (cy(a.direction) != 0 ? 1 : 2);
    const int sgn = axis == 0 ? cx(a.direction) : (axis == 1 ? cy(a.direction) : cz(a.direction));
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        const int c = axis == 0 ? cx(d) : (axis == 1 ? cy(d) : cz(d));
        if (c != -sgn)
            continue;
        C v = fn[d] * cs + (C(1) - cs) * f[d];
        if (CORRECTION)
            v = v - weight_t<C>(d) * rho_corr;
        Codec<S>::store_at(base, (uint64_t)plane<!EVEN>(d) * a.n + nk[shift_class(d)], v, d);
    }
}

// ---------------------------------------------------------------------------------------------
// initialisation and output
// ---------------------------------------------------------------------------------------------

// InitNavierStokesCompressible_Device (InitNavierStokesCompressible_Device.cu:44-215):
// equilibrium f - w of the node's (rho, u) into the node's read slots of one parity
template <class S, bool EVEN>
__global__ void __launch_bounds__(128) init_list_kernel(void *dist, uint64_t n, const uint32_t *nbx, const uint32_t *nby,
                                                        const uint32_t *nbz, const uint32_t *geo, const void *rho,
                                                        const void *ux, const void *uy, const void *uz)
{
    using C = typename Codec<S>::compute;
    const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const uint32_t g = geo[k];
    if (g == kGeoSolid || g == kGeoVoid)
        return;
    uint32_t nodes[8];
    list_nodes((uint32_t)k, nbx, nby, nbz, n, nodes);
    const C drho = static_cast<const C *>(rho)[k];
    const C vx = static_cast<const C *>(ux)[k], vy = static_cast<const C *>(uy)[k], vz = static_cast<const C *>(uz)[k];
    const C cu_sq = C(1.5) * (vx * vx + vy * vy + vz * vz);
    S *base = static_cast<S *>(dist);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        C v;
        if (d == 0) {
            v = weight_t<C>(0) * (drho - cu_sq * (C(1) + drho));
        } else {
            const C cu = cdot_rt<C>(d, vx, vy, vz);
            v = weight_t<C>(d) * (drho + (C(1) + drho) * (C(3) * cu + C(4.5) * cu * cu - cu_sq));
        }
        Codec<S>::store_at(base, (uint64_t)plane<EVEN>(d) * n + nodes[shift_class(d)], v, d);
    }
}

// The non-equilibrium parts of InitNavierStokesCompressibleNonEquilibrium_Device
// (InitNavierStokesCompressible_Device.cu:216-501), from the central-difference velocity gradients
// a = grad ux, b = grad uy, c = grad uz and omega, as 14 coefficients shared by opposite directions:
// 0 rest, 1 P00/M00, 2 0P0/0M0, 3 00P/00M, 4 PP0/MM0, 5 PM0/MP0, 6 P0P/M0M, 7 P0M/M0P, 8 0PP/0MM,
// 9 0PM/0MP, 10 PPP/MMM, 11 PPM/MMP, 12 PMP/MPM, 13 PMM/MPP. Every operation keeps the reference's
// order and types: its constants are double literals, so with real = float each coefficient is
// formed in double from float operands (float where both operands of a product or sum are float)
// and rounded to float once; the scale eps and the factor op are real 1.
template <class C>
__device__ __forceinline__ void init_neq_parts(C ax, C ay, C az, C bx, C by, C bz, C cx, C cy, C cz, C omega,
                                               C (&p)[14])
{
    const C eps = C(1), op = C(1), o = omega;
    p[1] = (C)(eps * ((5. * ax * o + 5. * by * o + 5. * cz * o - 8. * ax * op + 4. * by * op + 4. * cz * op)
                      / (54. * o * op)));
    p[2] = (C)(p[1] + eps * ((2. * (ax - by)) / (9. * o)));
    p[3] = (C)(p[1] + eps * ((2. * (ax - cz)) / (9. * o)));
    p[4] = (C)(eps * (-(5. * cz * o + 3. * (ay + bx) * op - 2. * cz * op + ax * (5. * o + op) + by * (5. * o + op))
                      / (54. * o * op)));
    p[5] = (C)(p[4] + eps * ((ay + bx) / (9. * o)));
    p[6] = (C)(eps * (-(5. * cz * o + by * (5. * o - 2. * op) + 3. * (az + cx) * op + cz * op + ax * (5. * o + op))
                      / (54. * o * op)));
    p[7] = (C)(p[6] + eps * ((az + cx) / (9. * o)));
    p[8] = (C)(eps * (-(5. * ax * o + 5. * by * o + 5. * cz * o - 2. * ax * op + by * op + 3. * bz * op + 3. * cy * op
                        + cz * op)
                      / (54. * o * op)));
    p[9] = (C)(p[8] + eps * ((bz + cy) / (9. * o)));
    p[0] = (C)(eps * ((5. * (ax + by + cz)) / (9. * op)));
    p[10] = (C)(eps * (-(ay + az + bx + bz + cx + cy) / (72. * o)));
    p[11] = (C)(-p[10] - eps * ((ay + bx) / (36. * o)));
    p[12] = (C)(-p[10] - eps * ((az + cx) / (36. * o)));
    p[13] = (C)(-p[10] - eps * ((bz + cy) / (36. * o)));
}
// the coefficient of direction d (D3Q27 numbering of lattice.cuh)
__host__ __device__ constexpr int init_neq_part_of(int d)
{
    constexpr int8_t t[27] = { 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 13, 12, 11, 11, 12, 13, 10 };
    return t[d];
}

// InitNavierStokesCompressibleNonEquilibrium_Device: the equilibrium of init_list_kernel plus
// (1 + drho) times the direction's non-equilibrium part, from the velocities of the six face
// neighbours (the -1 ones reached from neighborInverse, the node at -1 in x, y and z). The
// equilibrium is rounded to the storage's real type before the part is added, as the reference
// stores it and then adds; the 16-bit forms encode the sum once. Solid and void nodes get 96 in
// their rest slot, as the reference writes there.
template <class S, bool EVEN>
__global__ void __launch_bounds__(128) init_neq_list_kernel(void *dist, uint64_t n, const uint32_t *nbx,
                                                            const uint32_t *nby, const uint32_t *nbz,
                                                            const uint32_t *nb_inverse, const uint32_t *geo,
                                                            const void *rho, const void *ux, const void *uy,
                                                            const void *uz, typename Codec<S>::compute omega)
{
    using C = typename Codec<S>::compute;
    const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    S *base = static_cast<S *>(dist);
    const uint32_t g = geo[k];
    if (g == kGeoSolid || g == kGeoVoid) {
        Codec<S>::store_at(base, (uint64_t)plane<EVEN>(0) * n + k, C(96), 0);
        return;
    }
    uint32_t nodes[8];
    list_nodes((uint32_t)k, nbx, nby, nbz, n, nodes);
    const C *U = static_cast<const C *>(ux), *V = static_cast<const C *>(uy), *W = static_cast<const C *>(uz);
    const C drho = static_cast<const C *>(rho)[k];
    const C vx = U[k], vy = V[k], vz = W[k];
    // face neighbours: +1 from the neighbour lists, -1 from the -1/-1/-1 node stepped back up
    const uint32_t px = VFB_NODE(nbx[k], n), py = VFB_NODE(nby[k], n), pz = VFB_NODE(nbz[k], n);
    const uint32_t mxyz = VFB_NODE(nb_inverse[k], n);
    const uint32_t mx = VFB_NODE(nbz[VFB_NODE(nby[mxyz], n)], n);
    const uint32_t my = VFB_NODE(nbz[VFB_NODE(nbx[mxyz], n)], n);
    const uint32_t mz = VFB_NODE(nby[VFB_NODE(nbx[mxyz], n)], n);
    const C ax = (U[px] - U[mx]) / C(2), ay = (U[py] - U[my]) / C(2), az = (U[pz] - U[mz]) / C(2);
    const C bx = (V[px] - V[mx]) / C(2), by = (V[py] - V[my]) / C(2), bz = (V[pz] - V[mz]) / C(2);
    const C cx = (W[px] - W[mx]) / C(2), cy = (W[py] - W[my]) / C(2), cz = (W[pz] - W[mz]) / C(2);
    C part[14];
    init_neq_parts<C>(ax, ay, az, bx, by, bz, cx, cy, cz, omega, part);
    const C cu_sq = C(1.5) * (vx * vx + vy * vy + vz * vz);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        C v;
        if (d == 0) {
            v = weight_t<C>(0) * (drho - cu_sq * (C(1) + drho));
        } else {
            const C cu = cdot_rt<C>(d, vx, vy, vz);
            v = weight_t<C>(d) * (drho + (C(1) + drho) * (C(3) * cu + C(4.5) * cu * cu - cu_sq));
        }
        v = v + (C(1) + drho) * part[init_neq_part_of(d)];
        Codec<S>::store_at(base, (uint64_t)plane<EVEN>(d) * n + nodes[shift_class(d)], v, d);
    }
}

// the same equilibrium initialisation on a structured box (every node, or the masked ones)
template <class S, bool EVEN>
__global__ void __launch_bounds__(128) init_box_kernel(BoxCollideArgs<typename Codec<S>::compute> a, const void *rho,
                                                       const void *ux, const void *uy, const void *uz)
{
    using C = typename Codec<S>::compute;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= a.nx)
        return;
    const uint32_t k = (uint32_t)((uint64_t)a.nx * ((uint64_t)y + (uint64_t)a.ny * z) + x);
    if (a.mask && a.mask[k] == 0)
        return;
    const int xp = (x + 1 < a.nx) ? x + 1 : (a.periodic_x ? 0 : x);
    const int yp = (y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y);
    const int zp = (z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z);
    const uint32_t sx = (uint32_t)(xp - x), sy = (uint32_t)((yp - y) * a.nx), sz = (uint32_t)((int64_t)(zp - z) * a.nx * a.ny);
    const uint32_t nodes[8] = { k, k + sx, k + sy, k + sx + sy, k + sz, k + sx + sz, k + sy + sz, k + sx + sy + sz };
    const C drho = static_cast<const C *>(rho)[k];
    const C vx = static_cast<const C *>(ux)[k], vy = static_cast<const C *>(uy)[k], vz = static_cast<const C *>(uz)[k];
    const C cu_sq = C(1.5) * (vx * vx + vy * vy + vz * vz);
    S *base = static_cast<S *>(a.dist);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        C v;
        if (d == 0) {
            v = weight_t<C>(0) * (drho - cu_sq * (C(1) + drho));
        } else {
            const C cu = cdot_rt<C>(d, vx, vy, vz);
            v = weight_t<C>(d) * (drho + (C(1) + drho) * (C(3) * cu + C(4.5) * cu * cu - cu_sq));
        }
        Codec<S>::store_at(base, (uint64_t)plane<EVEN>(d) * a.pitch + nodes[shift_class(d)], v, d);
    }
}

// calculateMacroscopicQuantitiesCompressible_device (PostProcessor/MacroscopicQuantities.cu:194)
template <class S, bool EVEN>
__global__ void __launch_bounds__(128) macros_list_kernel(const void *dist, uint64_t n, const uint32_t *nbx,
                                                          const uint32_t *nby, const uint32_t *nbz, const uint32_t *geo,
                                                          void *rho_o, void *vx_o, void *vy_o, void *vz_o, void *p_o)
{
    using C = typename Codec<S>::compute;
    const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    C *rho = static_cast<C *>(rho_o), *vx = static_cast<C *>(vx_o), *vy = static_cast<C *>(vy_o), *vz = static_cast<C *>(vz_o);
    C *press = static_cast<C *>(p_o);
    if (press)
        press[k] = C(0);
    rho[k] = C(0);
    vx[k] = C(0);
    vy[k] = C(0);
    vz[k] = C(0);
    if (geo[k] != kGeoFluid)
        return;
    uint32_t nodes[8];
    list_nodes((uint32_t)k, nbx, nby, nbz, n, nodes);
    C f[27];
    gather_pre<S, EVEN>(static_cast<const S *>(dist), n, nodes, f);
    const C r = density_pyramid(f);
    const C ux = momentum_x(f) / (r + C(1)), uy = momentum_y(f) / (r + C(1)), uz = momentum_z(f) / (r + C(1));
    rho[k] = r;
    vx[k] = ux;
    vy[k] = uy;
    vz[k] = uz;
    if (press) {
        // getPressure (MacroscopicQuantities.h:139)
        press[k] = (f[1] + f[2] + f[3] + f[4] + f[5] + f[6]
                    + C(2) * (f[7] + f[8] + f[9] + f[10] + f[11] + f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18])
                    + C(3) * (f[19] + f[22] + f[21] + f[20] + f[23] + f[26] + f[25] + f[24])
                    - r - (ux * ux + uy * uy + uz * uz) * (C(1) + r)) * C(0.5) + r;
    }
}

// macroscopic fields of a structured box, written in compute type, from the pre-collision state
template <class S, bool EVEN>
__global__ void __launch_bounds__(128) macros_box_kernel(BoxCollideArgs<typename Codec<S>::compute> a)
{
    using C = typename Codec<S>::compute;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= a.nx)
        return;
    const uint32_t k = (uint32_t)((uint64_t)a.nx * ((uint64_t)y + (uint64_t)a.ny * z) + x);
    if (a.mask && a.mask[k] == 0) {
        a.rho[k] = C(0);
        a.vx[k] = C(0);
        a.vy[k] = C(0);
        a.vz[k] = C(0);
        return;
    }
    const int xp = (x + 1 < a.nx) ? x + 1 : (a.periodic_x ? 0 : x);
    const int yp = (y + 1 < a.ny) ? y + 1 : (a.periodic_y ? 0 : y);
    const int zp = (z + 1 < a.nz) ? z + 1 : (a.periodic_z ? 0 : z);
    const uint32_t sx = (uint32_t)(xp - x), sy = (uint32_t)((yp - y) * a.nx), sz = (uint32_t)((int64_t)(zp - z) * a.nx * a.ny);
    const uint32_t nodes[8] = { k, k + sx, k + sy, k + sx + sy, k + sz, k + sx + sz, k + sy + sz, k + sx + sy + sz };
    C f[27];
    gather_pre<S, EVEN>(static_cast<const S *>(a.dist), a.pitch, nodes, f);
    const C r = density_pyramid(f);
    a.rho[k] = r;
    a.vx[k] = momentum_x(f) / (r + C(1));
    a.vy[k] = momentum_y(f) / (r + C(1));
    a.vz[k] = momentum_z(f) / (r + C(1));
}

// FP64 mass and kinetic energy over a node list: per-block partials in a fixed order
template <class S, bool EVEN>
__global__ void __launch_bounds__(256) energy_list_kernel(const void *dist, uint64_t n, const uint32_t *nbx,
                                                          const uint32_t *nby, const uint32_t *nbz, const uint32_t *idx,
                                                          uint32_t n_idx, double *partials)
{
    using C = typename Codec<S>::compute;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0, e = 0.0;
    if (i < n_idx) {
        uint32_t nodes[8];
        list_nodes(__ldg(idx + i), nbx, nby, nbz, n, nodes);
        C f[27];
        gather_pre<S, EVEN>(static_cast<const S *>(dist), n, nodes, f);
        const C r = density_pyramid(f);
        const C inv_rho = C(1) / (r + C(1));
        const double ux = momentum_x(f) * inv_rho, uy = momentum_y(f) * inv_rho, uz = momentum_z(f) * inv_rho;
        m = 1.0 + (double)r;
        e = 0.5 * (1.0 + (double)r) * (ux * ux + uy * uy + uz * uz);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, o);
        e += __shfl_down_sync(0xffffffffu, e, o);
    }
    __shared__ double sm[2][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sm[0][warp] = m;
        sm[1][warp] = e;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double mm = 0.0, ee = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            mm += sm[0][w];
            ee += sm[1][w];
        }
        partials[2 * blockIdx.x] = mm;
        partials[2 * blockIdx.x + 1] = ee;
    }
}


// ---------------------------------------------------------------------------------------------
// refinement: interpolation between a coarse level and the fine level nested in it
// (GridScaling/scaleCoarseToFineCompressible.cu:305-528, scaleFineToCoarseCompressible.cu:76-124)
//
// Eight lanes per interpolation cell, one per corner (interp.cuh): each lane gathers its own
// corner's 27 populations, so a cell's source reads are spread over eight threads instead of one,
// and the coefficient sums are formed by shuffles in a fixed corner order.
// ---------------------------------------------------------------------------------------------
struct ScaleArgs {
    void *dist_coarse, *dist_fine;
    uint64_t n_coarse, n_fine;
    const uint32_t *nbx_c, *nby_c, *nbz_c;
    const uint32_t *nbx_f, *nby_f, *nbz_f;
    const uint32_t *coarse_cells;   // CF: MMM node of the coarse cell; FC: the coarse node at the cell centre
    const uint32_t *fine_cells;     // MMM node of the fine cell
    uint32_t n_cells;
    const void *ox, *oy, *oz;       // offsets of the expansion point, compute type (ICellNeigh)
    double omega_coarse, omega_fine;
};

// corner c = ix + 2 iy + 4 iz of the cell whose MMM node is `base`, stepping x, then y, then z
__device__ __forceinline__ uint32_t cell_corner(uint32_t base, int c, const uint32_t *__restrict__ nbx,
                                                const uint32_t *__restrict__ nby, const uint32_t *__restrict__ nbz,
                                                uint64_t n)
{
    (void)n;
    uint32_t k = VFB_NODE(base, n);
    if (c & 1)
        k = VFB_NODE(__ldg(nbx + k), n);
    if (c & 2)
        k = VFB_NODE(__ldg(nby + k), n);
    if (c & 4)
        k = VFB_NODE(__ldg(nbz + k), n);
    return k;
}

// coefficients of the cell of this lane's group: moments of the corner at node k (pre-collision
// populations of parity EVEN), gathered over the group by shuffles. Every lane of the warp calls it.
template <class S, bool EVEN>
__device__ __forceinline__ void cell_coefficients_of_group(const S *base, uint64_t n, uint32_t k, bool valid,
                                                           const uint32_t *nbx, const uint32_t *nby,
                                                           const uint32_t *nbz, typename Codec<S>::compute omega,
                                                           typename Codec<S>::compute xo, typename Codec<S>::compute yo,
                                                           typename Codec<S>::compute zo,
                                                           InterpCoef<typename Codec<S>::compute> &coef)
{
    using C = typename Codec<S>::compute;
    C m[9];
    if (valid) {
        uint32_t nodes[8];
        list_nodes(k, nbx, nby, nbz, n, nodes);
        C f[27];
        gather_pre<S, EVEN>(base, n, nodes, f);
        interp_node_moments(f, omega, m);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            m[i] = C(0);
    }
    CellSums<C> sums;
    gather_cell_sums(sums, m, (int)(threadIdx.x & 31u) & ~7);
    cell_coefficients(sums, xo, yo, zo, coef);
}

// scaleCoarseToFineCompressible_Device: moments of the coarse cell at the coarse parity with
// omega_coarse; the fine node of this lane's corner sits at (+-1/4)^3 in coarse-cell units and
// receives the interpolated populations (epsilon 1/2, omega_fine) as its pre-collision
// populations of the even parity
template <class S, bool COARSE_EVEN>
__global__ void __launch_bounds__(128) scale_cf_kernel(ScaleArgs a)
{
    using C = typename Codec<S>::compute;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t cell = t >> 3;
    const int corner = (int)(t & 7u);
    const bool valid = cell < a.n_cells;
    uint32_t k = 0;
    C xo = C(0), yo = C(0), zo = C(0);
    if (valid) {
        k = cell_corner(__ldg(a.coarse_cells + cell), corner, a.nbx_c, a.nby_c, a.nbz_c, a.n_coarse);
        xo = static_cast<const C *>(a.ox)[cell];
        yo = static_cast<const C *>(a.oy)[cell];
        zo = static_cast<const C *>(a.oz)[cell];
    }
    InterpCoef<C> coef;
    cell_coefficients_of_group<S, COARSE_EVEN>(static_cast<const S *>(a.dist_coarse), a.n_coarse, k, valid, a.nbx_c,
                                               a.nby_c, a.nbz_c, (C)a.omega_coarse, xo, yo, zo, coef);
    if (!valid)
        return;
    const C q = C(0.25);
    C f[27];
    interp_point<C, false>(coef, (C)a.omega_fine, C(0.5), (corner & 1) ? q : -q, (corner & 2) ? q : -q,
                           (corner & 4) ? q : -q, f);
    uint32_t nodes[8];
    list_nodes(cell_corner(__ldg(a.fine_cells + cell), corner, a.nbx_f, a.nby_f, a.nbz_f, a.n_fine), a.nbx_f, a.nby_f,
               a.nbz_f, a.n_fine, nodes);
    S *fine = static_cast<S *>(a.dist_fine);
#pragma unroll
    for (int d = 0; d < 27; ++d)
        Codec<S>::store_at(fine, (uint64_t)plane<true>(d) * a.n_fine + nodes[shift_class(d)], f[d], d);
}

// scaleFineToCoarseCompressible_Device: moments of the fine cell at the even parity with
// omega_fine; the coarse node at the cell centre receives the interpolated populations
// (epsilon 2, omega_coarse) as its pre-collision populations of the coarse parity. The eight lanes
// of the cell share the 27 stores.
template <class S, bool COARSE_EVEN>
__global__ void __launch_bounds__(128) scale_fc_kernel(ScaleArgs a)
{
    using C = typename Codec<S>::compute;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t cell = t >> 3;
    const int corner = (int)(t & 7u);
    const bool valid = cell < a.n_cells;
    uint32_t k = 0;
    C xo = C(0), yo = C(0), zo = C(0);
    if (valid) {
        k = cell_corner(__ldg(a.fine_cells + cell), corner, a.nbx_f, a.nby_f, a.nbz_f, a.n_fine);
        xo = static_cast<const C *>(a.ox)[cell];
        yo = static_cast<const C *>(a.oy)[cell];
        zo = static_cast<const C *>(a.oz)[cell];
    }
    InterpCoef<C> coef;
    cell_coefficients_of_group<S, true>(static_cast<const S *>(a.dist_fine), a.n_fine, k, valid, a.nbx_f, a.nby_f,
                                        a.nbz_f, (C)a.omega_fine, xo, yo, zo, coef);
    if (!valid)
        return;
    C f[27];
    interp_point<C, true>(coef, (C)a.omega_coarse, C(2), C(0), C(0), C(0), f);
    uint32_t nodes[8];
    list_nodes(__ldg(a.coarse_cells + cell), a.nbx_c, a.nby_c, a.nbz_c, a.n_coarse, nodes);
    S *coarse = static_cast<S *>(a.dist_coarse);
#pragma unroll
    for (int d = 0; d < 27; ++d)
        if ((d & 7) == corner)
            Codec<S>::store_at(coarse, (uint64_t)plane<COARSE_EVEN>(d) * a.n_coarse + nodes[shift_class(d)], f[d], d);
}


// ---------------------------------------------------------------------------------------------
// drag and lift by momentum exchange (PostProcessor/DragLift.cu:50-555)
// ---------------------------------------------------------------------------------------------
struct DragArgs {
    const void *dist;
    uint64_t n;
    const uint32_t *nbx, *nby, *nbz;
    NodeAddr box;
    const int32_t *k;           // geometry BC node indices
    const void *q27;            // q27[dir * nbc + i], compute type
    uint32_t nbc;
    double *dx, *dy, *dz;       // per node
};

// the pairs of the reference's bracket structure, per axis: four corner pairs, four edge pairs,
// the face pair; each (plus direction, minus direction)
__device__ __forceinline__ int drag_pair(int axis, int i, int side)
{
    constexpr int P[3][9][2] = {
        { { 25, 20 }, { 23, 22 }, { 21, 24 }, { 19, 26 }, { 13, 14 }, { 11, 12 }, { 9, 10 }, { 7, 8 }, { 1, 2 } },
        { { 20, 25 }, { 23, 22 }, { 24, 21 }, { 19, 26 }, { 17, 18 }, { 15, 16 }, { 10, 9 }, { 7, 8 }, { 3, 4 } },
        { { 20, 25 }, { 22, 23 }, { 21, 24 }, { 19, 26 }, { 18, 17 }, { 15, 16 }, { 14, 13 }, { 11, 12 }, { 5, 6 } }
    };
    return P[axis][i][side];
}

// minus the momentum sum of one axis, in double, with the reference's association:
// ((((c1 + c2) + c3) + c4) + (((e1 + e2) + e3) + e4)) + face, each term (f_p on_p) - (f_m on_m)
__device__ __forceinline__ double drag_axis(const double (&f)[27], const double (&on)[27], int axis)
{
    double t[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int p = drag_pair(axis, i, 0), m = drag_pair(axis, i, 1);
        t[i] = (f[p] * on[p]) - (f[m] * on[m]);
    }
    return -(((((t[0] + t[1]) + t[2]) + t[3]) + (((t[4] + t[5]) + t[6]) + t[7])) + t[8]);
}

// DragLiftPost27 (PRE = false): after the collision, the post-collision populations leaving the
// node along each cut link d (q_d in [0, 1]). DragLiftPre27 (PRE = true): after the parity swap,
// the pre-collision populations the node reads next, each weighted by the cut link of the opposite
// direction.
template <class S, bool EVEN, bool PRE>
__global__ void __launch_bounds__(128) drag_lift_kernel(DragArgs a)
{
    using C = typename Codec<S>::compute;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nbc)
        return;
    uint32_t nodes[8];
    node_slots((uint32_t)a.k[i], a.nbx, a.nby, a.nbz, a.n, a.box, nodes);
    const S *base = static_cast<const S *>(a.dist);
    C fc[27];
    if constexpr (PRE)
        gather_pre<S, EVEN>(base, a.n, nodes, fc);
    else
        gather_post<S, EVEN>(base, a.n, nodes, fc);
    const C *q = static_cast<const C *>(a.q27);
    double f[27], on[27];
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        f[d] = (double)fc[d];
        const C qd = q[(uint64_t)(PRE ? inv(d) : d) * a.nbc + i];
        on[d] = (qd >= C(0) && qd <= C(1)) ? 1.0 : 0.0;
    }
    a.dx[i] = drag_axis(f, on, 0);
    a.dy[i] = drag_axis(f, on, 1);
    a.dz[i] = drag_axis(f, on, 2);
}


// ---------------------------------------------------------------------------------------------
// domain pool: thousands of independent boxes of uneven sizes advanced by one persistent launch
// driven by a work list of node blocks
// ---------------------------------------------------------------------------------------------
template <class C>
struct PoolDomain {
    uint64_t dist_offset;        // elements from the arena start to plane 0 of this domain
    uint64_t pitch;              // elements per direction plane
    uint64_t mask_offset;        // bytes from the arena start to the node mask (nonzero = fluid)
    int nx, ny, nz;
    int flags;                   // bits 0-2: periodic x/y/z, bit 3: has a mask, bit 4: compacted collision
    K17Rates<C> rates;
    C fx, fy, fz;                // half accelerations
    double omega;                // the BC kernels' omega
    uint64_t noslip_offset;      // bytes from the arena start: int32 k[n_noslip]
    uint64_t noslip_cut_offset;  // bytes: uint32 cut[n_noslip] (bit d: q_d in [0, 1]), uint32 first[ceil(n / 32)]
    uint64_t noslip_q_offset;    // bytes: C q[] of the cut links, per 32 nodes direction by direction
                                 // (nodes ascending); first[c] = the links of nodes 0 .. 32 c - 1
    uint64_t noslip_guard_offset; // bytes: uint32 mask[n_noslip], uint32 first[n_noslip] (guarded directions),
                                  // uint32 guarded[n_guarded] (the list positions with a nonzero mask)
    uint64_t noslip_saved_offset; // bytes: C saved[] (their post-collision values, taken before the writes)
    uint64_t pressure_offset;    // bytes: int32 k[n], int32 kN[n], int32 direction[n], then C drho[n]
    uint64_t pressure_rho_offset;
    uint32_t n_noslip, n_pressure, n_guarded;
    FastDiv div_nx, div_ny;      // node k -> (x, y, z) without hardware division
};

// flags of a pool domain; kPoolCompact: the collision queues the fluid nodes of each warp
enum : int { kPoolPeriodicX = 1, kPoolPeriodicY = 2, kPoolPeriodicZ = 4, kPoolMask = 8, kPoolCompact = 16 };

template <class C>
struct PoolArgs {
    void *arena;
    const PoolDomain<C> *domains;
    const uint2 *items;          // {domain, first local node} per node block
    const uint32_t *n_items;     // device word, so a captured step keeps working after list changes
    int nodes_per_thread;
};

// What the collision of a pool domain's nodes needs of its record, read once per work item into
// the block's shared memory: the stores of the node loop may alias the record's global memory as
// far as the compiler can tell, so fields read through a reference to it are loaded again from
// global memory for every node (held in registers instead, they would cost occupancy).
template <class C>
struct PoolNodeCtx {
    uint64_t pitch;
    int nx, ny, nz, flags;
    FastDiv div_nx, div_ny;
    K17Rates<C> rates;
    C fx, fy, fz;
};
template <class C>
__device__ __forceinline__ PoolNodeCtx<C> load_pool_ctx(const PoolDomain<C> *p)
{
    PoolNodeCtx<C> c;
    c.pitch = __ldg(&p->pitch);
    c.nx = __ldg(&p->nx);
    c.ny = __ldg(&p->ny);
    c.nz = __ldg(&p->nz);
    c.flags = __ldg(&p->flags);
    c.div_nx.m = __ldg(&p->div_nx.m);
    c.div_nx.shift = __ldg(&p->div_nx.shift);
    c.div_ny.m = __ldg(&p->div_ny.m);
    c.div_ny.shift = __ldg(&p->div_ny.shift);
    static_assert(sizeof(K17Rates<C>) % sizeof(C) == 0, "K17Rates holds values of its type only");
    const C *src = reinterpret_cast<const C *>(&p->rates);
    C *dst = reinterpret_cast<C *>(&c.rates);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(K17Rates<C>) / sizeof(C)); ++i)
        dst[i] = __ldg(src + i);
    c.fx = __ldg(&p->fx);
    c.fy = __ldg(&p->fy);
    c.fz = __ldg(&p->fz);
    return c;
}

// one node of a pool domain: its slots, the K17 collision and the ET scatter
template <class S, bool EXACT, bool EVEN>
__device__ __forceinline__ void pool_collide_node(S *base, const PoolNodeCtx<typename Codec<S>::compute> &dm, uint32_t k)
{
    using C = typename Codec<S>::compute;
    const int nx = dm.nx, ny = dm.ny, nz = dm.nz, flags = dm.flags;
    const uint32_t yz = fast_div(k, dm.div_nx), x = k - yz * (uint32_t)nx;
    const uint32_t z = fast_div(yz, dm.div_ny), y = yz - z * (uint32_t)ny;
    const int xp = ((int)x + 1 < nx) ? (int)x + 1 : ((flags & kPoolPeriodicX) ? 0 : (int)x);
    const int yp = ((int)y + 1 < ny) ? (int)y + 1 : ((flags & kPoolPeriodicY) ? 0 : (int)y);
    const int zp = ((int)z + 1 < nz) ? (int)z + 1 : ((flags & kPoolPeriodicZ) ? 0 : (int)z);
    const uint32_t sx = (uint32_t)(xp - (int)x);
    const uint32_t sy = (uint32_t)((yp - (int)y) * nx);
    const uint32_t sz = (uint32_t)((int64_t)(zp - (int)z) * nx * ny);
    uint32_t nodes[8];
    nodes[0] = k;
    nodes[1] = k + sx;
    nodes[2] = k + sy;
    nodes[3] = k + sx + sy;
    nodes[4] = k + sz;
    nodes[5] = k + sx + sz;
    nodes[6] = k + sy + sz;
    nodes[7] = k + sx + sy + sz;
    C f[27];
    gather_pre<S, EVEN>(base, dm.pitch, nodes, f);
    C drho, vx, vy, vz;
    collide<C, EXACT>(f, dm.rates, dm.fx, dm.fy, dm.fz, drho, vx, vy, vz);
    scatter_post<S, EVEN>(base, dm.pitch, nodes, f);
}

// The pool's collision: a persistent grid over {domain, first node} items of blockDim x
// nodes_per_thread nodes. Warp w of a block owns the 32-node segments it.y + w 32 + j blockDim.
// By default every lane collides its node of each segment, skipping solid nodes. In a domain
// flagged kPoolCompact (porous media, where most segments mix fluid and solid nodes) the warp
// queues the fluid nodes of its segments in shared memory (a ballot per segment, in node order)
// and collides them 32 at a time, so lanes are not left idle on solid nodes. Each node's arithmetic
// is the same either way.
// two resident blocks of 256 threads (or four of 128) for the FP32-arithmetic forms: at most 128
// registers, the budget every FP32 collision fits without spills; FP64 takes what it needs
template <class S>
constexpr int pool_min_blocks() { return sizeof(typename Codec<S>::compute) == 8 ? 1 : 2; }

template <class S, bool EXACT, bool EVEN>
__global__ void __launch_bounds__(256, pool_min_blocks<S>()) k17_pool_kernel(PoolArgs<typename Codec<S>::compute> a)
{
    using C = typename Codec<S>::compute;
    __shared__ uint32_t queue[8][64];
    __shared__ PoolNodeCtx<C> ctx;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lanes_below = (1u << lane) - 1u;
    const uint32_t n_items = __ldg(a.n_items);
    const uint32_t span = blockDim.x * (uint32_t)a.nodes_per_thread;
    for (uint32_t w = blockIdx.x; w < n_items; w += gridDim.x) {
        const uint2 it = a.items[w];
        const PoolDomain<C> *dp = a.domains + it.x;
        __syncthreads();                 // every thread is done with the previous item's record
        if (threadIdx.x == 0)
            ctx = load_pool_ctx(dp);
        __syncthreads();
        const PoolNodeCtx<C> &dm = ctx;
        const uint32_t nodes_total = (uint32_t)dm.nx * (uint32_t)dm.ny * (uint32_t)dm.nz;
        S *base = static_cast<S *>(a.arena) + __ldg(&dp->dist_offset);
        const uint32_t end = min(it.y + span, nodes_total);
        const uint8_t *mask =
            (dm.flags & kPoolMask) ? static_cast<const uint8_t *>(a.arena) + __ldg(&dp->mask_offset) : nullptr;
        if (!(dm.flags & kPoolCompact)) {
#pragma unroll 1
            for (uint32_t k = it.y + threadIdx.x; k < end; k += blockDim.x) {
                if (mask && __ldg(mask + k) == 0)
                    continue;
                pool_collide_node<S, EXACT, EVEN>(base, dm, k);
            }
            continue;
        }
        uint32_t *q = queue[warp];
        uint32_t pending = 0;            // queued fluid nodes (the same in every lane)
#pragma unroll 1
        for (uint32_t seg = it.y + 32u * warp; seg < end; seg += blockDim.x) {
            const uint32_t k = seg + lane;
            const bool fluid = k < end && __ldg(mask + k) != 0;
            const uint32_t ballot = __ballot_sync(0xffffffffu, fluid);
            if (fluid)
                q[pending + __popc(ballot & lanes_below)] = k;
            pending += __popc(ballot);
            __syncwarp();
            if (pending >= 32u) {
                pool_collide_node<S, EXACT, EVEN>(base, dm, q[lane]);
                pending -= 32u;
                const uint32_t rest = lane < pending ? q[32u + lane] : 0u;
                __syncwarp();
                if (lane < pending)
                    q[lane] = rest;
                __syncwarp();
            }
        }
        if (lane < pending)
            pool_collide_node<S, EXACT, EVEN>(base, dm, q[lane]);
        __syncwarp();
    }
}


// FP64 mass sum(1 + drho) of the fluid nodes of every work item of a pool, one block per item, at
// the parity the next step reads (the watchdog's reduction: a non-finite population makes the sum
// non-finite). Fixed order within a block: per-thread sums, warp shuffles, then the warps in order.
template <class S, bool EVEN>
__global__ void __launch_bounds__(256) pool_mass_kernel(PoolArgs<typename Codec<S>::compute> a, double *partials)
{
    using C = typename Codec<S>::compute;
    const uint2 it = a.items[blockIdx.x];
    const PoolDomain<C> &dm = a.domains[it.x];
    const uint32_t nodes_total = (uint32_t)dm.nx * (uint32_t)dm.ny * (uint32_t)dm.nz;
    const uint32_t span = blockDim.x * (uint32_t)a.nodes_per_thread;
    const uint32_t end = min(it.y + span, nodes_total);
    const S *base = static_cast<const S *>(a.arena) + dm.dist_offset;
    const uint8_t *mask = (dm.flags & kPoolMask) ? static_cast<const uint8_t *>(a.arena) + dm.mask_offset : nullptr;
    const NodeAddr box{ dm.nx, dm.ny, dm.nz, dm.flags & 7 };
    double m = 0.0;
    for (uint32_t k = it.y + threadIdx.x; k < end; k += blockDim.x) {
        if (mask && __ldg(mask + k) == 0)
            continue;
        uint32_t nodes[8];
        box_nodes(k, box, nodes);
        C f[27];
        gather_pre<S, EVEN>(base, dm.pitch, nodes, f);
        m += 1.0 + (double)density_pyramid(f);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        m += __shfl_down_sync(0xffffffffu, m, o);
    __shared__ double warp_sums[8];
    if ((threadIdx.x & 31) == 0)
        warp_sums[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (unsigned w = 0; w < (blockDim.x + 31) / 32; ++w)
            t += warp_sums[w];
        partials[blockIdx.x] = t;
    }
}

// The boundary conditions of every domain of a pool, one launch per kind: a persistent grid over
// {domain, first BC node} items of 128 BC nodes. No-slip: NoSlipInterpolatedCompressible after the
// collision (current parity); pressure: PressureNonEquilibriumCompressible after the parity swap.
// Box addressing per domain, as the structured box's BC lists.
template <class C>
struct PoolBCArgs {
    void *arena;
    const PoolDomain<C> *domains;
    const uint2 *items;
    const uint32_t *n_items;
};

// Links cut from both ends (two BC nodes of one list joined by a link that clips the geometry):
// each node's write lands in the slot the other reads. Before the no-slip kernel writes anything,
// the values in those slots (bit d of a node's mask: its post-collision population d) are saved,
// and the no-slip kernel reads them from there, so every node sees the collision's values. The
// work list runs over the guarded nodes only ({domain, first position in guarded[]} items).
template <class S, bool EVEN>
__global__ void __launch_bounds__(128) pool_noslip_guard_kernel(PoolBCArgs<typename Codec<S>::compute> a)
{
    using C = typename Codec<S>::compute;
    const uint32_t n_items = __ldg(a.n_items);
    for (uint32_t w = blockIdx.x; w < n_items; w += gridDim.x) {
        const uint2 it = a.items[w];
        const PoolDomain<C> &dm = a.domains[it.x];
        const uint32_t g = it.y + threadIdx.x;
        if (g >= dm.n_guarded)
            continue;
        char *arena = static_cast<char *>(a.arena);
        const uint32_t *guard = reinterpret_cast<const uint32_t *>(arena + dm.noslip_guard_offset);
        const uint32_t i = guard[2ull * dm.n_noslip + g];
        const uint32_t mask = guard[i];
        const int32_t *k = reinterpret_cast<const int32_t *>(arena + dm.noslip_offset);
        C *saved = reinterpret_cast<C *>(arena + dm.noslip_saved_offset) + guard[dm.n_noslip + i];
        const NodeAddr box{ dm.nx, dm.ny, dm.nz, dm.flags & 7 };
        uint32_t nodes[8];
        box_nodes((uint32_t)k[i], box, dm.div_nx, dm.div_ny, nodes);
        const S *base = static_cast<const S *>(a.arena) + dm.dist_offset;
        int r = 0;
#pragma unroll
        for (int d = 1; d < 27; ++d)
            if ((mask >> d) & 1u)
                saved[r++] = Codec<S>::load(base + (uint64_t)plane<EVEN>(inv(d)) * dm.pitch + nodes[shift_class(inv(d))], d);
    }
}

// Interpolated no-slip over the pool's lists, one warp per 32 BC nodes, in two phases.
//   nodes: lane i gathers node i's post-collision populations (guarded ones from the saved copy),
//          forms its moments, and puts both with its slot nodes in the warp's shared memory;
//   links: the warp's cut links (node, direction), listed direction by direction with the nodes
//          ascending, are spread over the lanes, each computing and storing one link's value.
// Every lane does useful work in the second phase, where a thread per node would step through all
// 26 directions with the lanes of uncut ones idle. The arithmetic is bc_moments / bc_link_value,
// as in bc_interpolated_node, so the values are the same bits.
constexpr int kLinkWarps = 4;        // warps per block of the link kernel
constexpr int kLinkRow = 33;         // padded row of the shared tables (a link's node and direction spread its bank)

template <class C>
struct LinkTile {
    C p[27 * kLinkRow];
    C m[5 * 32];                     // drho, ux, uy, uz, cu_sq
    uint32_t nodes[8 * kLinkRow];
    uint16_t links[32 * 26];         // lane | direction << 5
};

// resident blocks per SM: 8 for FP32 storage (64 registers; 8 shared tiles fit), 7 for the 16-bit
// forms, 4 for FP64 (its tiles are twice as large)
template <class S, bool EVEN>
__global__ void __launch_bounds__(128, sizeof(S) == 8 ? 4 : (sizeof(S) == 4 ? 8 : 7))
    pool_noslip_kernel(PoolBCArgs<typename Codec<S>::compute> a)
{
    using C = typename Codec<S>::compute;
    __shared__ LinkTile<C> tiles[kLinkWarps];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    LinkTile<C> &t = tiles[warp];
    const uint32_t n_items = __ldg(a.n_items);
    for (uint32_t w = blockIdx.x; w < n_items; w += gridDim.x) {
        const uint2 it = a.items[w];
        const PoolDomain<C> &dm = a.domains[it.x];
        const uint32_t i0 = it.y + 32u * warp;
        if (i0 >= dm.n_noslip)
            continue;
        const char *arena = static_cast<const char *>(a.arena);
        S *base = static_cast<S *>(a.arena) + dm.dist_offset;
        const uint32_t *cut_mask = reinterpret_cast<const uint32_t *>(arena + dm.noslip_cut_offset);
        const uint32_t i = i0 + lane;
        uint32_t cut = 0;
        if (i < dm.n_noslip) {
            const int32_t *k = reinterpret_cast<const int32_t *>(arena + dm.noslip_offset);
            const uint32_t *guard = reinterpret_cast<const uint32_t *>(arena + dm.noslip_guard_offset);
            const NodeAddr box{ dm.nx, dm.ny, dm.nz, dm.flags & 7 };
            uint32_t nodes[8];
            box_nodes((uint32_t)k[i], box, dm.div_nx, dm.div_ny, nodes);
            cut = cut_mask[i];
            const uint32_t gm = guard[i];
            C p[27];
            gather_post<S, EVEN>(base, dm.pitch, nodes, p);
            if (gm) {
                const C *saved = reinterpret_cast<const C *>(arena + dm.noslip_saved_offset) + guard[dm.n_noslip + i];
                int r = 0;
#pragma unroll
                for (int d = 1; d < 27; ++d)
                    if ((gm >> d) & 1u)
                        p[d] = saved[r++];
            }
            const BCMoments<C> m = bc_moments<C, kBCCompressible>(p);
#pragma unroll
            for (int d = 0; d < 27; ++d)
                t.p[d * kLinkRow + lane] = p[d];
#pragma unroll
            for (int c = 0; c < 8; ++c)
                t.nodes[c * kLinkRow + lane] = nodes[c];
            t.m[0 * 32 + lane] = m.drho;
            t.m[1 * 32 + lane] = m.ux;
            t.m[2 * 32 + lane] = m.uy;
            t.m[3 * 32 + lane] = m.uz;
            t.m[4 * 32 + lane] = m.cu_sq;
        }
        // the warp's link list, direction by direction and the nodes in order within a direction
        // (the order of the link q in the arena): 32 consecutive links mostly share a direction,
        // so their shared-memory rows are read from distinct banks and their stores land in one
        // plane at neighbouring nodes
        const uint32_t lanes_below = (1u << lane) - 1u;
        uint32_t total = 0;
#pragma unroll
        for (int d = 1; d < 27; ++d) {
            const bool has = (cut >> d) & 1u;
            const uint32_t ballot = __ballot_sync(0xffffffffu, has);
            if (has)
                t.links[total + __popc(ballot & lanes_below)] = (uint16_t)(lane | ((uint32_t)d << 5));
            total += __popc(ballot);
        }
        __syncwarp();
        const C *q = reinterpret_cast<const C *>(arena + dm.noslip_q_offset) + cut_mask[dm.n_noslip + i0 / 32u];
        const C omega = (C)dm.omega;
        for (uint32_t l = lane; l < total; l += 32u) {
            const uint32_t e = t.links[l];
            const uint32_t nl = e & 31u;
            const int d = (int)(e >> 5);
            const int di = inv(d);
            BCMoments<C> m;
            m.drho = t.m[0 * 32 + nl];
            m.ux = t.m[1 * 32 + nl];
            m.uy = t.m[2 * 32 + nl];
            m.uz = t.m[3 * 32 + nl];
            m.cu_sq = t.m[4 * 32 + nl];
            const C v = bc_link_value<C, false, kBCCompressible>(t.p[d * kLinkRow + nl], t.p[di * kLinkRow + nl], q[l],
                                                                 weight_rt<C>(d), cdot_link<C>(d, m.ux, m.uy, m.uz), C(0),
                                                                 m, omega);
            Codec<S>::store_at_rt(base, (uint64_t)plane<!EVEN>(di) * dm.pitch + t.nodes[shift_class_rt(di) * kLinkRow + nl],
                                  v, di);
        }
        __syncwarp();
    }
}

template <class S, bool EVEN>
__global__ void __launch_bounds__(128) pool_pressure_kernel(PoolBCArgs<typename Codec<S>::compute> a)
{
    using C = typename Codec<S>::compute;
    const uint32_t n_items = __ldg(a.n_items);
    for (uint32_t w = blockIdx.x; w < n_items; w += gridDim.x) {
        const uint2 it = a.items[w];
        const PoolDomain<C> &dm = a.domains[it.x];
        const uint32_t i = it.y + threadIdx.x;
        if (i >= dm.n_pressure)
            continue;
        const char *arena = static_cast<const char *>(a.arena);
        const int32_t *k = reinterpret_cast<const int32_t *>(arena + dm.pressure_offset);
        const int32_t *kn = k + dm.n_pressure;
        const int32_t *dir = kn + dm.n_pressure;
        const C *rho = reinterpret_cast<const C *>(arena + dm.pressure_rho_offset);
        const NodeAddr box{ dm.nx, dm.ny, dm.nz, dm.flags & 7 };
        uint32_t nk[8], nn[8];
        box_nodes((uint32_t)k[i], box, nk);
        box_nodes((uint32_t)kn[i], box, nn);
        bc_pressure_neq_node<S, EVEN, false>(static_cast<S *>(a.arena) + dm.dist_offset, dm.pitch, nk, nn, rho[i],
                                             dir[i]);
    }
}

// ---------------------------------------------------------------------------------------------
// seeded per-step perturbation of a velocity inlet: u_i(t) = u0_i (1 + a (2 U - 1)), U uniform in
// [0, 1) from the counter-based Philox-4x32-10 generator (Salmon et al., SC'11) keyed by the seed,
// counted by (node, step)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mulhilo(uint32_t a, uint32_t b, uint32_t &hi)
{
    const uint64_t p = (uint64_t)a * b;
    hi = (uint32_t)(p >> 32);
    return (uint32_t)p;
}

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, hi1;
        const uint32_t lo0 = mulhilo(0xD2511F53u, c.x, hi0);
        const uint32_t lo1 = mulhilo(0xCD9E8D57u, c.z, hi1);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

template <class C>
__global__ void __launch_bounds__(256) inlet_perturbation_kernel(const C *base_x, const C *base_y, const C *base_z,
                                                                 C *ux, C *uy, C *uz, uint32_t n, uint64_t seed,
                                                                 uint64_t step, double amplitude)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint4 r = philox4x32_10(make_uint4(i, (uint32_t)step, (uint32_t)(step >> 32), 0u),
                                  make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    const double u01 = (double)r.x * (1.0 / 4294967296.0);
    const C factor = (C)(1.0 + amplitude * (2.0 * u01 - 1.0));
    ux[i] = base_x[i] * factor;
    uy[i] = base_y[i] * factor;
    uz[i] = base_z[i] * factor;
}

} // namespace VFB_NS
} // namespace vfb
