// Host-side launch layer between the C ABI (abi.cu) and the device kernels (kernels.cuh).
//
// The kernels are compiled in one translation unit per (arithmetic variant, storage type);
// each unit defines Launchers<S> of its variant namespace. abi.cu dispatches on the runtime
// storage and arithmetic choice.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>

#include "addr.h"
#include "vfb.h"

namespace vfb {
struct e3m12_t; // the E3M12 storage element (storage.cuh)

// an NVTX range for the lifetime of the object (the steps of boxes and pools, for ncu --nvtx and
// other NVTX tools; a no-op without one attached)
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
} // namespace vfb

namespace vfb {

// a structured box as the kernels see it
struct BoxState {
    void *dist;
    uint64_t pitch;               // elements per direction plane
    int nx, ny, nz;
    int periodic_x, periodic_y, periodic_z;
    const uint8_t *mask;          // device, nullable
    double omega;
    double fx, fy, fz;            // half acceleration
    double lim[3];
    int variant;                  // 0: choose, 1: direct loads, 2: TMA-staged (nx % 32 == 0), 3: async copies
    int async_blocks_per_sm;      // async kernel: resident blocks per SM (0: 3)
    int async_smem_kb;            // async kernel: shared-memory configuration to pad to (0: carve-out hint only)
    int *status;                  // device status word (DeviceError), nullable
};

// block shape of the box kernels: x extent of a block (multiple of 32, at most 128)
inline int box_block_x(int nx)
{
    int b = ((nx + 31) / 32) * 32;
    return b > 128 ? 128 : b;
}
// upper bound of the per-step energy partials any box kernel writes (one per warp of the direct
// kernel's grid; the persistent kernels write fewer)
inline uint64_t box_blocks(const BoxState &b)
{
    const int bx = box_block_x(b.nx);
    return (uint64_t)((b.nx + bx - 1) / bx) * (uint64_t)b.ny * (uint64_t)b.nz * (uint64_t)(bx / 32);
}

// a pool domain's record as the host describes it (offsets in bytes from the arena start, except
// dist_offset in elements)
struct PoolDomainSpec {
    uint64_t dist_offset, pitch, mask_offset;
    int nx, ny, nz, flags;
    double omega;
    double lim[3];
    double half_force[3];
    uint64_t noslip_offset, noslip_cut_offset, noslip_q_offset, noslip_guard_offset, noslip_saved_offset,
        pressure_offset, pressure_rho_offset;
    uint32_t n_noslip, n_guarded, n_pressure;
};

#define VFB_DECLARE_LAUNCHERS                                                                                        \
    template <class S>                                                                                               \
    struct Launchers {                                                                                               \
        static cudaError_t k17_list(const vfb_level *L, const uint32_t *idx, uint32_t n, int tmpl, cudaStream_t s,   \
                                    const uint32_t *slots = nullptr, uint64_t slots_stride = 0);             \
        static cudaError_t k17_list_staged(const vfb_level *L, const uint32_t *slots, uint64_t slots_stride,       \
                                           uint32_t n, int *status, cudaStream_t s);                               \
        static cudaError_t bc(const vfb_level *L, const vfb_bc *bc, int kind, cudaStream_t s,                        \
                              const NodeAddr *box = nullptr, void *snap = nullptr,                                   \
                              const uint32_t *guard = nullptr, void *saved = nullptr);                               \
        static cudaError_t pressure(const vfb_level *L, const vfb_directional_bc *bc, cudaStream_t s,                \
                                    const NodeAddr *box = nullptr, int kind = 0);                                    \
        static cudaError_t inlet_perturbation(const void *base, void *vel, uint32_t n, uint64_t seed,                \
                                              uint64_t step, double amplitude, cudaStream_t s);                      \
        static cudaError_t init_list(const vfb_level *L, cudaStream_t s);                                          \
        static cudaError_t init_neq_list(const vfb_level *L, const uint32_t *nb_inverse, cudaStream_t s);          \
        static cudaError_t macros_list(const vfb_level *L, cudaStream_t s);                                        \
        static cudaError_t energy_list(const vfb_level *L, const uint32_t *idx, uint32_t n, double *partials,     \
                                       cudaStream_t s);                                                            \
        static cudaError_t box_collide(const BoxState &b, bool even, double *partials, uint64_t *n_partials,        \
                                       cudaStream_t s);                                                            \
        static cudaError_t box_collide_planes(const BoxState &b, bool even, int z0, int z1, cudaStream_t s);       \
        static cudaError_t box_collide_border(const BoxState &b, bool even, int z, void *up, void *down,           \
                                              cudaStream_t s);                                                     \
        static cudaError_t box_init(const BoxState &b, bool even, const void *rho, const void *ux, const void *uy, \
                                    const void *uz, cudaStream_t s);                                               \
        static cudaError_t box_macros(const BoxState &b, bool even, void *rho, void *ux, void *uy, void *uz,       \
                                      cudaStream_t s);                                                             \
        static cudaError_t pool_collide(void *arena, const void *domains, const uint2 *items,                      \
                                        const uint32_t *n_items, int nodes_per_thread, bool even, unsigned grid,   \
                                        unsigned block, cudaStream_t s);                                           \
        static const void *pool_kernel(bool even);                                                                \
        static size_t pool_domain_bytes();                                                                        \
        static void pool_domain(void *out, const PoolDomainSpec &spec);                                            \
        static cudaError_t pool_mass(void *arena, const void *domains, const uint2 *items, uint32_t n_items,       \
                                     int nodes_per_thread, int threads, bool even, double *partials,              \
                                     cudaStream_t s);                                                              \
        static cudaError_t pool_bcs(void *arena, const void *domains, const uint2 *noslip_items,                   \
                                    const uint32_t *n_noslip_items, const uint2 *guard_items,                      \
                                    const uint32_t *n_guard_items, const uint2 *pressure_items,                    \
                                    const uint32_t *n_pressure_items, bool even, unsigned grid, cudaStream_t s);   \
        static cudaError_t drag_lift(const vfb_level *L, const vfb_bc *bc, bool pre, double *dx, double *dy,        \
                                     double *dz, cudaStream_t s, const NodeAddr *box = nullptr);                     \
        static cudaError_t bounds_error(uint64_t *record);                                                        \
        static cudaError_t scale(const vfb_level *coarse, const vfb_level *fine, const vfb_interpolation_cells *cells, \
                                 const vfb_interpolation_cell_neighbor *offsets, bool fine_to_coarse, cudaStream_t s); \
    };

// BC kinds of Launchers::bc
enum BCKind : int { kNoSlipBB = 0, kNoSlipInterp = 1, kVelocityBB = 2, kVelocityInterp = 3, kNoSlipInterpIncomp = 4,
                    kVelocityInterpIncomp = 5, kVelocityWithPressure = 6, kSlipInterp = 7 };
// pressure-list kernels of Launchers::pressure
enum PressureKind : int { kPressureNeqComp = 0, kPressureNeqIncomp = 1, kOutflowNonReflecting = 2,
                          kOutflowPressureCorrection = 3 };

namespace fast {
VFB_DECLARE_LAUNCHERS
}
namespace exact {
VFB_DECLARE_LAUNCHERS
}

// message for vfb_last_error() of the calling thread
void set_last_error(const char *msg);
// the argument checks every reference-layout entry point applies to a level (VFB_OK or the status,
// with the message set)
int check_level_status(const vfb_level *level);
// VFB_OK for cudaSuccess, else the status the entry points report for e (out of memory or a CUDA
// error), with "what: <CUDA message>" as the message
int cuda_error_status(cudaError_t e, const char *what);

// deterministic reduction of per-block {mass, energy} partials into out[2] (device)
cudaError_t reduce_partials(const double *partials, uint64_t blocks, double *out, cudaStream_t s);
// calcDragLift's sum of pre - post over n nodes (x, y, z arrays of n doubles each) into out[3]
// on the device; scratch holds 3 * ceil(n / 256) doubles; a fixed order for a given n
cudaError_t drag_lift_sum(const double *const pre[3], const double *const post[3], uint32_t n, double *scratch,
                          double *out, cudaStream_t s);

// the same for many partials: up to kReduceMaxChunks blocks reduce contiguous chunks into scratch
// (2 * kReduceMaxChunks doubles), one block reduces those; a fixed order for a given count
constexpr uint64_t kReduceDirect = 8192, kReduceMaxChunks = 1024;
cudaError_t reduce_partials_wide(const double *partials, uint64_t blocks, double *scratch, double *out, cudaStream_t s);

} // namespace vfb
