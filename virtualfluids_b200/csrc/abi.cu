// C ABI of the library (include/vfb.h): argument checks, dispatch on storage and arithmetic,
// the kernel and boundary-condition registries, the step driver and structured boxes.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "guards.h"
#include "k17.cuh"
#include "launch.h"
#include "vfb.h"

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string &msg)
{
    g_last_error = msg;
    return status;
}

int cuda_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess)
        return VFB_OK;
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? VFB_ERR_OUT_OF_MEMORY : VFB_ERR_CUDA;
}

inline cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }

bool storage_ok(int s) { return s >= VFB_STORAGE_F64 && s <= VFB_STORAGE_E3M12; }
size_t storage_bytes(int s) { return s == VFB_STORAGE_F64 ? 8 : s == VFB_STORAGE_F32 ? 4 : 2; }
size_t real_bytes(int s) { return s == VFB_STORAGE_F64 ? 8 : 4; }

int check_level(const vfb_level *L)
{
    if (!L)
        return fail(VFB_ERR_INVALID_ARGUMENT, "level is NULL");
    if (!storage_ok(L->storage))
        return fail(VFB_ERR_INVALID_ARGUMENT, "unknown storage format");
    if (L->arith != VFB_ARITH_FAST && L->arith != VFB_ARITH_EXACT)
        return fail(VFB_ERR_INVALID_ARGUMENT, "unknown arithmetic mode");
    if (L->arith == VFB_ARITH_EXACT && L->storage > VFB_STORAGE_F32)
        return fail(VFB_ERR_UNSUPPORTED, "exact arithmetic is built for F64 and F32 storage only");
    if (!L->distributions || !L->neighbor_x || !L->neighbor_y || !L->neighbor_z)
        return fail(VFB_ERR_INVALID_ARGUMENT, "level distributions or neighbour lists are NULL");
    if (L->number_of_nodes == 0 || L->number_of_nodes > 0xffffffffull)
        return fail(VFB_ERR_INVALID_ARGUMENT, "number_of_nodes must be in [1, 2^32)");
    if (!(L->omega > 0.0 && L->omega < 2.0))
        return fail(VFB_ERR_INVALID_ARGUMENT, "omega must lie in (0, 2)");
    return VFB_OK;
}

// call F with Launchers<S> of the chosen variant
#define VFB_DISPATCH(storage, arith, CALL)                                                                            \
    [&]() -> cudaError_t {                                                                                             \
        if ((arith) == VFB_ARITH_EXACT) {                                                                              \
            switch (storage) {                                                                                         \
            case VFB_STORAGE_F64: { using LA = vfb::exact::Launchers<double>; return CALL; }                            \
            case VFB_STORAGE_F32: { using LA = vfb::exact::Launchers<float>; return CALL; }                             \
            default: return cudaErrorInvalidValue;                                                                     \
            }                                                                                                          \
        }                                                                                                              \
        switch (storage) {                                                                                             \
        case VFB_STORAGE_F64: { using LA = vfb::fast::Launchers<double>; return CALL; }                                 \
        case VFB_STORAGE_F32: { using LA = vfb::fast::Launchers<float>; return CALL; }                                  \
        case VFB_STORAGE_F16: { using LA = vfb::fast::Launchers<__half>; return CALL; }                                 \
        case VFB_STORAGE_BF16: { using LA = vfb::fast::Launchers<__nv_bfloat16>; return CALL; }                         \
        case VFB_STORAGE_E3M12: { using LA = vfb::fast::Launchers<vfb::e3m12_t>; return CALL; }                         \
        default: return cudaErrorInvalidValue;                                                                         \
        }                                                                                                              \
    }()

struct KernelEntry {
    const char *name;
    int id;
};
// Kernel/KernelTypes.h:35-46 lists the reference's names; this build registers K17 (TurbulenceModel::None)
const KernelEntry kKernels[] = { { "K17CompressibleNavierStokes", VFB_KERNEL_K17_COMPRESSIBLE_NAVIER_STOKES } };

} // namespace

// ---------------------------------------------------------------------------------------------
// deterministic partial-sum reduction
// ---------------------------------------------------------------------------------------------
namespace vfb {
// block g sums the partial pairs [g * chunk, min((g + 1) * chunk, blocks)) into out[2g], out[2g + 1]:
// each thread strides through the chunk, then a fixed shared-memory tree (blockDim a power of two)
__global__ void __launch_bounds__(1024) reduce_partials_kernel(const double *__restrict__ p, uint64_t blocks,
                                                               uint64_t chunk, double *out)
{
    __shared__ double sm[2][1024];
    const uint64_t lo = blockIdx.x * chunk, hi = lo + chunk < blocks ? lo + chunk : blocks;
    double m = 0.0, e = 0.0;
    for (uint64_t b = lo + threadIdx.x; b < hi; b += blockDim.x) {
        m += p[2 * b];
        e += p[2 * b + 1];
    }
    sm[0][threadIdx.x] = m;
    sm[1][threadIdx.x] = e;
    __syncthreads();
    for (unsigned s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sm[0][threadIdx.x] += sm[0][threadIdx.x + s];
            sm[1][threadIdx.x] += sm[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * blockIdx.x] = sm[0][0];
        out[2 * blockIdx.x + 1] = sm[1][0];
    }
}

// calcDragLift (DragLift.cpp:66-73): per block, the sums of pre - post over its nodes (three
// doubles, a fixed shared-memory tree); a second pass adds the blocks in order
struct DragSumArgs {
    const double *pre[3], *post[3];
};

__global__ void __launch_bounds__(256) drag_lift_sum_kernel(DragSumArgs a, uint32_t n, double *partials)
{
    __shared__ double sm[3][256];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        sm[c][threadIdx.x] = i < n ? a.pre[c][i] - a.post[c][i] : 0.0;
    __syncthreads();
    for (unsigned s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                sm[c][threadIdx.x] += sm[c][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 3)
        partials[3 * blockIdx.x + threadIdx.x] = sm[threadIdx.x][0];
}

__global__ void __launch_bounds__(256) drag_lift_total_kernel(const double *__restrict__ partials, uint32_t blocks,
                                                              double *out)
{
    __shared__ double sm[3][256];
    double acc[3] = { 0.0, 0.0, 0.0 };
    for (uint32_t b = threadIdx.x; b < blocks; b += blockDim.x)
#pragma unroll
        for (int a = 0; a < 3; ++a)
            acc[a] += partials[3 * b + a];
#pragma unroll
    for (int a = 0; a < 3; ++a)
        sm[a][threadIdx.x] = acc[a];
    __syncthreads();
    for (unsigned s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
#pragma unroll
            for (int a = 0; a < 3; ++a)
                sm[a][threadIdx.x] += sm[a][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 3)
        out[threadIdx.x] = sm[threadIdx.x][0];
}

cudaError_t drag_lift_sum(const double *const pre[3], const double *const post[3], uint32_t n, double *scratch,
                          double *out, cudaStream_t s)
{
    const uint32_t blocks = (n + 255u) / 256u;
    if (blocks == 0)
        return cudaMemsetAsync(out, 0, 3 * sizeof(double), s);
    DragSumArgs a;
    for (int c = 0; c < 3; ++c) {
        a.pre[c] = pre[c];
        a.post[c] = post[c];
    }
    drag_lift_sum_kernel<<<blocks, 256, 0, s>>>(a, n, scratch);
    drag_lift_total_kernel<<<1, 256, 0, s>>>(scratch, blocks, out);
    return cudaGetLastError();
}

void set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

int check_level_status(const vfb_level *level) { return check_level(level); }
int cuda_error_status(cudaError_t e, const char *what) { return cuda_status(e, what); }

cudaError_t reduce_partials(const double *partials, uint64_t blocks, double *out, cudaStream_t s)
{
    reduce_partials_kernel<<<1, 1024, 0, s>>>(partials, blocks, blocks, out);
    return cudaGetLastError();
}

cudaError_t reduce_partials_wide(const double *partials, uint64_t blocks, double *scratch, double *out, cudaStream_t s)
{
    if (blocks <= kReduceDirect)
        return reduce_partials(partials, blocks, out, s);
    const uint64_t g = std::min<uint64_t>(kReduceMaxChunks, (blocks + 2047) / 2048);
    const uint64_t chunk = (blocks + g - 1) / g;
    reduce_partials_kernel<<<(unsigned)g, 256, 0, s>>>(partials, blocks, chunk, scratch);
    reduce_partials_kernel<<<1, 1024, 0, s>>>(scratch, g, g, out);
    return cudaGetLastError();
}
} // namespace vfb

// ---------------------------------------------------------------------------------------------
// library
// ---------------------------------------------------------------------------------------------
extern "C" {

int vfb_abi_version(void) { return VFB_ABI_VERSION; }

const char *vfb_last_error(void) { return g_last_error.c_str(); }

const char *vfb_status_string(int status)
{
    switch (status) {
    case VFB_OK: return "ok";
    case VFB_ERR_INVALID_ARGUMENT: return "invalid argument";
    case VFB_ERR_UNKNOWN_KERNEL: return "KernelFactory does not know the KernelType.";
    case VFB_ERR_BC_UNSET: return "a boundary condition has nodes but no kernel";
    case VFB_ERR_SCALING_UNSET: return "more than one level but no grid scaling kernel";
    case VFB_ERR_CUDA: return "CUDA error";
    case VFB_ERR_OUT_OF_MEMORY: return "out of device memory";
    case VFB_ERR_UNSUPPORTED: return "not supported by this build";
    case VFB_ERR_WATCHDOG: return "non-finite populations or mass drift";
    default: return "unknown status";
    }
}

int vfb_bounds_checked(void)
{
#ifdef VFB_BOUNDS_CHECK
    return 1;
#else
    return 0;
#endif
}

int vfb_bounds_check_status(uint64_t *bad_index, uint64_t *node_count)
{
    if (!bad_index || !node_count)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *bad_index = 0;
    *node_count = 0;
#ifndef VFB_BOUNDS_CHECK
    return fail(VFB_ERR_UNSUPPORTED, "this library is built without bounds checks (libvfb_checked.so has them)");
#else
    cudaError_t e = cudaDeviceSynchronize();
    uint64_t recs[7] = {};
    if (e == cudaSuccess) e = vfb::exact::Launchers<double>::bounds_error(&recs[0]);
    if (e == cudaSuccess) e = vfb::exact::Launchers<float>::bounds_error(&recs[1]);
    if (e == cudaSuccess) e = vfb::fast::Launchers<double>::bounds_error(&recs[2]);
    if (e == cudaSuccess) e = vfb::fast::Launchers<float>::bounds_error(&recs[3]);
    if (e == cudaSuccess) e = vfb::fast::Launchers<__half>::bounds_error(&recs[4]);
    if (e == cudaSuccess) e = vfb::fast::Launchers<__nv_bfloat16>::bounds_error(&recs[5]);
    if (e == cudaSuccess) e = vfb::fast::Launchers<vfb::e3m12_t>::bounds_error(&recs[6]);
    if (e != cudaSuccess)
        return cuda_status(e, "bounds-check record");
    for (uint64_t r : recs)
        if (r) {
            *bad_index = (r & 0xffffffffull) - 1;
            *node_count = r >> 32;
            return fail(VFB_ERR_INVALID_ARGUMENT, "a kernel met a node index beyond its level's node count");
        }
    return VFB_OK;
#endif
}

int vfb_synchronize(void *stream)
{
    return cuda_status(stream ? cudaStreamSynchronize(as_stream(stream)) : cudaDeviceSynchronize(), "synchronize");
}

int vfb_lattice_tables(int32_t cx[27], int32_t cy[27], int32_t cz[27], int32_t inv[27], double w[27])
{
    if (!cx || !cy || !cz || !inv || !w)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL table");
    for (int d = 0; d < 27; ++d) {
        cx[d] = vfb::cx(d);
        cy[d] = vfb::cy(d);
        cz[d] = vfb::cz(d);
        inv[d] = vfb::inv(d);
        w[d] = vfb::weight_t<double>(d);
    }
    return VFB_OK;
}

int vfb_k17_rates(double omega, double rates[6])
{
    if (!rates)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL rates");
    const vfb::K17Rates<double> r = vfb::make_k17_rates<double>(omega, 0.01, 0.01, 0.01);
    rates[0] = r.OxyyPxzz;
    rates[1] = r.OxyyMxzz;
    rates[2] = r.Oxyz;
    rates[3] = r.factorA;
    rates[4] = r.factorB;
    rates[5] = -r.neg_iwm;
    return VFB_OK;
}

int vfb_kernel_lookup(const char *name, int32_t *kernel_id)
{
    if (!name || !kernel_id)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL name or id");
    for (const KernelEntry &e : kKernels)
        if (std::strcmp(e.name, name) == 0) {
            *kernel_id = e.id;
            return VFB_OK;
        }
    return fail(VFB_ERR_UNKNOWN_KERNEL, std::string("KernelFactory does not know the KernelType: ") + name);
}

int vfb_kernel_count(void) { return (int)(sizeof(kKernels) / sizeof(kKernels[0])); }

const char *vfb_kernel_name(int index)
{
    if (index < 0 || index >= vfb_kernel_count())
        return nullptr;
    return kKernels[index].name;
}

// ---------------------------------------------------------------------------------------------
// (1) reference-layout entry points
// ---------------------------------------------------------------------------------------------
static int run_k17(const vfb_level *level, const uint32_t *idx, uint32_t size, int32_t tmpl, const uint32_t *slots,
                   uint64_t slots_stride, void *stream);

int vfb_k17_run_on_indices(const vfb_level *level, const uint32_t *idx, uint32_t size, int32_t tmpl, void *stream)
{
    return run_k17(level, idx, size, tmpl, nullptr, 0, stream);
}

static int run_k17(const vfb_level *level, const uint32_t *idx, uint32_t size, int32_t tmpl, const uint32_t *slots,
                   uint64_t slots_stride, void *stream)
{
    int st = check_level(level);
    if (st)
        return st;
    if (tmpl < VFB_COLLISION_DEFAULT || tmpl > VFB_COLLISION_SUBDOMAIN_BORDER)
        return fail(VFB_ERR_INVALID_ARGUMENT, "Invalid CollisionTemplate");
    if (size && !idx)
        return fail(VFB_ERR_INVALID_ARGUMENT, "fluid node indices are NULL");
    const bool wm = tmpl != VFB_COLLISION_DEFAULT && tmpl != VFB_COLLISION_APPLY_BODY_FORCE;
    const bool bf = tmpl == VFB_COLLISION_APPLY_BODY_FORCE || tmpl == VFB_COLLISION_ALL_FEATURES || tmpl == VFB_COLLISION_SUBDOMAIN_BORDER;
    if (wm && (!level->rho || !level->velocity_x || !level->velocity_y || !level->velocity_z))
        return fail(VFB_ERR_INVALID_ARGUMENT, "macroscopic output arrays are NULL");
    if (bf && (!level->body_force_x || !level->body_force_y || !level->body_force_z))
        return fail(VFB_ERR_INVALID_ARGUMENT, "body force arrays are NULL");
    const cudaError_t e = VFB_DISPATCH(level->storage, level->arith,
                                       LA::k17_list(level, idx, size, tmpl, as_stream(stream), slots, slots_stride));
    return cuda_status(e, "K17CompressibleNavierStokes launch");
}

static int run_bc(const vfb_level *level, const vfb_bc *bc, int kind, bool velocity, void *stream,
                  void *snap = nullptr)
{
    int st = check_level(level);
    if (st)
        return st;
    if (!bc)
        return fail(VFB_ERR_INVALID_ARGUMENT, "bc is NULL");
    if (bc->number_of_bc_nodes && (!bc->k || !bc->q27))
        return fail(VFB_ERR_INVALID_ARGUMENT, "bc node indices or q27 are NULL");
    if (velocity && bc->number_of_bc_nodes && (!bc->vx || !bc->vy || !bc->vz))
        return fail(VFB_ERR_INVALID_ARGUMENT, "bc velocities are NULL");
    const cudaError_t e = VFB_DISPATCH(level->storage, level->arith,
                                       LA::bc(level, bc, kind, as_stream(stream), nullptr, snap));
    return cuda_status(e, "boundary condition launch");
}

int vfb_noslip_bounce_back(const vfb_level *level, const vfb_bc *bc, void *stream)
{
    return run_bc(level, bc, vfb::kNoSlipBB, false, stream);
}
int vfb_noslip_interpolated_compressible(const vfb_level *level, const vfb_bc *bc, void *stream)
{
    return run_bc(level, bc, vfb::kNoSlipInterp, false, stream);
}
int vfb_velocity_bounce_back(const vfb_level *level, const vfb_bc *bc, void *stream)
{
    return run_bc(level, bc, vfb::kVelocityBB, true, stream);
}
int vfb_velocity_interpolated_compressible(const vfb_level *level, const vfb_bc *bc, void *stream)
{
    return run_bc(level, bc, vfb::kVelocityInterp, true, stream);
}

int vfb_slip_compressible(const vfb_level *level, const vfb_bc *bc, void *stream)
{
    return run_bc(level, bc, vfb::kSlipInterp, false, stream);
}

int vfb_noslip_interpolated_incompressible(const vfb_level *level, const vfb_bc *bc, void *stream)
{
    return run_bc(level, bc, vfb::kNoSlipInterpIncomp, false, stream);
}
int vfb_velocity_interpolated_incompressible(const vfb_level *level, const vfb_bc *bc, void *stream)
{
    return run_bc(level, bc, vfb::kVelocityInterpIncomp, true, stream);
}
int vfb_velocity_with_pressure_interpolated_compressible(const vfb_level *level, const vfb_bc *bc, void *stream)
{
    return run_bc(level, bc, vfb::kVelocityWithPressure, true, stream);
}

static int run_directional(const vfb_level *level, const vfb_directional_bc *bc, int kind, const char *what,
                           void *stream)
{
    int st = check_level(level);
    if (st)
        return st;
    if (!bc)
        return fail(VFB_ERR_INVALID_ARGUMENT, "bc is NULL");
    if (bc->direction < VFB_DIR_P00 || bc->direction > VFB_DIR_00M)
        return fail(VFB_ERR_INVALID_ARGUMENT, "direction must be one of the six face directions");
    if (bc->number_of_bc_nodes && (!bc->k || !bc->k_neighbor || (!bc->rho_bc && kind < vfb::kOutflowNonReflecting)))
        return fail(VFB_ERR_INVALID_ARGUMENT, "pressure bc arrays are NULL");
    const cudaError_t e = VFB_DISPATCH(level->storage, level->arith,
                                       LA::pressure(level, bc, as_stream(stream), nullptr, kind));
    return cuda_status(e, what);
}

int vfb_pressure_non_equilibrium_compressible(const vfb_level *level, const vfb_directional_bc *bc, void *stream)
{
    return run_directional(level, bc, vfb::kPressureNeqComp, "PressureNonEquilibriumCompressible launch", stream);
}
int vfb_pressure_non_equilibrium_incompressible(const vfb_level *level, const vfb_directional_bc *bc, void *stream)
{
    return run_directional(level, bc, vfb::kPressureNeqIncomp, "PressureNonEquilibriumIncompressible launch", stream);
}
int vfb_outflow_non_reflecting(const vfb_level *level, const vfb_directional_bc *bc, void *stream)
{
    return run_directional(level, bc, vfb::kOutflowNonReflecting, "OutflowNonReflecting launch", stream);
}
int vfb_outflow_non_reflecting_pressure_correction(const vfb_level *level, const vfb_directional_bc *bc, void *stream)
{
    return run_directional(level, bc, vfb::kOutflowPressureCorrection, "OutflowNonReflectingPressureCorrection launch",
                           stream);
}

static int run_scaling(const vfb_level *coarse, const vfb_level *fine, const vfb_interpolation_cells *cells,
                       const vfb_interpolation_cell_neighbor *offsets, bool fine_to_coarse, void *stream)
{
    int st = check_level(coarse);
    if (st)
        return st;
    st = check_level(fine);
    if (st)
        return st;
    if (!cells || !offsets)
        return fail(VFB_ERR_INVALID_ARGUMENT, "cells or offsets is NULL");
    if (coarse->storage != fine->storage || coarse->arith != fine->arith)
        return fail(VFB_ERR_INVALID_ARGUMENT, "coarse and fine level must share storage and arithmetic");
    if (coarse->distributions == fine->distributions)
        return fail(VFB_ERR_INVALID_ARGUMENT, "coarse and fine level share one population array");
    if (cells->number_of_cells &&
        (!cells->fine_cell_indices || !cells->coarse_cell_indices || !offsets->x || !offsets->y || !offsets->z))
        return fail(VFB_ERR_INVALID_ARGUMENT, "interpolation cell arrays are NULL");
    if (cells->number_of_cells > (1u << 28))
        return fail(VFB_ERR_INVALID_ARGUMENT, "number_of_cells must be below 2^28");
    const cudaError_t e = VFB_DISPATCH(coarse->storage, coarse->arith,
                                       LA::scale(coarse, fine, cells, offsets, fine_to_coarse, as_stream(stream)));
    return cuda_status(e, fine_to_coarse ? "scaleFineToCoarseCompressible launch" : "scaleCoarseToFineCompressible launch");
}

int vfb_scale_coarse_to_fine_compressible(const vfb_level *coarse, const vfb_level *fine,
                                          const vfb_interpolation_cells *cells,
                                          const vfb_interpolation_cell_neighbor *offsets, void *stream)
{
    return run_scaling(coarse, fine, cells, offsets, false, stream);
}

int vfb_scale_fine_to_coarse_compressible(const vfb_level *coarse, const vfb_level *fine,
                                          const vfb_interpolation_cells *cells,
                                          const vfb_interpolation_cell_neighbor *offsets, void *stream)
{
    return run_scaling(coarse, fine, cells, offsets, true, stream);
}

static int run_drag_lift(const vfb_level *level, const vfb_bc *bc, bool pre, double *dx, double *dy, double *dz,
                         void *stream)
{
    int st = check_level(level);
    if (st)
        return st;
    if (!bc)
        return fail(VFB_ERR_INVALID_ARGUMENT, "geometry bc is NULL");
    if (bc->number_of_bc_nodes && (!bc->k || !bc->q27 || !dx || !dy || !dz))
        return fail(VFB_ERR_INVALID_ARGUMENT, "drag/lift arrays are NULL");
    const cudaError_t e = VFB_DISPATCH(level->storage, level->arith, LA::drag_lift(level, bc, pre, dx, dy, dz, as_stream(stream)));
    return cuda_status(e, pre ? "DragLiftPre27 launch" : "DragLiftPost27 launch");
}

int vfb_drag_lift_post_27(const vfb_level *level, const vfb_bc *geometry_bc, double *drag_x, double *drag_y,
                          double *drag_z, void *stream)
{
    return run_drag_lift(level, geometry_bc, false, drag_x, drag_y, drag_z, stream);
}

int vfb_drag_lift_pre_27(const vfb_level *level, const vfb_bc *geometry_bc, double *drag_x, double *drag_y,
                         double *drag_z, void *stream)
{
    return run_drag_lift(level, geometry_bc, true, drag_x, drag_y, drag_z, stream);
}

size_t vfb_drag_lift_workspace_bytes(uint32_t n)
{
    return (size_t)(3 * ((n + 255u) / 256u) + 3) * sizeof(double);
}

int vfb_drag_lift_force(const double *pre_x, const double *pre_y, const double *pre_z, const double *post_x,
                        const double *post_y, const double *post_z, uint32_t n, void *workspace, size_t workspace_bytes,
                        double force[3], void *stream)
{
    if (!force || !workspace || (n && (!pre_x || !pre_y || !pre_z || !post_x || !post_y || !post_z)))
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (workspace_bytes < vfb_drag_lift_workspace_bytes(n))
        return fail(VFB_ERR_INVALID_ARGUMENT, "workspace too small");
    if ((reinterpret_cast<uintptr_t>(workspace) & 7u) != 0)
        return fail(VFB_ERR_INVALID_ARGUMENT, "workspace must be 8-byte aligned");
    cudaStream_t s = as_stream(stream);
    double *scratch = static_cast<double *>(workspace);
    double *result = scratch + 3 * ((n + 255u) / 256u);
    const double *pre[3] = { pre_x, pre_y, pre_z }, *post[3] = { post_x, post_y, post_z };
    cudaError_t e = vfb::drag_lift_sum(pre, post, n, scratch, result, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(force, result, 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    return cuda_status(e, "drag/lift sum");
}

int vfb_init_navier_stokes_compressible(const vfb_level *level, void *stream)
{
    int st = check_level(level);
    if (st)
        return st;
    if (!level->type_of_grid_node || !level->rho || !level->velocity_x || !level->velocity_y || !level->velocity_z)
        return fail(VFB_ERR_INVALID_ARGUMENT, "init needs typeOfGridNode, rho and velocities");
    const cudaError_t e = VFB_DISPATCH(level->storage, level->arith, LA::init_list(level, as_stream(stream)));
    return cuda_status(e, "InitNavierStokesCompressible launch");
}

int vfb_init_navier_stokes_compressible_non_equilibrium(const vfb_level *level, const uint32_t *neighbor_inverse,
                                                        void *stream)
{
    int st = check_level(level);
    if (st)
        return st;
    if (!level->type_of_grid_node || !level->rho || !level->velocity_x || !level->velocity_y || !level->velocity_z)
        return fail(VFB_ERR_INVALID_ARGUMENT, "init needs typeOfGridNode, rho and velocities");
    if (!neighbor_inverse)
        return fail(VFB_ERR_INVALID_ARGUMENT, "the non-equilibrium init needs neighborInverse");
    const cudaError_t e =
        VFB_DISPATCH(level->storage, level->arith, LA::init_neq_list(level, neighbor_inverse, as_stream(stream)));
    return cuda_status(e, "InitNavierStokesCompressibleNonEquilibrium launch");
}

int vfb_calc_macroscopic_compressible(const vfb_level *level, void *stream)
{
    int st = check_level(level);
    if (st)
        return st;
    if (!level->type_of_grid_node || !level->rho || !level->velocity_x || !level->velocity_y || !level->velocity_z)
        return fail(VFB_ERR_INVALID_ARGUMENT, "macroscopic output needs typeOfGridNode, rho and velocities");
    const cudaError_t e = VFB_DISPATCH(level->storage, level->arith, LA::macros_list(level, as_stream(stream)));
    return cuda_status(e, "calculateMacroscopicQuantitiesCompressible launch");
}

size_t vfb_mass_energy_workspace_bytes(uint32_t size)
{
    const uint64_t blocks = (size + 255u) / 256u;
    return (size_t)(2 * blocks + 2) * sizeof(double);
}

int vfb_mass_energy(const vfb_level *level, const uint32_t *idx, uint32_t size, void *workspace, size_t workspace_bytes,
                    double out[2], void *stream)
{
    int st = check_level(level);
    if (st)
        return st;
    if (!out || (size && !idx) || !workspace)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (workspace_bytes < vfb_mass_energy_workspace_bytes(size))
        return fail(VFB_ERR_INVALID_ARGUMENT, "workspace too small");
    if ((reinterpret_cast<uintptr_t>(workspace) & 7u) != 0)
        return fail(VFB_ERR_INVALID_ARGUMENT, "workspace must be 8-byte aligned");
    const uint64_t blocks = (size + 255u) / 256u;
    double *partials = static_cast<double *>(workspace);
    double *result = partials + 2 * blocks;
    cudaStream_t s = as_stream(stream);
    if (size == 0) {
        out[0] = out[1] = 0.0;
        return VFB_OK;
    }
    cudaError_t e = VFB_DISPATCH(level->storage, level->arith, LA::energy_list(level, idx, size, partials, s));
    if (e == cudaSuccess)
        e = vfb::reduce_partials(partials, blocks, result, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, result, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    return cuda_status(e, "mass/energy reduction");
}

// ---------------------------------------------------------------------------------------------
// boundary-condition factory
// ---------------------------------------------------------------------------------------------
int vfb_bc_factory_velocity(int32_t variant, vfb_bc_fn *fn)
{
    if (!fn)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL fn");
    *fn = nullptr;
    switch (variant) {
    case VFB_VELOCITY_BOUNCE_BACK: *fn = vfb_velocity_bounce_back; return VFB_OK;
    case VFB_VELOCITY_INTERPOLATED_COMPRESSIBLE: *fn = vfb_velocity_interpolated_compressible; return VFB_OK;
    case VFB_VELOCITY_NOT_SPECIFIED: return VFB_OK;
    case VFB_VELOCITY_INTERPOLATED_INCOMPRESSIBLE: *fn = vfb_velocity_interpolated_incompressible; return VFB_OK;
    case VFB_VELOCITY_WITH_PRESSURE_INTERPOLATED_COMPRESSIBLE:
        *fn = vfb_velocity_with_pressure_interpolated_compressible;
        return VFB_OK;
    default: return fail(VFB_ERR_INVALID_ARGUMENT, "unknown VelocityBC");
    }
}

int vfb_bc_factory_noslip(int32_t variant, vfb_bc_fn *fn)
{
    if (!fn)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL fn");
    *fn = nullptr;
    switch (variant) {
    case VFB_NOSLIP_DELAY_BOUNCE_BACK: return VFB_OK; // BoundaryConditionFactory.cpp: empty function
    case VFB_NOSLIP_BOUNCE_BACK: *fn = vfb_noslip_bounce_back; return VFB_OK;
    case VFB_NOSLIP_INTERPOLATED_COMPRESSIBLE: *fn = vfb_noslip_interpolated_compressible; return VFB_OK;
    case VFB_NOSLIP_INTERPOLATED_INCOMPRESSIBLE: *fn = vfb_noslip_interpolated_incompressible; return VFB_OK;
    default: return fail(VFB_ERR_INVALID_ARGUMENT, "unknown NoSlipBC");
    }
}

int vfb_bc_factory_slip(int32_t variant, vfb_bc_fn *fn)
{
    if (!fn)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL fn");
    *fn = nullptr;
    switch (variant) {
    case VFB_SLIP_COMPRESSIBLE: *fn = vfb_slip_compressible; return VFB_OK;
    case VFB_SLIP_NOT_SPECIFIED: return VFB_OK;
    case VFB_SLIP_TURBULENT_VISCOSITY_COMPRESSIBLE:
        return fail(VFB_ERR_UNSUPPORTED, "SlipTurbulentViscosityCompressible needs a turbulence model");
    default: return fail(VFB_ERR_INVALID_ARGUMENT, "unknown SlipBC");
    }
}

int vfb_bc_factory_pressure(int32_t variant, vfb_directional_bc_fn *fn)
{
    if (!fn)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL fn");
    *fn = nullptr;
    switch (variant) {
    case VFB_PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE: *fn = vfb_pressure_non_equilibrium_compressible; return VFB_OK;
    case VFB_PRESSURE_NOT_SPECIFIED: return VFB_OK;
    case VFB_PRESSURE_NON_EQUILIBRIUM_INCOMPRESSIBLE: *fn = vfb_pressure_non_equilibrium_incompressible; return VFB_OK;
    case VFB_PRESSURE_OUTFLOW_NON_REFLECTIVE: *fn = vfb_outflow_non_reflecting; return VFB_OK;
    case VFB_PRESSURE_OUTFLOW_NON_REFLECTIVE_PRESSURE_CORRECTION:
        *fn = vfb_outflow_non_reflecting_pressure_correction;
        return VFB_OK;
    default: return fail(VFB_ERR_INVALID_ARGUMENT, "unknown PressureBC");
    }
}

// ---------------------------------------------------------------------------------------------
// grid-scaling factory (GridScalingFactory.cpp: ScaleCompressible -> scale*Compressible<turb>)
// ---------------------------------------------------------------------------------------------
static int scaling_factory(int32_t variant, int32_t turbulent, vfb_scaling_fn impl, vfb_scaling_fn *fn)
{
    if (!fn)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL fn");
    *fn = nullptr;
    switch (variant) {
    case VFB_SCALE_COMPRESSIBLE:
        if (turbulent)
            return fail(VFB_ERR_UNSUPPORTED, "grid scaling with turbulent viscosity not built");
        *fn = impl;
        return VFB_OK;
    case VFB_SCALE_NOT_SPECIFIED: return VFB_OK;
    default: return fail(VFB_ERR_INVALID_ARGUMENT, "unknown GridScaling");
    }
}

int vfb_scaling_factory_fine_to_coarse(int32_t variant, int32_t has_turbulent_viscosity, vfb_scaling_fn *fn)
{
    return scaling_factory(variant, has_turbulent_viscosity, vfb_scale_fine_to_coarse_compressible, fn);
}

int vfb_scaling_factory_coarse_to_fine(int32_t variant, int32_t has_turbulent_viscosity, vfb_scaling_fn *fn)
{
    return scaling_factory(variant, has_turbulent_viscosity, vfb_scale_coarse_to_fine_compressible, fn);
}

} // extern "C"

// ---------------------------------------------------------------------------------------------
// (2a) step driver
// ---------------------------------------------------------------------------------------------
namespace {
// One refinement level of the driver: the LBMSimulationParameter fields of that level and its BC
// lists (Parameter::getParD(level)).
struct SimLevel {
    bool has_level = false;
    vfb_level level{};
    const uint32_t *fluid = nullptr;
    uint32_t n_fluid = 0;
    vfb_bc velocity{};
    vfb_bc_fn velocity_fn = nullptr;
    bool velocity_set = false;
    vfb_bc noslip{};
    vfb_bc_fn noslip_fn = nullptr;
    bool noslip_set = false;
    std::vector<vfb_directional_bc> pressure;
    std::vector<vfb_directional_bc_fn> pressure_fn;
    vfb_bc slip{};
    vfb_bc_fn slip_fn = nullptr;
    bool slip_set = false;
    vfb_bc geometry{};
    vfb_bc_fn geometry_fn = nullptr;
    bool geometry_set = false;
    // drag and lift on the geometry nodes (caller-owned device memory)
    double *drag_work = nullptr;      // pre x, y, z; post x, y, z (6 * n); block partials
    double *drag_history = nullptr;   // 3 doubles per step, ring of drag_history_len steps
    uint32_t drag_history_len = 0;
    uint64_t drag_steps = 0;
    // interpolation cells between this level and the next finer one (fineToCoarse,
    // neighborFineToCoarse, coarseToFine, neighborCoarseToFine of the coarse level)
    vfb_interpolation_cells fc{}, cf{};
    vfb_interpolation_cell_neighbor fc_offsets{}, cf_offsets{};
    // neighbour slot table of the fluid-node list (library-owned, built by set_level)
    // per post-collision BC list: its post-collision values taken before the list writes (27 doubles
    // per node, enough for every storage), so that the BCs of a list never read each other's writes
    void *snap[4] = { nullptr, nullptr, nullptr, nullptr };   // velocity, no-slip, geometry, slip
    uint32_t snap_nodes[4] = { 0, 0, 0, 0 };
    // a fluid list that is a whole periodic box in x-fastest order from node box_first (checked at
    // set_level against the neighbour arrays): collided with arithmetic addressing
    bool regular = false;
    int box_dims[3] = { 0, 0, 0 };
    uint32_t box_first = 0;
    uint32_t *slots = nullptr;        // 8 arrays of slots_stride entries, then the kernels' status word
    uint64_t slots_stride = 0;
    size_t slots_nodes = 0;
    const void *slots_key[4] = { nullptr, nullptr, nullptr, nullptr };

    int *status() const { return reinterpret_cast<int *>(slots + 8 * slots_stride); }
    void free_slots()
    {
        if (slots)
            cudaFree(slots);
        slots = nullptr;
        slots_stride = 0;
        slots_nodes = 0;
        for (auto &p : slots_key)
            p = nullptr;
    }
    void free_snaps()
    {
        for (int i = 0; i < 4; ++i) {
            if (snap[i])
                cudaFree(snap[i]);
            snap[i] = nullptr;
            snap_nodes[i] = 0;
        }
    }
    ~SimLevel()
    {
        free_slots();
        free_snaps();
    }
    SimLevel() = default;
    SimLevel(const SimLevel &) = delete;
    SimLevel &operator=(const SimLevel &) = delete;
    SimLevel(SimLevel &&o) noexcept { *this = std::move(o); }
    SimLevel &operator=(SimLevel &&o) noexcept
    {
        if (this != &o) {
            free_slots();
            free_snaps();
            for (int i = 0; i < 4; ++i) {
                snap[i] = o.snap[i];
                snap_nodes[i] = o.snap_nodes[i];
                o.snap[i] = nullptr;
                o.snap_nodes[i] = 0;
            }
            has_level = o.has_level; level = o.level; fluid = o.fluid; n_fluid = o.n_fluid;
            velocity = o.velocity; velocity_fn = o.velocity_fn; velocity_set = o.velocity_set;
            noslip = o.noslip; noslip_fn = o.noslip_fn; noslip_set = o.noslip_set;
            slip = o.slip; slip_fn = o.slip_fn; slip_set = o.slip_set;
            pressure = std::move(o.pressure); pressure_fn = std::move(o.pressure_fn);
            geometry = o.geometry; geometry_fn = o.geometry_fn; geometry_set = o.geometry_set;
            drag_work = o.drag_work; drag_history = o.drag_history; drag_history_len = o.drag_history_len;
            drag_steps = o.drag_steps; fc = o.fc; cf = o.cf; fc_offsets = o.fc_offsets; cf_offsets = o.cf_offsets;
            regular = o.regular; box_first = o.box_first;
            for (int i = 0; i < 3; ++i)
                box_dims[i] = o.box_dims[i];
            slots = o.slots; slots_stride = o.slots_stride; slots_nodes = o.slots_nodes;
            for (int i = 0; i < 4; ++i)
                slots_key[i] = o.slots_key[i];
            o.slots = nullptr;
            o.slots_nodes = 0;
        }
        return *this;
    }
};
} // namespace

// Phase timers of the step driver, in the phases of the reference's TimeStepTimer
// (Output/TimeStepTimer.h: collision, post- and pre-collision BCs) plus the two interpolation
// directions. With timing on, each phase of a run is bracketed by CUDA events on the run's stream;
// the run synchronises once at its end and adds the elapsed times up. The events are reused.
struct PhaseTimers {
    bool on = false;
    double ms[VFB_PHASES] = {};
    uint64_t steps = 0;
    std::vector<cudaEvent_t> free_events;
    struct Pending {
        int phase;
        cudaEvent_t start, stop;
    };
    std::vector<Pending> pending;
    cudaEvent_t take()
    {
        if (!free_events.empty()) {
            cudaEvent_t e = free_events.back();
            free_events.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return e;
    }
    // add up the pending phases (the caller has synchronised their stream)
    cudaError_t collect()
    {
        cudaError_t err = cudaSuccess;
        for (const Pending &p : pending) {
            float t = 0.0f;
            const cudaError_t e = cudaEventElapsedTime(&t, p.start, p.stop);
            if (e == cudaSuccess)
                ms[p.phase] += t;
            else if (err == cudaSuccess)
                err = e;
            free_events.push_back(p.start);
            free_events.push_back(p.stop);
        }
        pending.clear();
        return err;
    }
    ~PhaseTimers()
    {
        for (const Pending &p : pending) {
            cudaEventDestroy(p.start);
            cudaEventDestroy(p.stop);
        }
        for (cudaEvent_t e : free_events)
            cudaEventDestroy(e);
    }
};

const char *const kPhaseNames[VFB_PHASES] = { "collision", "postCollisionBC", "preCollisionBC", "scalingFineToCoarse",
                                              "scalingCoarseToFine" };

// an NVTX range of the phase's name and, with timing on, its two events
class PhaseScope {
public:
    PhaseScope(PhaseTimers &t, int phase, void *stream) : t_(t), phase_(phase), stream_(static_cast<cudaStream_t>(stream))
    {
        nvtxRangePushA(kPhaseNames[phase]);
        if (t_.on && (start_ = t_.take()) != nullptr)
            cudaEventRecord(start_, stream_);
    }
    ~PhaseScope()
    {
        if (start_) {
            cudaEvent_t stop = t_.take();
            if (stop) {
                cudaEventRecord(stop, stream_);
                t_.pending.push_back({ phase_, start_, stop });
            } else {
                t_.free_events.push_back(start_);
            }
        }
        nvtxRangePop();
    }
    PhaseScope(const PhaseScope &) = delete;
    PhaseScope &operator=(const PhaseScope &) = delete;

private:
    PhaseTimers &t_;
    int phase_;
    cudaStream_t stream_;
    cudaEvent_t start_ = nullptr;
};

// The step loop captured as a CUDA graph: `steps` coarse steps (an even number, so every level
// ends at the parity it started from) recorded once on a stream and replayed. Any change of the
// configuration drops it; a replay is taken only when every level's parity equals the one it was
// captured at, else the graph is captured again.
struct StepGraph {
    int32_t steps = 0;              // coarse steps per graph, 0 = off
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;
    std::vector<int> parity;        // every level's parity at capture
    bool warm = false;              // a step has run directly since the last change (lazy buffers exist)
    void drop()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        exec = nullptr;
        stream = nullptr;
        parity.clear();
    }
    ~StepGraph() { drop(); }
};

struct vfb_simulation {
    int kernel_id = 0;
    std::vector<SimLevel> levels = std::vector<SimLevel>(1);
    int32_t cursor = 0;               // the level the setters configure
    int32_t neighbor_tables = 1;      // 0 chain, 1 slot tables, 2 slot tables staged by bulk copies
    bool scaling_set = false;         // GridScalingFactory given
    vfb_scaling_fn scale_fc = nullptr;
    vfb_scaling_fn scale_cf = nullptr;
    PhaseTimers timers;
    StepGraph graph;
};

// every setter: a captured step no longer matches the configuration
static void config_changed(vfb_simulation *sim)
{
    sim->graph.drop();
    sim->graph.warm = false;
}

static SimLevel &current(vfb_simulation *sim) { return sim->levels[(size_t)sim->cursor]; }

// the seven +1 neighbour nodes (x, y, xy, z, xz, yz, xyz) of every listed node, stored per slot so
// that the collision reads them with one coalesced load each instead of the neighborX/Y/Z chain
// (the order of the kernels' ListIndices: slot bit 0 = +x, bit 1 = +y, bit 2 = +z)
__global__ void list_slots_kernel(const uint32_t *__restrict__ idx, uint32_t n_idx, const uint32_t *__restrict__ nbx,
                                  const uint32_t *__restrict__ nby, const uint32_t *__restrict__ nbz,
                                  uint32_t *__restrict__ slots, uint64_t stride)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_idx)
        return;
    const uint32_t k = __ldg(idx + i);
    const uint32_t kx = __ldg(nbx + k), ky = __ldg(nby + k), kz = __ldg(nbz + k);
    const uint32_t kxy = __ldg(nby + kx);
    const uint32_t out[8] = { k, kx, ky, kxy, kz, __ldg(nbz + kx), __ldg(nbz + ky), __ldg(nbz + kxy) };
#pragma unroll
    for (int j = 0; j < 8; ++j)
        slots[(size_t)j * stride + i] = out[j];
}

// every entry i of the fluid list must be node first + i and have the +1 neighbours of a periodic
// dx * dy * dz box numbered x fastest from `first`; *bad counts the entries that are not
__global__ void regular_box_check_kernel(const uint32_t *__restrict__ fluid, uint32_t n, const uint32_t *__restrict__ nbx,
                                         const uint32_t *__restrict__ nby, const uint32_t *__restrict__ nbz,
                                         uint32_t first, uint32_t dx, uint32_t dy, uint32_t dz, unsigned *bad)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t x = i % dx, y = (i / dx) % dy, z = i / (dx * dy);
    const uint32_t k = first + i;
    bool ok = __ldg(fluid + i) == k;
    ok = ok && __ldg(nbx + k) == first + (x + 1) % dx + dx * (y + dy * z);
    ok = ok && __ldg(nby + k) == first + x + dx * ((y + 1) % dy + dy * z);
    ok = ok && __ldg(nbz + k) == first + x + dx * (y + dy * ((z + 1) % dz));
    if (!ok)
        atomicAdd(bad, 1u);
}

// Whether a level's fluid list is a whole periodic box numbered x fastest (the numbering of the
// reference's grid builder for a box without solids): the box's size comes from the first node's
// +y and +z neighbours, and a kernel checks every entry and its three neighbours against it.
static int detect_regular_box(SimLevel &S)
{
    S.regular = false;
    const vfb_level &L = S.level;
    const uint32_t n = S.n_fluid;
    // the 16-bit forms hash each slot's offset into their stochastic rounding: a box over the
    // shifted array would round differently, so they keep the list kernel
    if (L.storage != VFB_STORAGE_F64 && L.storage != VFB_STORAGE_F32)
        return VFB_OK;
    if (n < 2 || !L.neighbor_x || !L.neighbor_y || !L.neighbor_z)
        return VFB_OK;
    uint32_t first = 0, last = 0, ny0 = 0, nz0 = 0;
    cudaError_t e = cudaMemcpy(&first, S.fluid, sizeof first, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(&last, S.fluid + (n - 1), sizeof last, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "reading the fluid list");
    if ((uint64_t)first + n > L.number_of_nodes || (uint64_t)last != (uint64_t)first + n - 1)
        return VFB_OK;
    e = cudaMemcpy(&ny0, L.neighbor_y + first, sizeof ny0, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(&nz0, L.neighbor_z + first, sizeof nz0, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "reading the neighbour arrays");
    if (ny0 <= first || nz0 <= first)
        return VFB_OK;
    const uint64_t dx = ny0 - first, dxy = (uint64_t)nz0 - first;
    if (dxy % dx != 0 || n % dxy != 0 || dx > (1u << 20) || dxy / dx > (1u << 20))
        return VFB_OK;
    const uint32_t dy = (uint32_t)(dxy / dx), dz = (uint32_t)(n / dxy);
    unsigned *bad = nullptr;
    e = cudaMalloc(&bad, sizeof(unsigned));
    if (e == cudaSuccess)
        e = cudaMemset(bad, 0, sizeof(unsigned));
    if (e == cudaSuccess) {
        regular_box_check_kernel<<<(n + 255) / 256, 256>>>(S.fluid, n, L.neighbor_x, L.neighbor_y, L.neighbor_z, first,
                                                          (uint32_t)dx, dy, dz, bad);
        e = cudaGetLastError();
    }
    unsigned n_bad = 1;
    if (e == cudaSuccess)
        e = cudaMemcpy(&n_bad, bad, sizeof n_bad, cudaMemcpyDeviceToHost);
    cudaFree(bad);
    if (e != cudaSuccess)
        return cuda_status(e, "checking for a regular box");
    if (n_bad == 0) {
        S.regular = true;
        S.box_first = first;
        S.box_dims[0] = (int)dx;
        S.box_dims[1] = (int)dy;
        S.box_dims[2] = (int)dz;
    }
    return VFB_OK;
}

// the list collision's force along one axis, forces * 1/2 * 2^-level formed in the compute type
// (double for F64 storage, float otherwise) as run_k17's launcher forms it, returned as a double
// that converts back to the same value
static double list_half_force(const vfb_level &L, int axis)
{
    if (L.storage == VFB_STORAGE_F64) {
        double f = 1.0;
        for (int i = 1; i <= L.level; ++i)
            f *= 2.0;
        return L.forces[axis] * 0.5 * (1.0 / f);
    }
    float f = 1.0f;
    for (int i = 1; i <= L.level; ++i)
        f *= 2.0f;
    return (double)((float)L.forces[axis] * 0.5f * (1.0f / f));
}

// a regular level as a structured box over the reference layout: the populations of node
// box_first + k at plane * numberOfNodes + box_first + k, the direct-load box kernel
static vfb::BoxState regular_box_state(const SimLevel &S)
{
    const vfb_level &L = S.level;
    const size_t elem = L.storage == VFB_STORAGE_F64 ? 8 : L.storage == VFB_STORAGE_F32 ? 4 : 2;
    vfb::BoxState b{};
    b.dist = static_cast<char *>(L.distributions) + (size_t)S.box_first * elem;
    b.pitch = L.number_of_nodes;
    b.nx = S.box_dims[0];
    b.ny = S.box_dims[1];
    b.nz = S.box_dims[2];
    b.periodic_x = b.periodic_y = b.periodic_z = 1;
    b.mask = nullptr;
    b.omega = L.omega;
    b.fx = list_half_force(L, 0);
    b.fy = list_half_force(L, 1);
    b.fz = list_half_force(L, 2);
    for (int i = 0; i < 3; ++i)
        b.lim[i] = L.quadric_limiters[i];
    b.variant = 1;
    b.status = nullptr;
    return b;
}

// The slot table of a level (the seven +1 neighbours of each fluid node, one array per slot),
// rebuilt when the fluid list or the neighbour arrays change. It costs 28 bytes per fluid node and
// replaces the four-deep chain of dependent neighborX/Y/Z loads in every collision.
static int build_slots(int32_t tables, SimLevel &S)
{
    const void *key[4] = { S.fluid, S.level.neighbor_x, S.level.neighbor_y, S.level.neighbor_z };
    if (!tables || S.n_fluid == 0) {
        S.free_slots();
        S.regular = false;
        return VFB_OK;
    }
    if (S.slots && S.slots_nodes == S.n_fluid && std::equal(key, key + 4, S.slots_key))
        return VFB_OK;
    S.free_slots();
    // whole 32-entry tiles (the staged kernel copies 128-byte rows), padding entries = node 0
    const uint64_t stride = ((uint64_t)S.n_fluid + 31) / 32 * 32;
    const size_t bytes = (size_t)8 * stride * sizeof(uint32_t) + 16;
    if (cudaMalloc(&S.slots, bytes) != cudaSuccess) {
        cudaGetLastError();
        S.slots = nullptr;
        return fail(VFB_ERR_OUT_OF_MEMORY, "no device memory for the neighbour slot table");
    }
    S.slots_stride = stride;
    cudaError_t e = cudaMemset(S.slots, 0, bytes);
    const unsigned B = 256, G = (unsigned)((S.n_fluid + B - 1) / B);
    if (e == cudaSuccess)
        list_slots_kernel<<<G, B>>>(S.fluid, S.n_fluid, S.level.neighbor_x, S.level.neighbor_y, S.level.neighbor_z,
                                    S.slots, stride);
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaDeviceSynchronize();   // visible to every stream the level is later run on
    if (e != cudaSuccess) {
        S.free_slots();
        return cuda_status(e, "neighbour slot table");
    }
    S.slots_nodes = S.n_fluid;
    std::copy(key, key + 4, S.slots_key);
    return detect_regular_box(S);      // the same fluid list and neighbour arrays as the table
}

extern "C" {

int vfb_simulation_create(const char *kernel_name, vfb_simulation **out)
{
    if (!out)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL out");
    *out = nullptr;
    int32_t id = 0;
    int st = vfb_kernel_lookup(kernel_name, &id);
    if (st)
        return st;
    vfb_simulation *s = new vfb_simulation();
    s->kernel_id = id;
    *out = s;
    return VFB_OK;
}

int vfb_simulation_destroy(vfb_simulation *sim)
{
    delete sim;
    return VFB_OK;
}

int vfb_simulation_use_level(vfb_simulation *sim, int32_t level)
{
    if (!sim)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL simulation");
    config_changed(sim);
    if (level < 0 || level > (int32_t)sim->levels.size() || level >= VFB_MAX_LEVELS)
        return fail(VFB_ERR_INVALID_ARGUMENT, "levels are added one at a time, from the coarsest, up to VFB_MAX_LEVELS");
    if (level == (int32_t)sim->levels.size())
        sim->levels.emplace_back();
    sim->cursor = level;
    return VFB_OK;
}

int vfb_simulation_set_neighbor_tables(vfb_simulation *sim, int32_t enable)
{
    if (!sim)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL simulation");
    config_changed(sim);
    if (enable < 0 || enable > 2)
        return fail(VFB_ERR_INVALID_ARGUMENT, "neighbour tables: 0 off, 1 direct loads, 2 staged copies");
    sim->neighbor_tables = enable;
    for (SimLevel &S : sim->levels) {
        if (!S.has_level)
            continue;
        int st = build_slots(sim->neighbor_tables, S);
        if (st)
            return st;
    }
    return VFB_OK;
}

int vfb_simulation_status(vfb_simulation *sim, int32_t *device_status, void *stream)
{
    if (!sim || !device_status)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaError_t e = cudaStreamSynchronize(as_stream(stream));
    int32_t worst = 0;
    for (SimLevel &S : sim->levels) {
        if (!S.slots || e != cudaSuccess)
            continue;
        int v = 0;
        e = cudaMemcpy(&v, S.status(), sizeof(int), cudaMemcpyDeviceToHost);
        worst = std::max(worst, (int32_t)v);
    }
    *device_status = worst;
    if (e != cudaSuccess)
        return cuda_status(e, "simulation status");
    return worst ? fail(VFB_ERR_CUDA, "a kernel gave up waiting for its staged copies") : VFB_OK;
}

int vfb_simulation_number_of_levels(const vfb_simulation *sim, int32_t *n)
{
    if (!sim || !n)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *n = (int32_t)sim->levels.size();
    return VFB_OK;
}

int vfb_simulation_set_level(vfb_simulation *sim, const vfb_level *level, const uint32_t *fluid, uint32_t n)
{
    if (!sim)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL simulation");
    config_changed(sim);
    int st = check_level(level);
    if (st)
        return st;
    if (n && !fluid)
        return fail(VFB_ERR_INVALID_ARGUMENT, "fluid node indices are NULL");
    if (level->level != sim->cursor)
        return fail(VFB_ERR_INVALID_ARGUMENT, "vfb_level::level must equal the selected level");
    SimLevel &S = current(sim);
    S.level = *level;
    S.fluid = fluid;
    S.n_fluid = n;
    S.has_level = true;
    return build_slots(sim->neighbor_tables, S);
}

int vfb_simulation_level_box_addressing(const vfb_simulation *sim, int32_t level, int32_t *box_addressing)
{
    if (!sim || !box_addressing || level < 0 || level >= (int32_t)sim->levels.size())
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument or no such level");
    const SimLevel &S = sim->levels[level];
    *box_addressing = (S.regular && sim->neighbor_tables != 0) ? 1 : 0;
    return VFB_OK;
}

// ---------------------------------------------------------------------------------------------
// prepared collisions: one fluid-node list of a level with its slot table and box addressing, for
// callers that keep their own step loop (the reference's KernelImp::run / runOnIndices)
// ---------------------------------------------------------------------------------------------
struct vfb_k17_plan {
    SimLevel S;
};

int vfb_k17_plan_create(const vfb_level *level, const uint32_t *idx, uint32_t size, vfb_k17_plan **plan)
{
    if (!plan)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL plan");
    *plan = nullptr;
    int st = check_level(level);
    if (st)
        return st;
    if (size && !idx)
        return fail(VFB_ERR_INVALID_ARGUMENT, "fluid node indices are NULL");
    auto *p = new vfb_k17_plan();
    p->S.level = *level;
    p->S.fluid = idx;
    p->S.n_fluid = size;
    p->S.has_level = true;
    st = build_slots(1, p->S);
    if (st) {
        delete p;
        return st;
    }
    *plan = p;
    return VFB_OK;
}

int vfb_k17_plan_run(vfb_k17_plan *plan, const vfb_level *level, int32_t collision_template, void *stream)
{
    if (!plan)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL plan");
    int st = check_level(level);
    if (st)
        return st;
    SimLevel &S = plan->S;
    if (level->number_of_nodes != S.level.number_of_nodes || level->neighbor_x != S.level.neighbor_x ||
        level->neighbor_y != S.level.neighbor_y || level->neighbor_z != S.level.neighbor_z ||
        level->storage != S.level.storage)
        return fail(VFB_ERR_INVALID_ARGUMENT, "the level's node count, neighbour arrays or storage differ from the plan's");
    S.level = *level;                 // parity, omega, forces and the arrays of this call
    if (collision_template == VFB_COLLISION_DEFAULT && S.regular) {
        const vfb::BoxState b = regular_box_state(S);
        const cudaError_t e = VFB_DISPATCH(level->storage, level->arith,
                                           LA::box_collide(b, level->is_even_timestep != 0, nullptr, nullptr,
                                                           as_stream(stream)));
        return cuda_status(e, "K17CompressibleNavierStokes launch");
    }
    return run_k17(level, S.fluid, S.n_fluid, collision_template, S.slots, S.slots_stride, stream);
}

int vfb_k17_plan_box_addressing(const vfb_k17_plan *plan, int32_t *box_addressing)
{
    if (!plan || !box_addressing)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *box_addressing = plan->S.regular ? 1 : 0;
    return VFB_OK;
}

int vfb_k17_plan_destroy(vfb_k17_plan *plan)
{
    delete plan;
    return VFB_OK;
}

int vfb_simulation_set_velocity_bc(vfb_simulation *sim, const vfb_bc *bc, int32_t variant)
{
    if (!sim || !bc)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    config_changed(sim);
    vfb_bc_fn fn = nullptr;
    int st = vfb_bc_factory_velocity(variant, &fn);
    if (st)
        return st;
    SimLevel &S = current(sim);
    S.velocity = *bc;
    S.velocity_fn = fn;
    S.velocity_set = true;
    return VFB_OK;
}

int vfb_simulation_set_noslip_bc(vfb_simulation *sim, const vfb_bc *bc, int32_t variant)
{
    if (!sim || !bc)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    config_changed(sim);
    vfb_bc_fn fn = nullptr;
    int st = vfb_bc_factory_noslip(variant, &fn);
    if (st)
        return st;
    SimLevel &S = current(sim);
    S.noslip = *bc;
    S.noslip_fn = fn;
    S.noslip_set = true;
    return VFB_OK;
}

int vfb_simulation_set_slip_bc(vfb_simulation *sim, const vfb_bc *bc, int32_t variant)
{
    if (!sim || !bc)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    config_changed(sim);
    vfb_bc_fn fn = nullptr;
    int st = vfb_bc_factory_slip(variant, &fn);
    if (st)
        return st;
    SimLevel &S = current(sim);
    S.slip = *bc;
    S.slip_fn = fn;
    S.slip_set = true;
    return VFB_OK;
}

int vfb_simulation_add_pressure_bc(vfb_simulation *sim, const vfb_directional_bc *bc, int32_t variant)
{
    if (!sim || !bc)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    config_changed(sim);
    vfb_directional_bc_fn fn = nullptr;
    int st = vfb_bc_factory_pressure(variant, &fn);
    if (st)
        return st;
    SimLevel &S = current(sim);
    S.pressure.push_back(*bc);
    S.pressure_fn.push_back(fn);
    return VFB_OK;
}

// BoundaryConditionKernelManager.cpp:67-80: a BC that has nodes needs a kernel; the delayed
// no-slip bounce-back is the one BC whose "kernel" is deliberately empty.
int vfb_simulation_set_geometry_bc(vfb_simulation *sim, const vfb_bc *bc, int32_t variant)
{
    if (!sim || !bc)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    config_changed(sim);
    vfb_bc_fn fn = nullptr;
    int st = vfb_bc_factory_noslip(variant, &fn);
    if (st)
        return st;
    SimLevel &S = current(sim);
    S.geometry = *bc;
    S.geometry_fn = fn;
    S.geometry_set = true;
    return VFB_OK;
}

// BoundaryConditionFactory::getGeometryBoundaryConditionPost (BoundaryConditionFactory.cpp:206-216):
// the geometry BC is a velocity, a no-slip or a slip BC
int vfb_simulation_set_geometry_bc_of(vfb_simulation *sim, const vfb_bc *bc, int32_t family, int32_t variant)
{
    if (!sim || !bc)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    vfb_bc_fn fn = nullptr;
    int st;
    switch (family) {
    case VFB_GEOMETRY_VELOCITY: st = vfb_bc_factory_velocity(variant, &fn); break;
    case VFB_GEOMETRY_NOSLIP: st = vfb_bc_factory_noslip(variant, &fn); break;
    case VFB_GEOMETRY_SLIP: st = vfb_bc_factory_slip(variant, &fn); break;
    default: return fail(VFB_ERR_INVALID_ARGUMENT, "geometry BC family must be velocity, no-slip or slip");
    }
    if (st)
        return st;
    if (family == VFB_GEOMETRY_VELOCITY && bc->number_of_bc_nodes && (!bc->vx || !bc->vy || !bc->vz))
        return fail(VFB_ERR_INVALID_ARGUMENT, "a velocity geometry BC needs its wall velocities");
    config_changed(sim);
    SimLevel &S = current(sim);
    S.geometry = *bc;
    S.geometry_fn = fn;
    S.geometry_set = true;
    return VFB_OK;
}

size_t vfb_simulation_drag_lift_workspace_bytes(uint32_t number_of_geometry_nodes)
{
    return (size_t)6 * number_of_geometry_nodes * sizeof(double) + vfb_drag_lift_workspace_bytes(number_of_geometry_nodes);
}

int vfb_simulation_set_drag_lift(vfb_simulation *sim, void *workspace, size_t workspace_bytes, double *force_history,
                                 uint32_t history_steps)
{
    if (!sim)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL simulation");
    config_changed(sim);
    SimLevel &S = current(sim);
    if (!workspace) {
        S.drag_work = nullptr;
        S.drag_history = nullptr;
        S.drag_history_len = 0;
        return VFB_OK;
    }
    if (!S.geometry_set)
        return fail(VFB_ERR_INVALID_ARGUMENT, "drag and lift need a geometry boundary condition");
    if (!force_history || history_steps == 0)
        return fail(VFB_ERR_INVALID_ARGUMENT, "drag and lift need a force history of at least one step");
    if (workspace_bytes < vfb_simulation_drag_lift_workspace_bytes(S.geometry.number_of_bc_nodes))
        return fail(VFB_ERR_INVALID_ARGUMENT, "workspace too small");
    if ((reinterpret_cast<uintptr_t>(workspace) & 7u) != 0)
        return fail(VFB_ERR_INVALID_ARGUMENT, "workspace must be 8-byte aligned");
    S.drag_work = static_cast<double *>(workspace);
    S.drag_history = force_history;
    S.drag_history_len = history_steps;
    S.drag_steps = 0;
    return VFB_OK;
}

int vfb_simulation_set_scaling_factory(vfb_simulation *sim, int32_t variant, int32_t has_turbulent_viscosity)
{
    if (!sim)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL simulation");
    config_changed(sim);
    vfb_scaling_fn fc = nullptr, cf = nullptr;
    int st = vfb_scaling_factory_fine_to_coarse(variant, has_turbulent_viscosity, &fc);
    if (st)
        return st;
    st = vfb_scaling_factory_coarse_to_fine(variant, has_turbulent_viscosity, &cf);
    if (st)
        return st;
    sim->scale_fc = fc;
    sim->scale_cf = cf;
    sim->scaling_set = true;
    return VFB_OK;
}

int vfb_simulation_set_interpolation_cells(vfb_simulation *sim, int32_t coarse_level,
                                           const vfb_interpolation_cells *fine_to_coarse,
                                           const vfb_interpolation_cell_neighbor *fine_to_coarse_offsets,
                                           const vfb_interpolation_cells *coarse_to_fine,
                                           const vfb_interpolation_cell_neighbor *coarse_to_fine_offsets)
{
    if (!sim || !fine_to_coarse || !fine_to_coarse_offsets || !coarse_to_fine || !coarse_to_fine_offsets)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    config_changed(sim);
    if (coarse_level < 0 || coarse_level + 1 >= (int32_t)sim->levels.size())
        return fail(VFB_ERR_INVALID_ARGUMENT, "coarse_level and the level above it must have been added");
    const vfb_interpolation_cells *c[2] = { fine_to_coarse, coarse_to_fine };
    const vfb_interpolation_cell_neighbor *o[2] = { fine_to_coarse_offsets, coarse_to_fine_offsets };
    for (int i = 0; i < 2; ++i)
        if (c[i]->number_of_cells &&
            (!c[i]->fine_cell_indices || !c[i]->coarse_cell_indices || !o[i]->x || !o[i]->y || !o[i]->z))
            return fail(VFB_ERR_INVALID_ARGUMENT, "interpolation cell arrays are NULL");
    SimLevel &S = sim->levels[(size_t)coarse_level];
    S.fc = *fine_to_coarse;
    S.fc_offsets = *fine_to_coarse_offsets;
    S.cf = *coarse_to_fine;
    S.cf_offsets = *coarse_to_fine_offsets;
    return VFB_OK;
}

int vfb_simulation_check(const vfb_simulation *sim)
{
    if (!sim)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL simulation");
    const size_t nl = sim->levels.size();
    for (size_t l = 0; l < nl; ++l) {
        const SimLevel &S = sim->levels[l];
        if (!S.has_level)
            return fail(VFB_ERR_INVALID_ARGUMENT, "level " + std::to_string(l) + " is not set");
        if (S.velocity_set && S.velocity.number_of_bc_nodes > 0 && !S.velocity_fn)
            return fail(VFB_ERR_BC_UNSET, "Velocity boundary condition has nodes but no kernel");
        if (S.slip_set && S.slip.number_of_bc_nodes > 0 && !S.slip_fn)
            return fail(VFB_ERR_BC_UNSET, "Slip boundary condition has nodes but no kernel");
        for (size_t i = 0; i < S.pressure.size(); ++i)
            if (S.pressure[i].number_of_bc_nodes > 0 && !S.pressure_fn[i])
                return fail(VFB_ERR_BC_UNSET, "Pressure boundary condition has nodes but no kernel");
        if (S.level.storage != sim->levels[0].level.storage || S.level.arith != sim->levels[0].level.arith)
            return fail(VFB_ERR_INVALID_ARGUMENT, "all levels must share storage and arithmetic");
    }
    // GridScalingKernelManager ctor (GridScalingKernelManager.cpp:45-62, checkScalingFunction)
    if (nl > 1) {
        if (!sim->scaling_set)
            return fail(VFB_ERR_SCALING_UNSET, "There is more than one level, but no scalingFactory was provided.");
        for (size_t l = 0; l + 1 < nl; ++l) {
            if (!sim->scale_fc && sim->levels[l].fc.number_of_cells > 0)
                return fail(VFB_ERR_SCALING_UNSET, "The scaling function scalingFineToCoarse was not set!");
            if (!sim->scale_cf && sim->levels[l].cf.number_of_cells > 0)
                return fail(VFB_ERR_SCALING_UNSET, "The scaling function scalingCoarseToFine was not set!");
        }
    }
    return VFB_OK;
}

// the kernel kind behind a factory function, for the driver's snapshot launches
static int bc_kind_of(vfb_bc_fn fn, bool &velocity)
{
    velocity = true;
    if (fn == vfb_velocity_bounce_back) return vfb::kVelocityBB;
    if (fn == vfb_velocity_interpolated_compressible) return vfb::kVelocityInterp;
    if (fn == vfb_velocity_interpolated_incompressible) return vfb::kVelocityInterpIncomp;
    if (fn == vfb_velocity_with_pressure_interpolated_compressible) return vfb::kVelocityWithPressure;
    velocity = false;
    if (fn == vfb_slip_compressible) return vfb::kSlipInterp;
    if (fn == vfb_noslip_bounce_back) return vfb::kNoSlipBB;
    if (fn == vfb_noslip_interpolated_compressible) return vfb::kNoSlipInterp;
    if (fn == vfb_noslip_interpolated_incompressible) return vfb::kNoSlipInterpIncomp;
    return -1;
}

// a post-collision BC list through its factory function, reading the list's snapshot
static int run_list(SimLevel &S, int which, vfb_bc_fn fn, const vfb_bc &bc, void *stream)
{
    if (!fn || bc.number_of_bc_nodes == 0)
        return VFB_OK;
    bool velocity = false;
    const int kind = bc_kind_of(fn, velocity);
    if (kind < 0)
        return fn(&S.level, &bc, stream);
    if (S.snap_nodes[which] < bc.number_of_bc_nodes) {
        if (S.snap[which])
            cudaFree(S.snap[which]);
        S.snap[which] = nullptr;
        S.snap_nodes[which] = 0;
        if (cudaMalloc(&S.snap[which], (size_t)27 * bc.number_of_bc_nodes * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            S.snap[which] = nullptr;
            return fail(VFB_ERR_OUT_OF_MEMORY, "no device memory for a boundary-condition snapshot");
        }
        S.snap_nodes[which] = bc.number_of_bc_nodes;
    }
    return run_bc(&S.level, &bc, kind, velocity, stream, S.snap[which]);
}

static int run_geometry_post(SimLevel &S, void *stream)
{
    vfb_level &L = S.level;
    const uint32_t ng = S.geometry.number_of_bc_nodes;
    if (!S.geometry_set || ng == 0)
        return VFB_OK;
    if (S.drag_work) {
        double *w = S.drag_work;
        int st = vfb_drag_lift_post_27(&L, &S.geometry, w + 3 * (size_t)ng, w + 4 * (size_t)ng, w + 5 * (size_t)ng, stream);
        if (st)
            return st;
    }
    return run_list(S, 2, S.geometry_fn, S.geometry, stream);
}

static int run_geometry_pre(SimLevel &S, void *stream)
{
    vfb_level &L = S.level;
    const uint32_t ng = S.geometry.number_of_bc_nodes;
    if (!S.geometry_set || ng == 0 || !S.drag_work)
        return VFB_OK;
    double *w = S.drag_work;
    int st = vfb_drag_lift_pre_27(&L, &S.geometry, w, w + ng, w + 2 * (size_t)ng, stream);
    if (st)
        return st;
    const double *pre[3] = { w, w + ng, w + 2 * (size_t)ng };
    const double *post[3] = { w + 3 * (size_t)ng, w + 4 * (size_t)ng, w + 5 * (size_t)ng };
    double *out = S.drag_history + 3 * (S.drag_steps % S.drag_history_len);
    const cudaError_t e = vfb::drag_lift_sum(pre, post, ng, w + 6 * (size_t)ng, out, as_stream(stream));
    ++S.drag_steps;
    return cuda_status(e, "drag/lift sum");
}

// one time step of one level: collision, post-collision BCs (velocity, no-slip, geometry), parity
// toggle, pre-collision BCs (pressure) (UpdateGrid27.cpp:66-84)
static int step_level(vfb_simulation *sim, SimLevel &S, void *stream)
{
    vfb_level &L = S.level;
    int st;
    {
    PhaseScope phase(sim->timers, VFB_PHASE_COLLISION, stream);
    if (S.regular && sim->neighbor_tables != 0) {
        const vfb::BoxState b = regular_box_state(S);
        const cudaError_t e = VFB_DISPATCH(L.storage, L.arith,
                                           LA::box_collide(b, L.is_even_timestep != 0, nullptr, nullptr,
                                                           as_stream(stream)));
        st = cuda_status(e, "K17CompressibleNavierStokes launch");
    } else if (S.slots && sim->neighbor_tables == 2) {
        const cudaError_t e = VFB_DISPATCH(L.storage, L.arith,
                                           LA::k17_list_staged(&L, S.slots, S.slots_stride, S.n_fluid, S.status(),
                                                               as_stream(stream)));
        st = cuda_status(e, "K17CompressibleNavierStokes launch");
    } else {
        st = run_k17(&L, S.fluid, S.n_fluid, VFB_COLLISION_DEFAULT, S.slots, S.slots_stride, stream);
    }
    if (st)
        return st;
    }
    {
        PhaseScope phase(sim->timers, VFB_PHASE_POST_COLLISION_BC, stream);
        if ((st = run_list(S, 0, S.velocity_fn, S.velocity, stream)) != VFB_OK)
            return st;
        if ((st = run_list(S, 1, S.noslip_fn, S.noslip, stream)) != VFB_OK)
            return st;
        if ((st = run_list(S, 3, S.slip_fn, S.slip, stream)) != VFB_OK)    // UpdateGrid27.cpp:240
            return st;
        st = run_geometry_post(S, stream);
        if (st)
            return st;
    }
    L.is_even_timestep = !L.is_even_timestep;
    PhaseScope phase(sim->timers, VFB_PHASE_PRE_COLLISION_BC, stream);
    st = run_geometry_pre(S, stream);
    if (st)
        return st;
    for (size_t i = 0; i < S.pressure.size(); ++i) {
        if (!S.pressure_fn[i] || !S.pressure[i].number_of_bc_nodes)
            continue;
        st = S.pressure_fn[i](&L, &S.pressure[i], stream);
        if (st)
            return st;
    }
    return VFB_OK;
}

// UpdateGrid27::updateGrid (UpdateGrid27.cpp:54-95): a level that has a finer one first lets it
// take two steps, then takes its own, then interpolates fine to coarse and coarse to fine
// (Refinement_noExchange, RefinementStrategy.cpp:169-178).
static int update_level(vfb_simulation *sim, size_t l, void *stream)
{
    const bool has_finer = l + 1 < sim->levels.size();
    int st;
    if (has_finer) {
        if ((st = update_level(sim, l + 1, stream)) != VFB_OK)
            return st;
        if ((st = update_level(sim, l + 1, stream)) != VFB_OK)
            return st;
    }
    SimLevel &S = sim->levels[l];
    if ((st = step_level(sim, S, stream)) != VFB_OK)
        return st;
    if (has_finer) {
        SimLevel &F = sim->levels[l + 1];
        if (sim->scale_fc && S.fc.number_of_cells) {
            PhaseScope phase(sim->timers, VFB_PHASE_SCALING_FC, stream);
            if ((st = sim->scale_fc(&S.level, &F.level, &S.fc, &S.fc_offsets, stream)) != VFB_OK)
                return st;
        }
        if (sim->scale_cf && S.cf.number_of_cells) {
            PhaseScope phase(sim->timers, VFB_PHASE_SCALING_CF, stream);
            if ((st = sim->scale_cf(&S.level, &F.level, &S.cf, &S.cf_offsets, stream)) != VFB_OK)
                return st;
        }
    }
    return VFB_OK;
}

static std::vector<int> parities(const vfb_simulation *sim)
{
    std::vector<int> p;
    for (const SimLevel &S : sim->levels)
        p.push_back(S.level.is_even_timestep);
    return p;
}

// capture sim->graph.steps coarse steps on `stream` (nothing runs); the host's per-level parity
// is put back to where the capture started, since the captured steps have not happened yet
static int capture_steps(vfb_simulation *sim, cudaStream_t stream)
{
    StepGraph &G = sim->graph;
    G.drop();
    const std::vector<int> start = parities(sim);
    cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
        return cuda_status(e, "beginning the capture of the step loop");
    int st = VFB_OK;
    for (int32_t t = 0; t < G.steps && st == VFB_OK; ++t)
        st = update_level(sim, 0, stream);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(stream, &g);
    for (size_t l = 0; l < sim->levels.size(); ++l)
        sim->levels[l].level.is_even_timestep = start[l];
    if (st == VFB_OK && e == cudaSuccess)
        e = cudaGraphInstantiate(&G.exec, g, 0);
    if (g)
        cudaGraphDestroy(g);
    if (st != VFB_OK)
        return st;
    if (e != cudaSuccess) {
        G.exec = nullptr;
        return cuda_status(e, "capturing the step loop");
    }
    G.stream = stream;
    G.parity = start;
    return VFB_OK;
}

int vfb_simulation_run(vfb_simulation *sim, uint32_t steps, void *stream)
{
    int st = vfb_simulation_check(sim);
    if (st)
        return st;
    nvtxRangePushA("vfb_simulation_run");
    uint32_t done = 0;
    StepGraph &G = sim->graph;
    bool drag = false;
    for (const SimLevel &S : sim->levels)
        drag = drag || (S.drag_work != nullptr && S.geometry_set && S.geometry.number_of_bc_nodes);
    // graphs: a stream of the caller's (capture needs one), no event timers, no per-step drag history
    if (G.steps > 0 && stream != nullptr && !sim->timers.on && !drag) {
        const cudaStream_t s = as_stream(stream);
        for (; !G.warm && done < steps && st == VFB_OK; ++done) {
            st = update_level(sim, 0, stream);     // lazy buffers come to exist outside a capture
            G.warm = st == VFB_OK;
        }
        while (st == VFB_OK && steps - done >= (uint32_t)G.steps) {
            if (!G.exec || G.stream != s || G.parity != parities(sim))
                st = capture_steps(sim, s);
            if (st == VFB_OK)
                st = cuda_status(cudaGraphLaunch(G.exec, s), "replaying the step loop");
            if (st == VFB_OK)
                done += (uint32_t)G.steps;    // an even number of steps: every parity as it was
        }
    }
    for (uint32_t t = done; t < steps && st == VFB_OK; ++t)
        st = update_level(sim, 0, stream);
    nvtxRangePop();
    if (sim->timers.on && !sim->timers.pending.empty()) {
        cudaError_t e = cudaStreamSynchronize(as_stream(stream));
        if (e == cudaSuccess)
            e = sim->timers.collect();
        if (e != cudaSuccess && st == VFB_OK)
            st = cuda_status(e, "phase timers");
        sim->timers.steps += steps;
    }
    return st;
}

int vfb_simulation_set_graph(vfb_simulation *sim, int32_t steps)
{
    if (!sim)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL simulation");
    if (steps < 0 || steps % 2 != 0 || steps > 1024)
        return fail(VFB_ERR_INVALID_ARGUMENT, "steps per graph must be 0 (off) or an even number up to 1024");
    config_changed(sim);
    sim->graph.steps = steps;
    return VFB_OK;
}

int vfb_simulation_set_timing(vfb_simulation *sim, int32_t on)
{
    if (!sim)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL simulation");
    config_changed(sim);
    sim->timers.on = on != 0;
    return VFB_OK;
}

int vfb_simulation_phase_times(vfb_simulation *sim, double *ms, uint64_t *steps, int32_t reset)
{
    if (!sim || !ms)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    for (int i = 0; i < VFB_PHASES; ++i)
        ms[i] = sim->timers.ms[i];
    if (steps)
        *steps = sim->timers.steps;
    if (reset) {
        for (double &v : sim->timers.ms)
            v = 0.0;
        sim->timers.steps = 0;
    }
    return VFB_OK;
}

int vfb_simulation_is_even_timestep(const vfb_simulation *sim, int32_t *is_even)
{
    return vfb_simulation_level_is_even_timestep(sim, 0, is_even);
}

int vfb_simulation_level_is_even_timestep(const vfb_simulation *sim, int32_t level, int32_t *is_even)
{
    if (!sim || !is_even)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (level < 0 || level >= (int32_t)sim->levels.size())
        return fail(VFB_ERR_INVALID_ARGUMENT, "no such level");
    *is_even = sim->levels[(size_t)level].level.is_even_timestep;
    return VFB_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------------------------
// (2b) structured boxes
// ---------------------------------------------------------------------------------------------
struct vfb_box {
    vfb_box_desc desc{};
    vfb::BoxState state{};
    bool even = true;
    uint64_t n = 0;
    void *dist = nullptr;
    uint8_t *mask = nullptr;
    double *partials = nullptr;     // per-block energy partials of one step
    uint64_t blocks = 0;
    double *energy_ring = nullptr;  // per-step results before they are copied out
    uint32_t ring_steps = 0;
    void *staging = nullptr;        // 4 real fields for init and output
    int *status = nullptr;          // device status word of the kernels (DeviceError)
    uint64_t launches = 0;          // kernels this box has launched
    uint64_t steps = 0;             // time steps done (counter of the inlet perturbation)
    // boundary conditions in box indices (device copies owned by the box)
    struct List {
        vfb_bc bc{};
        vfb_bc_fn fn = nullptr;
        int kind = -1;              // vfb::BCKind, -1 = no kernel
        std::vector<void *> owned;
        uint32_t *guard = nullptr;  // guard table of the list (guards.h), nullptr when nothing is guarded
        void *saved = nullptr;      // the guarded values, saved before the list writes
    } velocity, noslip, slip, geometry;
    struct Pressure {
        vfb_directional_bc bc{};
        int kind = 0;                 // vfb::PressureKind
        std::vector<void *> owned;
    };
    double outflow_correction = 0.0;
    std::vector<Pressure> pressure;
    void *velocity_base = nullptr;  // unperturbed inlet velocities (3 x n reals)
    uint64_t perturb_seed = 0;
    double perturb_amplitude = 0.0;
    double *drag_work = nullptr;    // 6 n doubles + sum scratch
    double *drag_history = nullptr;
    uint32_t drag_history_len = 0;
    uint64_t drag_steps = 0;
};

namespace {
constexpr uint32_t kRingSteps = 1024;

void free_list(vfb_box::List &l)
{
    for (void *p : l.owned)
        cudaFree(p);
    l = vfb_box::List();
}

void box_free(vfb_box *b)
{
    if (!b)
        return;
    free_list(b->velocity);
    free_list(b->noslip);
    free_list(b->slip);
    free_list(b->geometry);
    for (auto &p : b->pressure)
        for (void *q : p.owned)
            cudaFree(q);
    b->pressure.clear();
    cudaFree(b->velocity_base);
    cudaFree(b->drag_work);
    cudaFree(b->dist);
    cudaFree(b->mask);
    cudaFree(b->partials);
    cudaFree(b->energy_ring);
    cudaFree(b->staging);
    cudaFree(b->status);
}
} // namespace

extern "C" {

int vfb_box_create(const vfb_box_desc *d, vfb_box **out)
{
    if (!d || !out)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (d->nx < 2 || d->ny < 2 || d->nz < 2 || d->ny > 65535 || d->nz > 65535)
        return fail(VFB_ERR_INVALID_ARGUMENT, "box extents must be >= 2 (ny, nz <= 65535)");
    const uint64_t n = (uint64_t)d->nx * d->ny * d->nz;
    if (n >= 0xffffffffull)
        return fail(VFB_ERR_INVALID_ARGUMENT, "box has too many nodes for 32-bit indices");
    if (!storage_ok(d->storage))
        return fail(VFB_ERR_INVALID_ARGUMENT, "unknown storage format");
    if (d->arith != VFB_ARITH_FAST && d->arith != VFB_ARITH_EXACT)
        return fail(VFB_ERR_INVALID_ARGUMENT, "unknown arithmetic mode");
    if (d->arith == VFB_ARITH_EXACT && d->storage > VFB_STORAGE_F32)
        return fail(VFB_ERR_UNSUPPORTED, "exact arithmetic is built for F64 and F32 storage only");
    if (!(d->omega > 0.0 && d->omega < 2.0))
        return fail(VFB_ERR_INVALID_ARGUMENT, "omega must lie in (0, 2)");
    if ((!d->periodic_x || !d->periodic_y || !d->periodic_z) && !d->mask)
        return fail(VFB_ERR_INVALID_ARGUMENT, "a non-periodic box needs a mask with a solid border");
    vfb_box *b = new vfb_box();
    b->desc = *d;
    b->desc.mask = nullptr;
    b->n = n;
    // planes padded to 256 bytes so every plane starts aligned
    const size_t sb = storage_bytes(d->storage);
    const uint64_t align_el = 256 / sb;
    const uint64_t pitch = (n + align_el - 1) / align_el * align_el;
    cudaError_t e = cudaMalloc(&b->dist, pitch * 27 * sb);
    if (e == cudaSuccess && d->mask) {
        e = cudaMalloc((void **)&b->mask, n);
        if (e == cudaSuccess)
            e = cudaMemcpy(b->mask, d->mask, n, cudaMemcpyHostToDevice);
    }
    vfb::BoxState &s = b->state;
    s.dist = b->dist;
    s.pitch = pitch;
    s.nx = d->nx;
    s.ny = d->ny;
    s.nz = d->nz;
    s.periodic_x = d->periodic_x;
    s.periodic_y = d->periodic_y;
    s.periodic_z = d->periodic_z;
    s.mask = b->mask;
    s.omega = d->omega;
    s.fx = d->forces[0] * 0.5;
    s.fy = d->forces[1] * 0.5;
    s.fz = d->forces[2] * 0.5;
    for (int i = 0; i < 3; ++i)
        s.lim[i] = d->quadric_limiters[i];
    b->blocks = vfb::box_blocks(s);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&b->partials, 2 * (b->blocks + vfb::kReduceMaxChunks) * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&b->energy_ring, 2 * (size_t)kRingSteps * sizeof(double));
    b->ring_steps = kRingSteps;
    if (e == cudaSuccess)
        e = cudaMalloc(&b->staging, 4 * n * real_bytes(d->storage));
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&b->status, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemset(b->status, 0, sizeof(int));
    s.status = b->status;
    s.variant = 0;
    s.async_blocks_per_sm = 0;
    s.async_smem_kb = 0;
    if (e != cudaSuccess) {
        box_free(b);
        delete b;
        return cuda_status(e, "box allocation");
    }
    *out = b;
    return VFB_OK;
}

int vfb_box_destroy(vfb_box *box)
{
    box_free(box);
    delete box;
    return VFB_OK;
}

int vfb_box_device_bytes(const vfb_box *box, uint64_t *bytes)
{
    if (!box || !bytes)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    const uint64_t sb = storage_bytes(box->desc.storage);
    *bytes = box->state.pitch * 27 * sb + (box->mask ? box->n : 0) + 2 * box->blocks * 8 + 2 * (uint64_t)box->ring_steps * 8
           + 4 * box->n * real_bytes(box->desc.storage);
    return VFB_OK;
}

int vfb_box_init(vfb_box *box, const void *rho, const void *ux, const void *uy, const void *uz, int32_t from_host,
                 void *stream)
{
    if (!box || !rho || !ux || !uy || !uz)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = as_stream(stream);
    const size_t rb = real_bytes(box->desc.storage), fb = box->n * rb;
    const void *f[4] = { rho, ux, uy, uz };
    const void *dev[4];
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
        if (from_host) {
            void *dst = static_cast<char *>(box->staging) + i * fb;
            e = cudaMemcpyAsync(dst, f[i], fb, cudaMemcpyHostToDevice, s);
            dev[i] = dst;
        } else {
            dev[i] = f[i];
        }
    }
    // PreProcessorImp::init (PreProcessorImp.cpp:50-58): odd parity, then even
    if (e == cudaSuccess)
        e = VFB_DISPATCH(box->desc.storage, box->desc.arith, LA::box_init(box->state, false, dev[0], dev[1], dev[2], dev[3], s));
    if (e == cudaSuccess)
        e = VFB_DISPATCH(box->desc.storage, box->desc.arith, LA::box_init(box->state, true, dev[0], dev[1], dev[2], dev[3], s));
    box->even = true;
    return cuda_status(e, "box init");
}

namespace {

// the box as a level of the boundary, drag and init launchers (plane stride = pitch; neighbours by
// index arithmetic)
vfb_level box_level(const vfb_box *b)
{
    vfb_level L{};
    L.storage = b->desc.storage;
    L.arith = b->desc.arith;
    L.is_even_timestep = b->even ? 1 : 0;
    L.number_of_nodes = b->state.pitch;
    L.distributions = b->dist;
    L.omega = b->desc.omega;
    return L;
}

vfb::NodeAddr box_addr(const vfb_box *b)
{
    return vfb::NodeAddr{ b->desc.nx, b->desc.ny, b->desc.nz,
                          (b->desc.periodic_x ? 1 : 0) | (b->desc.periodic_y ? 2 : 0) | (b->desc.periodic_z ? 4 : 0) };
}

cudaError_t box_run_list(vfb_box *b, const vfb_box::List &l, cudaStream_t s)
{
    if (l.kind < 0 || l.bc.number_of_bc_nodes == 0)
        return cudaSuccess;
    const vfb_level L = box_level(b);
    const vfb::NodeAddr a = box_addr(b);
    ++b->launches;
    if (l.guard)
        ++b->launches;
    return VFB_DISPATCH(b->desc.storage, b->desc.arith, LA::bc(&L, &l.bc, l.kind, s, &a, nullptr, l.guard, l.saved));
}

// one step's boundary work around the collision, in the order of vfb_simulation_run
cudaError_t box_post_collision(vfb_box *b, cudaStream_t s)
{
    cudaError_t e = cudaSuccess;
    if (b->velocity_base && b->velocity.bc.number_of_bc_nodes) {
        e = VFB_DISPATCH(b->desc.storage, b->desc.arith,
                         LA::inlet_perturbation(b->velocity_base, const_cast<void *>(b->velocity.bc.vx),
                                                b->velocity.bc.number_of_bc_nodes, b->perturb_seed, b->steps,
                                                b->perturb_amplitude, s));
        ++b->launches;
    }
    if (e == cudaSuccess)
        e = box_run_list(b, b->velocity, s);
    if (e == cudaSuccess)
        e = box_run_list(b, b->noslip, s);
    if (e == cudaSuccess)
        e = box_run_list(b, b->slip, s);        // runSlipBCKernelPost (UpdateGrid27.cpp:240)
    const uint32_t ng = b->geometry.bc.number_of_bc_nodes;
    if (e == cudaSuccess && b->drag_work && ng) {
        const vfb_level L = box_level(b);
        const vfb::NodeAddr a = box_addr(b);
        double *w = b->drag_work;
        e = VFB_DISPATCH(b->desc.storage, b->desc.arith,
                         LA::drag_lift(&L, &b->geometry.bc, false, w + 3 * (size_t)ng, w + 4 * (size_t)ng,
                                       w + 5 * (size_t)ng, s, &a));
        ++b->launches;
    }
    if (e == cudaSuccess)
        e = box_run_list(b, b->geometry, s);
    return e;
}

cudaError_t box_pre_collision(vfb_box *b, cudaStream_t s)
{
    cudaError_t e = cudaSuccess;
    const uint32_t ng = b->geometry.bc.number_of_bc_nodes;
    if (b->drag_work && ng) {
        const vfb_level L = box_level(b);
        const vfb::NodeAddr a = box_addr(b);
        double *w = b->drag_work;
        e = VFB_DISPATCH(b->desc.storage, b->desc.arith,
                         LA::drag_lift(&L, &b->geometry.bc, true, w, w + ng, w + 2 * (size_t)ng, s, &a));
        const double *pre[3] = { w, w + ng, w + 2 * (size_t)ng };
        const double *post[3] = { w + 3 * (size_t)ng, w + 4 * (size_t)ng, w + 5 * (size_t)ng };
        if (e == cudaSuccess)
            e = vfb::drag_lift_sum(pre, post, ng, w + 6 * (size_t)ng,
                                   b->drag_history + 3 * (b->drag_steps % b->drag_history_len), s);
        b->launches += 3;
        ++b->drag_steps;
    }
    for (size_t i = 0; i < b->pressure.size() && e == cudaSuccess; ++i) {
        const vfb_level L = box_level(b);
        const vfb::NodeAddr a = box_addr(b);
        vfb_level Lp = L;
        Lp.outflow_pressure_correction_factor = b->outflow_correction;
        e = VFB_DISPATCH(b->desc.storage, b->desc.arith,
                         LA::pressure(&Lp, &b->pressure[i].bc, s, &a, b->pressure[i].kind));
        ++b->launches;
    }
    return e;
}

} // namespace

int vfb_box_step(vfb_box *box, uint32_t steps, double *energy, int32_t energy_on_host, void *stream)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL box");
    const vfb::NvtxRange range("vfb_box_step");
    cudaStream_t s = as_stream(stream);
    cudaError_t e = cudaSuccess;
    uint32_t done = 0;
    while (done < steps && e == cudaSuccess) {
        const uint32_t chunk = energy && energy_on_host ? std::min<uint32_t>(steps - done, box->ring_steps) : steps - done;
        for (uint32_t t = 0; t < chunk && e == cudaSuccess; ++t) {
            double *partials = energy ? box->partials : nullptr;
            uint64_t n_partials = 0;
            e = VFB_DISPATCH(box->desc.storage, box->desc.arith,
                             LA::box_collide(box->state, box->even, partials, &n_partials, s));
            ++box->launches;
            if (e == cudaSuccess && energy) {
                double *dst = energy_on_host ? box->energy_ring + 2 * t : energy + 2 * (uint64_t)(done + t);
                e = vfb::reduce_partials_wide(box->partials, n_partials, box->partials + 2 * box->blocks, dst, s);
                box->launches += n_partials > vfb::kReduceDirect ? 2 : 1;
            }
            if (e == cudaSuccess)
                e = box_post_collision(box, s);
            box->even = !box->even;
            if (e == cudaSuccess)
                e = box_pre_collision(box, s);
            ++box->steps;
        }
        if (e == cudaSuccess && energy && energy_on_host)
            e = cudaMemcpyAsync(energy + 2 * (uint64_t)done, box->energy_ring, 2 * sizeof(double) * chunk,
                                cudaMemcpyDeviceToHost, s);
        done += chunk;
    }
    return cuda_status(e, "box step");
}

int vfb_box_fields(vfb_box *box, void *rho, void *ux, void *uy, void *uz, int32_t to_host, void *stream)
{
    if (!box || !rho || !ux || !uy || !uz)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = as_stream(stream);
    const size_t rb = real_bytes(box->desc.storage), fb = box->n * rb;
    void *out[4] = { rho, ux, uy, uz };
    void *dev[4];
    for (int i = 0; i < 4; ++i)
        dev[i] = to_host ? static_cast<char *>(box->staging) + i * fb : out[i];
    cudaError_t e = VFB_DISPATCH(box->desc.storage, box->desc.arith,
                                 LA::box_macros(box->state, box->even, dev[0], dev[1], dev[2], dev[3], s));
    for (int i = 0; i < 4 && e == cudaSuccess && to_host; ++i)
        e = cudaMemcpyAsync(out[i], dev[i], fb, cudaMemcpyDeviceToHost, s);
    return cuda_status(e, "box fields");
}

int vfb_box_status(vfb_box *box, int32_t *device_status, void *stream)
{
    if (!box || !device_status)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    int v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, box->status, sizeof(int), cudaMemcpyDeviceToHost, as_stream(stream));
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(as_stream(stream));
    *device_status = v;
    int st = cuda_status(e, "box status");
    if (st)
        return st;
    if (v != 0)
        return fail(VFB_ERR_CUDA, "a kernel of this box gave up waiting for its staged copies");
    return VFB_OK;
}

int vfb_box_set_kernel_variant(vfb_box *box, int32_t variant)
{
    if (!box || variant < 0 || variant > 5)
        return fail(VFB_ERR_INVALID_ARGUMENT, "variant must be 0 (choose), 1 (direct loads), 2 (TMA-staged), "
                                              "3 (per-thread async copies), 4 (packed FP32x2 pairs) or 5 "
                                              "(persistent, next node's loads in flight)");
    if (variant == 4 && (box->desc.storage == VFB_STORAGE_F64 || box->desc.arith == VFB_ARITH_EXACT))
        return fail(VFB_ERR_UNSUPPORTED, "packed FP32x2 pairs: FP32 arithmetic (F32, F16, BF16, E3M12 storage), FMA "
                                         "variant");
    if (variant == 3 && box->desc.storage > VFB_STORAGE_F32)
        return fail(VFB_ERR_UNSUPPORTED, "per-thread async copies move 4 or 8 bytes: F64 and F32 storage only");
    if (variant == 2 && box->desc.nx % 32 != 0)
        return fail(VFB_ERR_UNSUPPORTED, "the TMA-staged kernel needs nx % 32 == 0");
    box->state.variant = variant;
    return VFB_OK;
}

int vfb_box_set_bc(vfb_box *box, int32_t kind, int32_t variant, const int32_t *k, const void *q27, uint32_t n,
                   const void *ux, const void *uy, const void *uz)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL box");
    if (kind != VFB_BOX_BC_VELOCITY && kind != VFB_BOX_BC_NOSLIP && kind != VFB_BOX_BC_GEOMETRY &&
        kind != VFB_BOX_BC_SLIP)
        return fail(VFB_ERR_INVALID_ARGUMENT, "kind must be VFB_BOX_BC_VELOCITY, _NOSLIP, _GEOMETRY or _SLIP");
    if (n && (!k || !q27))
        return fail(VFB_ERR_INVALID_ARGUMENT, "node indices or q are NULL");
    if (kind == VFB_BOX_BC_VELOCITY && n && (!ux || !uy || !uz))
        return fail(VFB_ERR_INVALID_ARGUMENT, "a velocity BC needs the wall velocities");
    int bc_kind = -1;
    if (kind == VFB_BOX_BC_VELOCITY) {
        switch (variant) {
        case VFB_VELOCITY_BOUNCE_BACK: bc_kind = vfb::kVelocityBB; break;
        case VFB_VELOCITY_INTERPOLATED_COMPRESSIBLE: bc_kind = vfb::kVelocityInterp; break;
        case VFB_VELOCITY_INTERPOLATED_INCOMPRESSIBLE: bc_kind = vfb::kVelocityInterpIncomp; break;
        case VFB_VELOCITY_WITH_PRESSURE_INTERPOLATED_COMPRESSIBLE: bc_kind = vfb::kVelocityWithPressure; break;
        case VFB_VELOCITY_NOT_SPECIFIED: break;
        default: return fail(VFB_ERR_UNSUPPORTED, "velocity BC variant not built for boxes");
        }
    } else if (kind == VFB_BOX_BC_SLIP) {
        switch (variant) {
        case VFB_SLIP_COMPRESSIBLE: bc_kind = vfb::kSlipInterp; break;
        case VFB_SLIP_NOT_SPECIFIED: break;
        default: return fail(VFB_ERR_UNSUPPORTED, "slip BC variant not built for boxes");
        }
    } else {
        switch (variant) {
        case VFB_NOSLIP_DELAY_BOUNCE_BACK: break;
        case VFB_NOSLIP_BOUNCE_BACK: bc_kind = vfb::kNoSlipBB; break;
        case VFB_NOSLIP_INTERPOLATED_COMPRESSIBLE: bc_kind = vfb::kNoSlipInterp; break;
        case VFB_NOSLIP_INTERPOLATED_INCOMPRESSIBLE: bc_kind = vfb::kNoSlipInterpIncomp; break;
        default: return fail(VFB_ERR_UNSUPPORTED, "no-slip BC variant not built for boxes");
        }
    }
    const uint64_t nn = (uint64_t)box->desc.nx * box->desc.ny * box->desc.nz;
    for (uint32_t i = 0; i < n; ++i)
        if (k[i] < 0 || (uint64_t)k[i] >= nn)
            return fail(VFB_ERR_INVALID_ARGUMENT, "a BC node index lies outside the box");
    vfb_box::List &l = kind == VFB_BOX_BC_VELOCITY ? box->velocity
                     : kind == VFB_BOX_BC_NOSLIP ? box->noslip
                     : kind == VFB_BOX_BC_SLIP   ? box->slip
                                                 : box->geometry;
    free_list(l);
    if (kind == VFB_BOX_BC_VELOCITY) {
        cudaFree(box->velocity_base);
        box->velocity_base = nullptr;
    }
    if (kind == VFB_BOX_BC_GEOMETRY) {
        cudaFree(box->drag_work);
        box->drag_work = nullptr;
        box->drag_history = nullptr;
    }
    const size_t rb = real_bytes(box->desc.storage);
    void *dk = nullptr, *dq = nullptr, *dv = nullptr, *dg = nullptr, *ds = nullptr;
    cudaError_t e = cudaSuccess;
    // links cut from both ends between nodes of this list: which post-collision values to save
    std::vector<uint32_t> table;
    const int periodic = (box->desc.periodic_x ? 1 : 0) | (box->desc.periodic_y ? 2 : 0) | (box->desc.periodic_z ? 4 : 0);
    uint32_t n_saved = 0;
    if (n)
        n_saved = rb == 8 ? vfb::bc_guard_tables(k, static_cast<const double *>(q27), n, box->desc.nx, box->desc.ny,
                                                 box->desc.nz, periodic, table)
                          : vfb::bc_guard_tables(k, static_cast<const float *>(q27), n, box->desc.nx, box->desc.ny,
                                                 box->desc.nz, periodic, table);
    if (n) {
        e = cudaMalloc(&dk, n * sizeof(int32_t));
        if (e == cudaSuccess)
            e = cudaMemcpy(dk, k, n * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && n_saved) {
            e = cudaMalloc(&dg, table.size() * sizeof(uint32_t));
            if (e == cudaSuccess)
                e = cudaMemcpy(dg, table.data(), table.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
            if (e == cudaSuccess)
                e = cudaMalloc(&ds, (size_t)n_saved * rb);
        }
        if (e == cudaSuccess)
            e = cudaMalloc(&dq, (size_t)27 * n * rb);
        if (e == cudaSuccess)
            e = cudaMemcpy(dq, q27, (size_t)27 * n * rb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && kind == VFB_BOX_BC_VELOCITY) {
            e = cudaMalloc(&dv, (size_t)3 * n * rb);
            const void *src[3] = { ux, uy, uz };
            for (int a = 0; a < 3 && e == cudaSuccess; ++a)
                e = cudaMemcpy(static_cast<char *>(dv) + a * n * rb, src[a], n * rb, cudaMemcpyHostToDevice);
        }
    }
    if (e != cudaSuccess) {
        cudaFree(dk);
        cudaFree(dq);
        cudaFree(dv);
        cudaFree(dg);
        cudaFree(ds);
        return cuda_status(e, "box BC upload");
    }
    l.owned = { dk, dq, dv, dg, ds };
    l.guard = static_cast<uint32_t *>(dg);
    l.saved = ds;
    l.bc.k = static_cast<const int32_t *>(dk);
    l.bc.q27 = dq;
    l.bc.number_of_bc_nodes = n;
    if (dv) {
        l.bc.vx = dv;
        l.bc.vy = static_cast<char *>(dv) + n * rb;
        l.bc.vz = static_cast<char *>(dv) + 2 * n * rb;
    }
    l.kind = bc_kind;
    return VFB_OK;
}

int vfb_box_add_pressure_bc(vfb_box *box, int32_t variant, const int32_t *k, const int32_t *k_neighbor, const void *rho,
                            uint32_t n, int32_t direction)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL box");
    int pkind = 0;
    switch (variant) {
    case VFB_PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE: pkind = vfb::kPressureNeqComp; break;
    case VFB_PRESSURE_NON_EQUILIBRIUM_INCOMPRESSIBLE: pkind = vfb::kPressureNeqIncomp; break;
    case VFB_PRESSURE_OUTFLOW_NON_REFLECTIVE: pkind = vfb::kOutflowNonReflecting; break;
    case VFB_PRESSURE_OUTFLOW_NON_REFLECTIVE_PRESSURE_CORRECTION: pkind = vfb::kOutflowPressureCorrection; break;
    default: return fail(VFB_ERR_UNSUPPORTED, "pressure BC variant not built for boxes");
    }
    if (direction < VFB_DIR_P00 || direction > VFB_DIR_00M)
        return fail(VFB_ERR_INVALID_ARGUMENT, "direction must be one of the six face directions");
    if (n && (!k || !k_neighbor || !rho))
        return fail(VFB_ERR_INVALID_ARGUMENT, "pressure BC arrays are NULL");
    const uint64_t nn = (uint64_t)box->desc.nx * box->desc.ny * box->desc.nz;
    for (uint32_t i = 0; i < n; ++i)
        if (k[i] < 0 || (uint64_t)k[i] >= nn || k_neighbor[i] < 0 || (uint64_t)k_neighbor[i] >= nn)
            return fail(VFB_ERR_INVALID_ARGUMENT, "a pressure BC node index lies outside the box");
    const size_t rb = real_bytes(box->desc.storage);
    vfb_box::Pressure p;
    void *dk = nullptr, *dn = nullptr, *dr = nullptr;
    cudaError_t e = cudaSuccess;
    if (n) {
        e = cudaMalloc(&dk, n * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMemcpy(dk, k, n * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&dn, n * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMemcpy(dn, k_neighbor, n * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&dr, n * rb);
        if (e == cudaSuccess) e = cudaMemcpy(dr, rho, n * rb, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        cudaFree(dk);
        cudaFree(dn);
        cudaFree(dr);
        return cuda_status(e, "box pressure BC upload");
    }
    p.owned = { dk, dn, dr };
    p.bc = vfb_directional_bc{ static_cast<const int32_t *>(dk), static_cast<const int32_t *>(dn), dr, n, direction };
    p.kind = pkind;
    box->pressure.push_back(p);
    return VFB_OK;
}

int vfb_box_set_outflow_pressure_correction(vfb_box *box, double factor)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL box");
    box->outflow_correction = factor;
    return VFB_OK;
}

int vfb_box_set_velocity_perturbation(vfb_box *box, uint64_t seed, double amplitude)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL box");
    const uint32_t n = box->velocity.bc.number_of_bc_nodes;
    if (!n)
        return fail(VFB_ERR_INVALID_ARGUMENT, "set the velocity BC first");
    if (!(amplitude >= 0.0 && amplitude < 1.0))
        return fail(VFB_ERR_INVALID_ARGUMENT, "amplitude must lie in [0, 1)");
    const size_t bytes = (size_t)3 * n * real_bytes(box->desc.storage);
    if (!box->velocity_base) {
        cudaError_t e = cudaMalloc(&box->velocity_base, bytes);
        if (e == cudaSuccess)
            e = cudaMemcpy(box->velocity_base, box->velocity.bc.vx, bytes, cudaMemcpyDeviceToDevice);
        if (e != cudaSuccess) {
            cudaFree(box->velocity_base);
            box->velocity_base = nullptr;
            return cuda_status(e, "box velocity perturbation");
        }
    }
    box->perturb_seed = seed;
    box->perturb_amplitude = amplitude;
    return VFB_OK;
}

int vfb_box_set_drag_lift(vfb_box *box, double *force_history, uint32_t history_steps)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL box");
    const uint32_t ng = box->geometry.bc.number_of_bc_nodes;
    if (!ng)
        return fail(VFB_ERR_INVALID_ARGUMENT, "drag and lift need a geometry BC with nodes");
    if (!force_history || !history_steps)
        return fail(VFB_ERR_INVALID_ARGUMENT, "drag and lift need a force history of at least one step");
    if (!box->drag_work) {
        const cudaError_t e = cudaMalloc((void **)&box->drag_work,
                                         6 * (size_t)ng * sizeof(double) + vfb_drag_lift_workspace_bytes(ng));
        if (e != cudaSuccess)
            return cuda_status(e, "box drag workspace");
    }
    box->drag_history = force_history;
    box->drag_history_len = history_steps;
    box->drag_steps = 0;
    return VFB_OK;
}

int vfb_box_kernel_launches(const vfb_box *box, uint64_t *count)
{
    if (!box || !count)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *count = box->launches;
    return VFB_OK;
}

int vfb_box_set_launch_shape(vfb_box *box, int32_t blocks_per_sm, int32_t smem_kb)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "box is NULL");
    if (blocks_per_sm < 0 || blocks_per_sm > 8)
        return fail(VFB_ERR_INVALID_ARGUMENT, "blocks_per_sm must lie in [0, 8]");
    static const int kb[] = { 0, 64, 100, 132, 164, 196, 228 };
    if (std::find(std::begin(kb), std::end(kb), smem_kb) == std::end(kb))
        return fail(VFB_ERR_INVALID_ARGUMENT, "smem_kb must be 0, 64, 100, 132, 164, 196 or 228");
    box->state.async_blocks_per_sm = blocks_per_sm;
    box->state.async_smem_kb = smem_kb;
    return VFB_OK;
}

static int box_copy_populations(vfb_box *box, void *host_or_dev, const void *src_any, bool out, int32_t on_host,
                                void *stream)
{
    const size_t sb = storage_bytes(box->desc.storage);
    const size_t row = (size_t)box->n * sb, pitch = (size_t)box->state.pitch * sb;
    cudaStream_t s = as_stream(stream);
    const cudaMemcpyKind kind = on_host ? (out ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice)
                                        : cudaMemcpyDeviceToDevice;
    cudaError_t e = out ? cudaMemcpy2DAsync(host_or_dev, row, box->dist, pitch, row, 27, kind, s)
                        : cudaMemcpy2DAsync(box->dist, pitch, src_any, row, row, 27, kind, s);
    if (e == cudaSuccess && on_host)
        e = cudaStreamSynchronize(s);
    return cuda_status(e, "box population copy");
}

int vfb_box_read_populations(vfb_box *box, void *out, int32_t to_host, int32_t *is_even, void *stream)
{
    if (!box || !out || !is_even)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *is_even = box->even ? 1 : 0;
    return box_copy_populations(box, out, nullptr, true, to_host, stream);
}

int vfb_box_write_populations(vfb_box *box, const void *src, int32_t from_host, int32_t is_even, void *stream)
{
    if (!box || !src)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    const int st = box_copy_populations(box, nullptr, src, false, from_host, stream);
    if (st == VFB_OK)
        box->even = is_even != 0;
    return st;
}

int vfb_box_collide_planes(vfb_box *box, int32_t z_begin, int32_t z_end, void *stream)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL box");
    if (z_begin < 0 || z_end > box->desc.nz || z_begin > z_end)
        return fail(VFB_ERR_INVALID_ARGUMENT, "planes must satisfy 0 <= z_begin <= z_end <= nz");
    const cudaError_t e = VFB_DISPATCH(box->desc.storage, box->desc.arith,
                                       LA::box_collide_planes(box->state, box->even, z_begin, z_end, as_stream(stream)));
    if (z_end > z_begin)
        ++box->launches;
    return cuda_status(e, "box collision of planes");
}

int vfb_box_collide_border(vfb_box *box, int32_t z, void *up, void *down, void *stream)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL box");
    if (z < 0 || z + 1 >= box->desc.nz)
        return fail(VFB_ERR_INVALID_ARGUMENT, "the border plane must satisfy 0 <= z < nz - 1");
    const cudaError_t e = VFB_DISPATCH(box->desc.storage, box->desc.arith,
                                       LA::box_collide_border(box->state, box->even, z, up, down, as_stream(stream)));
    ++box->launches;
    return cuda_status(e, "box collision of a border plane");
}

int vfb_box_ipc_handle(const vfb_box *box, void *handle)
{
    if (!box || !handle)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    static_assert(sizeof(cudaIpcMemHandle_t) == VFB_IPC_HANDLE_BYTES, "IPC handle size");
    cudaIpcMemHandle_t h;
    const cudaError_t e = cudaIpcGetMemHandle(&h, box->dist);
    if (e != cudaSuccess)
        return cuda_status(e, "IPC handle of a population array");
    std::memcpy(handle, &h, sizeof h);
    return VFB_OK;
}

int vfb_ipc_open(const void *handle, void **ptr)
{
    if (!handle || !ptr)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaIpcMemHandle_t h;
    std::memcpy(&h, handle, sizeof h);
    *ptr = nullptr;
    return cuda_status(cudaIpcOpenMemHandle(ptr, h, cudaIpcMemLazyEnablePeerAccess), "opening an IPC handle");
}

int vfb_ipc_close(void *ptr)
{
    if (!ptr)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL pointer");
    return cuda_status(cudaIpcCloseMemHandle(ptr), "closing an IPC mapping");
}

int vfb_box_toggle_parity(vfb_box *box)
{
    if (!box)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL box");
    box->even = !box->even;
    ++box->steps;
    return VFB_OK;
}

int vfb_box_populations(const vfb_box *box, void **dist, uint64_t *pitch, int32_t *is_even)
{
    if (!box || !dist || !pitch || !is_even)
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *dist = box->dist;
    *pitch = box->state.pitch;
    *is_even = box->even ? 1 : 0;
    return VFB_OK;
}

} // extern "C"
