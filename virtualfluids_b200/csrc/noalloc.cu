// The FP64 mass / kinetic-energy reduction over a node list without any allocation.
//
// vfb_mass_energy needs device scratch for its per-block partial sums and takes it from the
// caller. Some callers cannot provide it: a host that owns every byte of device memory and gives
// libraries none, a time loop under a no-allocation policy, or code that must not call cudaMalloc
// because cudaMalloc can synchronise the device. vfb_mass_energy_no_alloc serves them from a
// fixed array in this file's device memory instead.
//
// The array is a file-scope __device__ variable: every GPU that loads the library holds it
// (about 1 MiB) until the process exits. Its host-side name is only a stand-in, so every call
// looks the array's device address up with cudaGetSymbolAddress on the current device. The first
// such lookup on a device loads the library's device code there, so the first call on a device
// should come before any stream capture; later lookups are cheap. The address is not cached: a
// cudaDeviceReset can reload the module at another address. All calls share the array: each call
// overwrites every entry it reads back (nothing has to start at zero), and calls that overlap on
// the GPU race on it.
#include <cuda_runtime.h>

#include <cstdint>

#include "launch.h"
#include "vfb.h"

namespace {

constexpr uint32_t kThreadsPerBlock = 256;                            // energy_list_kernel's block size
constexpr uint64_t kMaxBlocks = VFB_NO_ALLOC_MAX_NODES / kThreadsPerBlock;
static_assert(VFB_NO_ALLOC_MAX_NODES % kThreadsPerBlock == 0, "the node limit is a whole number of blocks");

// per-block {mass, energy} partials, then the two reduced sums
__device__ __align__(256) double g_mass_energy_scratch[2 * kMaxBlocks + 2];

// device address of the scratch array on the current device
cudaError_t scratch_address(double **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_mass_energy_scratch);
    if (e != cudaSuccess)
        return e;
    *out = static_cast<double *>(p);
    return cudaSuccess;
}

int fail(int status, const char *msg)
{
    vfb::set_last_error(msg);
    return status;
}

} // namespace

extern "C" {

int vfb_mass_energy_no_alloc(const vfb_level *level, const uint32_t *node_indices, uint32_t size, double out[2],
                             void *stream)
{
    // the same level checks as vfb_mass_energy, before any early return
    const int st = vfb::check_level_status(level);
    if (st)
        return st;
    if (!out || (size && !node_indices))
        return fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (size > VFB_NO_ALLOC_MAX_NODES)
        return fail(VFB_ERR_INVALID_ARGUMENT,
                    "vfb_mass_energy_no_alloc: more nodes than VFB_NO_ALLOC_MAX_NODES (16777216); "
                    "use vfb_mass_energy with caller workspace");
    if (size == 0) {
        out[0] = out[1] = 0.0;
        return VFB_OK;
    }
    double *scratch = nullptr;
    cudaError_t e = scratch_address(&scratch);
    if (e != cudaSuccess)
        return vfb::cuda_error_status(e, "cudaGetSymbolAddress of the reduction scratch array");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t blocks = (size + kThreadsPerBlock - 1) / kThreadsPerBlock;
    double *partials = scratch;
    double *result = scratch + 2 * kMaxBlocks;
    // the same partial-sum kernel and the same fixed-order reduction as vfb_mass_energy
    if (level->arith == VFB_ARITH_EXACT) {
        if (level->storage == VFB_STORAGE_F64)
            e = vfb::exact::Launchers<double>::energy_list(level, node_indices, size, partials, s);
        else
            e = vfb::exact::Launchers<float>::energy_list(level, node_indices, size, partials, s);
    } else {
        switch (level->storage) {
        case VFB_STORAGE_F64: e = vfb::fast::Launchers<double>::energy_list(level, node_indices, size, partials, s); break;
        case VFB_STORAGE_F32: e = vfb::fast::Launchers<float>::energy_list(level, node_indices, size, partials, s); break;
        case VFB_STORAGE_F16: e = vfb::fast::Launchers<__half>::energy_list(level, node_indices, size, partials, s); break;
        case VFB_STORAGE_E3M12:
            e = vfb::fast::Launchers<vfb::e3m12_t>::energy_list(level, node_indices, size, partials, s);
            break;
        default: e = vfb::fast::Launchers<__nv_bfloat16>::energy_list(level, node_indices, size, partials, s); break;
        }
    }
    if (e == cudaSuccess)
        e = vfb::reduce_partials(partials, blocks, result, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, result, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    return vfb::cuda_error_status(e, "mass/energy reduction (no allocation)");
}

} // extern "C"
