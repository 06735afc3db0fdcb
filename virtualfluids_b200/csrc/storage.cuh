// Storage formats of the population array.
//
// The reference stores "well-conditioned" populations f_i - w_i in `real` (float or double,
// src/basics/DataTypes.h:39-43; InitNavierStokesCompressible_Device.cu:175-202). Here the
// storage type is a runtime choice:
//   F64  : f - w as double, arithmetic in double (the reference's VF_DOUBLE_ACCURACY build)
//   F32  : f - w as float,  arithmetic in float  (the reference's default GPU build)
//   F16  : (f - w) / w as IEEE half,  arithmetic in float
//   BF16 : (f - w) / w as bfloat16,   arithmetic in float
// Dividing by the lattice weight puts all 27 directions on one scale, O(drho + 3 c.u), so the
// 16-bit formats spend their exponent range on the same magnitudes for every direction and
// small corner populations do not fall into the subnormal range. 1/w is 27/8, 27/2, 54 or 216.
//
// The direction argument d is always a loop index of a fully unrolled 27-direction loop, so
// weight(d) folds to a constant.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lattice.cuh"

namespace vfb {

enum StorageKind : int { kStoreF64 = 0, kStoreF32 = 1, kStoreF16 = 2, kStoreBF16 = 3 };

template <class S>
struct Codec;

template <>
struct Codec<double> {
    using compute = double;
    __device__ __forceinline__ static double load(const double *p, int) { return *p; }
    __device__ __forceinline__ static void store(double *p, double v, int) { *p = v; }
};

template <>
struct Codec<float> {
    using compute = float;
    __device__ __forceinline__ static float load(const float *p, int) { return *p; }
    __device__ __forceinline__ static void store(float *p, float v, int) { *p = v; }
};

template <>
struct Codec<__half> {
    using compute = float;
    __device__ __forceinline__ static float load(const __half *p, int d) { return __half2float(*p) * float(weight(d)); }
    __device__ __forceinline__ static void store(__half *p, float v, int d) { *p = __float2half_rn(v * float(1.0 / weight(d))); }
};

template <>
struct Codec<__nv_bfloat16> {
    using compute = float;
    __device__ __forceinline__ static float load(const __nv_bfloat16 *p, int d)
    {
        return __bfloat162float(*p) * float(weight(d));
    }
    __device__ __forceinline__ static void store(__nv_bfloat16 *p, float v, int d)
    {
        *p = __float2bfloat16_rn(v * float(1.0 / weight(d)));
    }
};

} // namespace vfb
