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
// The 16-bit formats round stochastically (below).
//
// The direction argument d of load / store_at is always a loop index of a fully unrolled
// 27-direction loop, so weight(d) folds to a constant; store_at_rt takes a run-time direction and
// picks the same constant by the direction's order.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "lattice.cuh"

namespace vfb {

enum StorageKind : int { kStoreF64 = 0, kStoreF32 = 1, kStoreF16 = 2, kStoreBF16 = 3 };

template <class S>
struct Codec;

// float(1 / w_d) for a run-time d: the constants the 16-bit stores scale by
__device__ __forceinline__ float inv_weight_rt(int d)
{
    const int o = order_rt(d);
    return o == 0 ? float(1.0 / weight(0)) : o == 1 ? float(1.0 / weight(1)) : o == 2 ? float(1.0 / weight(7))
                                                                                  : float(1.0 / weight(19));
}

template <>
struct Codec<double> {
    using compute = double;
    static constexpr bool kPairs = false;
    __device__ __forceinline__ static double load(const double *p, int) { return *p; }
    __device__ __forceinline__ static void store(double *p, double v, int) { *p = v; }
    __device__ __forceinline__ static void store_at(double *base, uint64_t off, double v, int) { base[off] = v; }
    __device__ __forceinline__ static void store_at_rt(double *base, uint64_t off, double v, int) { base[off] = v; }
};

template <>
struct Codec<float> {
    using compute = float;
    static constexpr bool kPairs = false;
    __device__ __forceinline__ static float load(const float *p, int) { return *p; }
    __device__ __forceinline__ static void store(float *p, float v, int) { *p = v; }
    __device__ __forceinline__ static void store_at(float *base, uint64_t off, float v, int) { base[off] = v; }
    __device__ __forceinline__ static void store_at_rt(float *base, uint64_t off, float v, int) { base[off] = v; }
};

// Stochastic rounding of the 16-bit stores. Rounding to nearest drops every change smaller than
// half a unit in the last place, so flows driven by small forces stall (a duct under a body force
// of 1e-6 per step ends percents away from FP64); rounding up or down with probability
// proportional to the distance keeps every store unbiased. The random bits are a hash of the
// value's bits and the slot's offset in its population array, so a run stays reproducible bit for
// bit (the same domain computes the same bits wherever its array lives), and they change whenever
// the value does. The conversion is sm_100a's cvt.rs (operand a lands in the upper half).
__device__ __forceinline__ uint32_t sr_bits(float v, uint64_t off)
{
    // two odd multipliers carry the value's (noisy) low mantissa bits and the slot offset into
    // every bit position; cheap, because the 16-bit forms are bound by arithmetic
    return (__float_as_uint(v) * 0x9E3779B1u) ^ ((uint32_t)off * 0x85EBCA77u) ^ (uint32_t)(off >> 32);
}

__device__ __forceinline__ __half half_sr(float v, uint32_t rbits)
{
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %1, %2;" : "=r"(d) : "f"(v), "r"(rbits));
    return __ushort_as_half((unsigned short)(d >> 16));
}

// two values in one conversion: a to the upper, b to the lower half of the result
__device__ __forceinline__ uint32_t half2_sr(float a, float b, uint32_t rbits)
{
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(rbits));
    return d;
}

__device__ __forceinline__ uint32_t bf162_sr(float a, float b, uint32_t rbits)
{
    uint32_t d;
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(rbits));
    return d;
}

__device__ __forceinline__ __nv_bfloat16 bf16_sr(float v, uint32_t rbits)
{
    uint32_t d;
    asm("cvt.rs.bf16x2.f32 %0, %1, %1, %2;" : "=r"(d) : "f"(v), "r"(rbits));
    return __ushort_as_bfloat16((unsigned short)(d >> 16));
}

template <>
struct Codec<__half> {
    using compute = float;
    static constexpr bool kPairs = true;
    __device__ __forceinline__ static void store_pair_at(__half *base, uint64_t off0, float v0, int d0, uint64_t off1,
                                                         float v1, int d1)
    {
        const float s0 = v0 * float(1.0 / weight(d0)), s1 = v1 * float(1.0 / weight(d1));
        const uint32_t h = half2_sr(s0, s1, sr_bits(s0, off0) ^ (__float_as_uint(s1) * 0xC2B2AE35u));
        base[off0] = __ushort_as_half((unsigned short)(h >> 16));
        base[off1] = __ushort_as_half((unsigned short)(h & 0xffffu));
    }
    // the decoding product is rounded on its own (never fused into a later addition), so a decoded
    // value is the same float wherever it is used or saved
    __device__ __forceinline__ static float load(const __half *p, int d) { return __fmul_rn(__half2float(*p), float(weight(d))); }
    __device__ __forceinline__ static void store_at(__half *base, uint64_t off, float v, int d)
    {
        const float s = v * float(1.0 / weight(d));
        base[off] = half_sr(s, sr_bits(s, off));
    }
    // store_at for a direction known only at run time (the same scale factors)
    __device__ __forceinline__ static void store_at_rt(__half *base, uint64_t off, float v, int d)
    {
        const float s = v * inv_weight_rt(d);
        base[off] = half_sr(s, sr_bits(s, off));
    }
};

template <>
struct Codec<__nv_bfloat16> {
    using compute = float;
    static constexpr bool kPairs = true;
    __device__ __forceinline__ static void store_pair_at(__nv_bfloat16 *base, uint64_t off0, float v0, int d0,
                                                         uint64_t off1, float v1, int d1)
    {
        const float s0 = v0 * float(1.0 / weight(d0)), s1 = v1 * float(1.0 / weight(d1));
        const uint32_t h = bf162_sr(s0, s1, sr_bits(s0, off0) ^ (__float_as_uint(s1) * 0xC2B2AE35u));
        base[off0] = __ushort_as_bfloat16((unsigned short)(h >> 16));
        base[off1] = __ushort_as_bfloat16((unsigned short)(h & 0xffffu));
    }
    __device__ __forceinline__ static float load(const __nv_bfloat16 *p, int d)
    {
        return __fmul_rn(__bfloat162float(*p), float(weight(d)));   // rounded on its own, as for FP16
    }
    __device__ __forceinline__ static void store_at(__nv_bfloat16 *base, uint64_t off, float v, int d)
    {
        const float s = v * float(1.0 / weight(d));
        base[off] = bf16_sr(s, sr_bits(s, off));
    }
    __device__ __forceinline__ static void store_at_rt(__nv_bfloat16 *base, uint64_t off, float v, int d)
    {
        const float s = v * inv_weight_rt(d);
        base[off] = bf16_sr(s, sr_bits(s, off));
    }
};

} // namespace vfb
