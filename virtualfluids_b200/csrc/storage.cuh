// Storage formats of the population array.
//
// The reference stores "well-conditioned" populations f_i - w_i in `real` (float or double,
// src/basics/DataTypes.h:39-43; InitNavierStokesCompressible_Device.cu:175-202). Here the
// storage type is a runtime choice:
//   F64  : f - w as double, arithmetic in double (the reference's VF_DOUBLE_ACCURACY build)
//   F32  : f - w as float,  arithmetic in float  (the reference's default GPU build)
//   F16  : (f - w) / w as IEEE half,  arithmetic in float
//   BF16 : (f - w) / w as bfloat16,   arithmetic in float
//   E3M12: (f - w) / w as a 16-bit float of 1 sign, 3 exponent and 12 significand bits (below),
//          arithmetic in float
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

enum StorageKind : int { kStoreF64 = 0, kStoreF32 = 1, kStoreF16 = 2, kStoreBF16 = 3, kStoreE3M12 = 4 };

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

// ---------------------------------------------------------------------------------------------
// E3M12: a 16-bit float for the 1/w-scaled populations g = (f - w)/w, with 12 significand bits
// (IEEE half has 10) bought with a narrower exponent: 1 sign, 3 exponent, 12 significand bits,
// exponent bias 7, no infinities and no NaN.
//   e in 1..7: (-1)^s 2^(e-7) (1 + m/4096)   normal, magnitudes in [2^-6, 2)
//   e = 0    : (-1)^s 2^-6 (m/4096)           subnormal, steps of 2^-18
// g is O(drho + 3 c.u) for every direction (|g| < 1 for |u| up to ~0.15), so the format keeps the
// half-precision range a lattice Boltzmann state uses and spends the freed exponent bits on the
// significand: stored values near 0.1 carry 4x less rounding noise than in IEEE half. Magnitudes
// of 2 and more, infinities and NaN saturate to +-(2 - 2^-12) (a diverging state then shows as a
// mass drift, not as NaN).
//
// The layout is the top 16 bits of a float scaled by 2^-120 and shifted right by 11: the format's
// exponent field is the float's (values below 2^-6 become float subnormals, whose bits continue
// the format's subnormals linearly), so encoding is an integer add of 11 random bits (stochastic
// rounding, as for the other 16-bit forms), a shift and a saturation, and decoding the reverse
// shift and one multiplication.
// ---------------------------------------------------------------------------------------------
struct e3m12_t {
    uint16_t bits;
};

namespace e3m12 {
__host__ __device__ __forceinline__ uint32_t bits_of(float x)
{
#if defined(__CUDA_ARCH__)
    return __float_as_uint(x);
#else
    uint32_t b;
    __builtin_memcpy(&b, &x, sizeof b);
    return b;
#endif
}
__host__ __device__ __forceinline__ float float_of(uint32_t b)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(b);
#else
    float x;
    __builtin_memcpy(&x, &b, sizeof x);
    return x;
#endif
}
// t = g 2^-120 (already scaled), r in [0, 2048): saturate |t| at the largest value (a float min,
// which also turns NaN into it), round up with probability proportional to the dropped part (the
// clamped magnitude plus r never carries past the largest pattern), put the sign back
__host__ __device__ __forceinline__ uint16_t encode_scaled(float t, uint32_t r)
{
    const float a = fminf(fabsf(t), 0x1.fffp-120f);   // (2 - 2^-12) 2^-120, bits 0x03fff800
    return (uint16_t)(((bits_of(t) >> 16) & 0x8000u) | ((bits_of(a) + r) >> 11));
}
// the stored value times 2^-120 (exact): the sign-extended pattern shifted left by 11, with the
// extension's copies of the sign cleared from the exponent field
__host__ __device__ __forceinline__ float decode_scaled(uint16_t h)
{
    return float_of(((uint32_t)(int32_t)(int16_t)h << 11) & 0x83fff800u);
}
// g from its bits, and the bits of g (r = 0: truncation toward zero; r in [0, 2048))
__host__ __device__ __forceinline__ float decode(uint16_t h) { return decode_scaled(h) * 0x1p120f; }
__host__ __device__ __forceinline__ uint16_t encode(float g, uint32_t r) { return encode_scaled(g * 0x1p-120f, r); }
} // namespace e3m12

template <>
struct Codec<e3m12_t> {
    using compute = float;
    static constexpr bool kPairs = true;
    // (1/w) 2^-120 and w 2^120 for direction d: power-of-two scalings of the other 16-bit forms'
    // float constants, folded into their one multiplication
    __device__ __forceinline__ static float enc_scale(int d) { return float(1.0 / weight(d)) * 0x1p-120f; }
    __device__ __forceinline__ static float dec_scale(int d) { return float(weight(d)) * 0x1p120f; }
    __device__ __forceinline__ static void store_pair_at(e3m12_t *base, uint64_t off0, float v0, int d0, uint64_t off1,
                                                         float v1, int d1)
    {
        const float t0 = v0 * enc_scale(d0), t1 = v1 * enc_scale(d1);
        // 11 random bits each from the upper bits of the hash (they mix all of the value's bits)
        const uint32_t r = sr_bits(t0, off0) ^ (__float_as_uint(t1) * 0xC2B2AE35u);
        base[off0].bits = e3m12::encode_scaled(t0, r >> 21);
        base[off1].bits = e3m12::encode_scaled(t1, (r >> 10) & 0x7ffu);
    }
    // rounded on its own, as for the other 16-bit forms
    __device__ __forceinline__ static float load(const e3m12_t *p, int d)
    {
        return __fmul_rn(e3m12::decode_scaled(p->bits), dec_scale(d));
    }
    __device__ __forceinline__ static void store_at(e3m12_t *base, uint64_t off, float v, int d)
    {
        const float t = v * enc_scale(d);
        base[off].bits = e3m12::encode_scaled(t, sr_bits(t, off) >> 21);
    }
    __device__ __forceinline__ static void store_at_rt(e3m12_t *base, uint64_t off, float v, int d)
    {
        const float t = v * (inv_weight_rt(d) * 0x1p-120f);
        base[off].bits = e3m12::encode_scaled(t, sr_bits(t, off) >> 21);
    }
};

} // namespace vfb
