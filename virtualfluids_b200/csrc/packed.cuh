// Packed FP32x2 arithmetic for sm_100a: two independent nodes' values in one 64-bit register pair,
// every add, multiply and fused multiply-add issued as one instruction for both (the sm_100
// __fadd2_rn / __fmul2_rn / __ffma2_rn operations, each lane rounded as the scalar operation).
// The K17 collision is generic over its arithmetic type, so instantiated with f2 it collides two
// nodes per thread at about half the instruction count of the arithmetic. A product feeding an
// addition becomes one fused multiply-add (f2mul), as the compiler contracts the scalar forms.
#pragma once

#include <cuda_runtime.h>

#include "k17.cuh"

namespace vfb {

struct f2 {
    float2 v;
    f2() = default;
    __host__ __device__ __forceinline__ f2(float a) : v{ a, a } {}
    __host__ __device__ __forceinline__ f2(double a) : v{ (float)a, (float)a } {}
    __host__ __device__ __forceinline__ f2(int a) : v{ (float)a, (float)a } {}
    __host__ __device__ __forceinline__ f2(float a, float b) : v{ a, b } {}
};

#ifdef __CUDA_ARCH__
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
#else
__host__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __forceinline__ float2 mul2(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
__host__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y)); }
#endif
__host__ __device__ __forceinline__ float2 neg2(float2 a) { return mul2(a, make_float2(-1.0f, -1.0f)); }
// a - b = b * (-1) + a: the product is exact, so one rounding as in the scalar subtraction
__host__ __device__ __forceinline__ float2 sub2(float2 a, float2 b) { return fma2(b, make_float2(-1.0f, -1.0f), a); }

// A product not yet rounded: added to or subtracted from a value it becomes one fused multiply-add,
// as the compiler contracts a * b + c in the scalar forms; used as a value it is rounded.
struct f2mul {
    float2 a, b;
    __host__ __device__ __forceinline__ operator f2() const { f2 r; r.v = mul2(a, b); return r; }
};

__host__ __device__ __forceinline__ f2 wrap(float2 v) { f2 r; r.v = v; return r; }
__host__ __device__ __forceinline__ f2mul operator*(f2 a, f2 b) { return f2mul{ a.v, b.v }; }
__host__ __device__ __forceinline__ f2mul operator*(f2mul a, f2 b) { return f2mul{ f2(a).v, b.v }; }
__host__ __device__ __forceinline__ f2mul operator*(f2 a, f2mul b) { return f2mul{ a.v, f2(b).v }; }
__host__ __device__ __forceinline__ f2mul operator*(f2mul a, f2mul b) { return f2mul{ f2(a).v, f2(b).v }; }
__host__ __device__ __forceinline__ f2 operator+(f2 a, f2 b) { return wrap(add2(a.v, b.v)); }
__host__ __device__ __forceinline__ f2 operator+(f2mul p, f2 c) { return wrap(fma2(p.a, p.b, c.v)); }
__host__ __device__ __forceinline__ f2 operator+(f2 c, f2mul p) { return wrap(fma2(p.a, p.b, c.v)); }
__host__ __device__ __forceinline__ f2 operator+(f2mul p, f2mul q) { return wrap(fma2(p.a, p.b, f2(q).v)); }
__host__ __device__ __forceinline__ f2 operator-(f2 a, f2 b) { return wrap(sub2(a.v, b.v)); }
__host__ __device__ __forceinline__ f2 operator-(f2mul p, f2 c) { return wrap(fma2(p.a, p.b, neg2(c.v))); }
__host__ __device__ __forceinline__ f2 operator-(f2 c, f2mul p) { return wrap(fma2(neg2(p.a), p.b, c.v)); }
__host__ __device__ __forceinline__ f2 operator-(f2mul p, f2mul q) { return wrap(fma2(p.a, p.b, neg2(f2(q).v))); }
__host__ __device__ __forceinline__ f2 operator-(f2 a) { return wrap(neg2(a.v)); }
__host__ __device__ __forceinline__ f2mul operator-(f2mul p) { return f2mul{ neg2(p.a), p.b }; }
__host__ __device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) { return wrap(fma2(a.v, b.v, c.v)); }
// division only occurs between constants (folded) and in the reciprocals below
__host__ __device__ __forceinline__ f2 operator/(f2 a, f2 b) { return f2(a.v.x / b.v.x, a.v.y / b.v.y); }
__host__ __device__ __forceinline__ f2 &operator+=(f2 &a, f2 b) { a = a + b; return a; }
__host__ __device__ __forceinline__ f2 &operator+=(f2 &a, f2mul p) { a = p + a; return a; }
__host__ __device__ __forceinline__ f2 &operator-=(f2 &a, f2 b) { a = a - b; return a; }
__host__ __device__ __forceinline__ f2 &operator-=(f2 &a, f2mul p) { a = a - p; return a; }
__host__ __device__ __forceinline__ f2 &operator*=(f2 &a, f2 b) { a = f2(a * b); return a; }
__host__ __device__ __forceinline__ bool operator==(f2 a, f2 b) { return a.v.x == b.v.x && a.v.y == b.v.y; }
__host__ __device__ __forceinline__ f2 fabs(f2 a) { return f2(fabsf(a.v.x), fabsf(a.v.y)); }

namespace k17detail {
template <>
__host__ __device__ __forceinline__ f2 fast_rcp<f2>(f2 x)
{
    return f2(fast_rcp<float>(x.v.x), fast_rcp<float>(x.v.y));
}
template <>
__host__ __device__ __forceinline__ f2 rho_rcp<f2>(f2 x)
{
    return f2(rho_rcp<float>(x.v.x), rho_rcp<float>(x.v.y));
}
template <>
__host__ __device__ __forceinline__ void limiter_inverses<f2>(const f2 (&d)[7], f2 (&iv)[7])
{
#pragma unroll
    for (int i = 0; i < 7; ++i)
        iv[i] = fast_rcp<f2>(d[i]);
}
} // namespace k17detail

__host__ __device__ __forceinline__ K17FastConst<f2> broadcast(const K17FastConst<float> &c)
{
    K17FastConst<f2> r;
    r.omega = f2(c.omega);
    r.OxyyPxzz = f2(c.OxyyPxzz);
    r.OxyyMxzz = f2(c.OxyyMxzz);
    r.Oxyz = f2(c.Oxyz);
    r.kA = f2(c.kA);
    r.kB = f2(c.kB);
    r.qP = f2(c.qP);
    r.qM = f2(c.qM);
    r.qD = f2(c.qD);
    return r;
}

// two nodes' K17 collisions (the fast arithmetic) with packed operations; fa, fb in place
__device__ __forceinline__ void collide_pair(float (&fa)[27], float (&fb)[27], const K17Rates<float> &r, float fx,
                                             float fy, float fz, float (&ma)[4], float (&mb)[4])
{
    f2 f[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = f2(fa[d], fb[d]);
    f2 drho, vx, vy, vz;
    k17_collide_fast<f2>(f, broadcast(make_k17_fast_const(r)), f2(fx), f2(fy), f2(fz), drho, vx, vy, vz);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        fa[d] = f[d].v.x;
        fb[d] = f[d].v.y;
    }
    ma[0] = drho.v.x; ma[1] = vx.v.x; ma[2] = vy.v.x; ma[3] = vz.v.x;
    mb[0] = drho.v.y; mb[1] = vx.v.y; mb[2] = vy.v.y; mb[3] = vz.v.y;
}

} // namespace vfb
