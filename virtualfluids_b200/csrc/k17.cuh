// K17 cumulant collision of one D3Q27 node, register resident.
//
// Algorithm: src/lbm/collision/K17CompressibleNavierStokes.h:88-591 (TurbulenceModel::None),
// with the chimera transforms of src/lbm/ChimeraTransformation.h:58-121 and the pyramid
// macroscopic sums of src/lbm/MacroscopicQuantities.h:55-137. The floating-point expression
// trees are kept as in the reference so that a build without FMA contraction (-fmad=false)
// reproduces the reference's host arithmetic bit for bit; the default build contracts
// products into FMAs.
//
// Differences in *work*, not in results:
//  * the omega-only rates (five rational functions and 1/omega - 1/2) are computed once on the
//    host and passed in (K17Rates);
//  * with the relaxation rates O4 = O5 = O6 = 1 that the reference hard-codes, the pre-collision
//    4th, 5th and 6th order cumulants are multiplied by zero (4th) or relaxed to exactly zero
//    (5th, 6th), so they are not computed here; for finite inputs this changes no value.
#pragma once
#include "lattice.cuh"

namespace vfb {

template <class T>
struct K17Rates {
    T omega;
    T OxyyPxzz, OxyyMxzz, Oxyz; // 3rd order rates (K17...h:251-255)
    T factorA, factorB;         // 4th order diffusion parameters (K17...h:272-273)
    T neg_iwm;                  // -(1/omega - 1/2)
    T qP, qM, qD;               // quadric limiters (Parameter.cpp:69 default 0.01)
    // omega-only subexpressions of the collision, each rounded as the reference rounds it in place
    T mhw;                      // 1/2 * (-omega) (exact)
    T w32;                      // omega * 3/2
    T m3w;                      // -3 * omega
    T c3a;                      // 3 * (1 + 1/2 * (-omega))
    T omOxyz, omOP, omOM;       // 1 - Oxyz, 1 - OxyyPxzz, 1 - OxyyMxzz
};

// host computation of the omega-only rates, expression for expression as the reference
template <class T>
inline K17Rates<T> make_k17_rates(T omega, T qP, T qM, T qD)
{
    K17Rates<T> r;
    const T w = omega;
    r.omega = w;
    r.OxyyPxzz = T(8) * (T(-2) + w) * (T(1) + T(2) * w) / (T(-8) - T(14) * w + T(7) * w * w);
    r.OxyyMxzz = T(8) * (T(-2) + w) * (T(-7) + T(4) * w) / (T(56) - T(50) * w + T(9) * w * w);
    r.Oxyz = T(24) * (T(-2) + w) * (T(-2) - T(7) * w + T(3) * w * w) / (T(48) + T(152) * w - T(130) * w * w + T(29) * w * w * w);
    r.factorA = (T(4) + T(2) * w - T(3) * w * w) / (T(2) - T(7) * w + T(5) * w * w);
    r.factorB = (T(4) + T(28) * w - T(14) * w * w) / (T(6) - T(21) * w + T(15) * w * w);
    r.neg_iwm = -(T(1) / w - T(0.5));
    r.qP = qP;
    r.qM = qM;
    r.qD = qD;
    r.mhw = T(0.5) * (-w);
    r.w32 = w * (T(3) / T(2));
    r.m3w = -T(3) * w;
    r.c3a = T(3) * (T(1) + T(0.5) * (-w));
    r.omOxyz = T(1) - r.Oxyz;
    r.omOP = T(1) - r.OxyyPxzz;
    r.omOM = T(1) - r.OxyyMxzz;
    return r;
}

namespace k17detail {

template <class T>
__host__ __device__ __forceinline__ void fwd_k(T &a, T &b, T &c, T v, T v2, T kinv, T k)
{
    const T s2 = a + c;
    const T s1 = c - a;
    T s0 = s2 + b;
    a = s0;
    s0 *= kinv;
    s0 += T(1);
    b = (s1 * kinv - s0 * v) * k;
    c = ((s2 - T(2) * s1 * v) * kinv + v2 * s0) * k;
}
template <class T>
__host__ __device__ __forceinline__ void bwd_k(T &a, T &b, T &c, T v, T v2, T kinv, T k)
{
    const T h = T(0.5);
    const T r0 = (((c - b) * h + b * v) * kinv + (a * kinv + T(1)) * (v2 - v) * h) * k;
    const T r1 = (((a - c) - T(2) * b * v) * kinv + (a * kinv + T(1)) * (-v2)) * k;
    c = (((c + b) * h + b * v) * kinv + (a * kinv + T(1)) * (v2 + v) * h) * k;
    a = r0;
    b = r1;
}
template <class T>
__host__ __device__ __forceinline__ void fwd(T &a, T &b, T &c, T v, T v2)
{
    const T s1 = (a + c) + b;
    const T s2 = c - a;
    c = (c + a) + (v2 * s1 - T(2) * v * s2);
    b = s2 - v * s1;
    a = s1;
}
template <class T>
__host__ __device__ __forceinline__ void bwd(T &a, T &b, T &c, T v, T v2)
{
    const T h = T(0.5);
    const T ra = (c + a * (v2 - v)) * h + b * (v - h);
    const T rb = ((a - c) - a * v2) - T(2) * b * v;
    c = (c + a * (v2 + v)) * h + b * (v + h);
    b = rb;
    a = ra;
}

// The transforms of the exact collision. They round exactly as fwd_k / bwd_k / bwd above, with
// fewer operations:
//  * 2 s v is formed as s (2 v), 2 v once per axis: (2 s) v and s (2 v) are the same real number,
//    rounded once;
//  * X (v^2 -+ v) 1/2 is formed as X ((v^2 -+ v) 1/2), the halved factor once per axis: halving is
//    exact, so both round X (v^2 -+ v) / 2 once. This holds for every operand whose products stay
//    out of the subnormal range (|X (v^2 -+ v)| >= 2^-1021 or zero); a velocity component of a
//    state made of finite populations of magnitude above 1e-300 never comes near it;
//  * x h + y (h = 1/2) is one fma(x, h, y): the product is exact, so the fused operation rounds
//    once where the reference rounds the exact product and then the sum.
template <class T>
__host__ __device__ __forceinline__ void fwd_kx(T &a, T &b, T &c, T v, T v2, T twov, T kinv, T k)
{
    const T s2 = a + c;
    const T s1 = c - a;
    T s0 = s2 + b;
    a = s0;
    s0 *= kinv;
    s0 += T(1);
    b = (s1 * kinv - s0 * v) * k;
    c = ((s2 - s1 * twov) * kinv + v2 * s0) * k;
}
template <class T>
__host__ __device__ __forceinline__ void bwd_kx(T &a, T &b, T &c, T v, T v2, T twov, T v2mv_h, T v2pv_h, T kinv, T k)
{
    const T h = T(0.5);
    const T a1 = a * kinv + T(1);
    const T bv = b * v;
    const T r0 = (fma(c - b, h, bv) * kinv + a1 * v2mv_h) * k;
    const T r1 = (((a - c) - b * twov) * kinv + a1 * (-v2)) * k;
    c = (fma(c + b, h, bv) * kinv + a1 * v2pv_h) * k;
    a = r0;
    b = r1;
}
template <class T>
__host__ __device__ __forceinline__ void bwdx(T &a, T &b, T &c, T v, T v2, T twov)
{
    const T h = T(0.5);
    const T ra = fma(c + a * (v2 - v), h, b * (v - h));
    const T rb = ((a - c) - a * v2) - b * twov;
    c = fma(c + a * (v2 + v), h, b * (v + h));
    b = rb;
    a = ra;
}

// chimera constants, as the reference writes them (c36o1, c1o36, c9o4, c4o9, ...)
template <class T> __host__ __device__ __forceinline__ T kinv_z(int a, int b)
{
    return (a != 1 && b != 1) ? T(36) : (a == 1 && b == 1) ? T(9) / T(4) : T(9);
}
template <class T> __host__ __device__ __forceinline__ T k_z(int a, int b)
{
    return (a != 1 && b != 1) ? T(1) / T(36) : (a == 1 && b == 1) ? T(4) / T(9) : T(1) / T(9);
}
template <class T> __host__ __device__ __forceinline__ T kinv_y(int a, int c)
{
    return a != 1 ? (c == 0 ? T(6) : T(18)) : (c == 0 ? T(3) / T(2) : T(9) / T(2));
}
template <class T> __host__ __device__ __forceinline__ T k_y(int a, int c)
{
    return a != 1 ? (c == 0 ? T(1) / T(6) : T(1) / T(18)) : (c == 0 ? T(2) / T(3) : T(2) / T(9));
}

} // namespace k17detail

// pyramid density (MacroscopicQuantities.h:55), f in direction order
template <class T>
__host__ __device__ __forceinline__ T density_pyramid(const T *f)
{
    const T corners = ((f[19] + f[26]) + (f[24] + f[21])) + ((f[20] + f[25]) + (f[22] + f[23]));
    const T edges = (((f[18] + f[17]) + (f[16] + f[15])) + ((f[14] + f[13]) + (f[12] + f[11]))) + ((f[10] + f[9]) + (f[8] + f[7]));
    const T faces = ((f[2] + f[1]) + (f[4] + f[3])) + (f[6] + f[5]);
    return ((corners + edges) + f[0]) + faces;
}
template <class T>
__host__ __device__ __forceinline__ T momentum_x(const T *f)
{
    return ((((f[19] - f[26]) + (f[21] - f[24])) + ((f[25] - f[20]) + (f[23] - f[22])))
          + (((f[13] - f[14]) + (f[11] - f[12])) + ((f[9] - f[10]) + (f[7] - f[8]))))
          + (f[1] - f[2]);
}
template <class T>
__host__ __device__ __forceinline__ T momentum_y(const T *f)
{
    return ((((f[19] - f[26]) + (f[24] - f[21])) + ((f[20] - f[25]) + (f[23] - f[22])))
          + (((f[17] - f[18]) + (f[15] - f[16])) + ((f[10] - f[9]) + (f[7] - f[8]))))
          + (f[3] - f[4]);
}
template <class T>
__host__ __device__ __forceinline__ T momentum_z(const T *f)
{
    return ((((f[19] - f[26]) + (f[21] - f[24])) + ((f[20] - f[25]) + (f[22] - f[23])))
          + (((f[18] - f[17]) + (f[15] - f[16])) + ((f[14] - f[13]) + (f[11] - f[12]))))
          + (f[5] - f[6]);
}

// In place on f[27] (direction order). fx, fy, fz: half the acceleration, already scaled.
// Returns drho and the velocity including the half force (MacroscopicValues).
template <class T, bool EXACT>
__host__ __device__ __forceinline__ void k17_collide(T *f, const K17Rates<T> &r, T fx, T fy, T fz, T &drho_out, T &vx_out,
                                            T &vy_out, T &vz_out)
{
    using namespace k17detail;
    const T drho = density_pyramid(f);
    const T oneOverRho = T(1) / (drho + T(1));
    T vx = momentum_x(f) * oneOverRho;
    T vy = momentum_y(f) * oneOverRho;
    T vz = momentum_z(f) * oneOverRho;
    vx += fx;
    vy += fy;
    vz += fz;
    const T vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
    const T twovx = T(2) * vx, twovy = T(2) * vy, twovz = T(2) * vz;

    T m[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        m[m3(d)] = f[d];
#define M(a, b, c) m[(a) * 9 + (b) * 3 + (c)]

#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            fwd_kx(M(a, b, 0), M(a, b, 1), M(a, b, 2), vz, vz2, twovz, kinv_z<T>(a, b), k_z<T>(a, b));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; c += 1) {
            if (c == 1)
                fwd(M(a, 0, 1), M(a, 1, 1), M(a, 2, 1), vy, vy2);
            else
                fwd_kx(M(a, 0, c), M(a, 1, c), M(a, 2, c), vy, vy2, twovy, kinv_y<T>(a, c), k_y<T>(a, c));
        }
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (b == 0 && c == 0)
                fwd_kx(M(0, 0, 0), M(1, 0, 0), M(2, 0, 0), vx, vx2, twovx, T(1), T(1));
            else if (b == 2 && c == 2) // K17...h:222: K^-1 = 3, K = 1/9 on this line
                fwd_kx(M(0, 2, 2), M(1, 2, 2), M(2, 2, 2), vx, vx2, twovx, T(3), T(1) / T(9));
            else if ((b == 2 && c == 0) || (b == 0 && c == 2))
                fwd_kx(M(0, b, c), M(1, b, c), M(2, b, c), vx, vx2, twovx, T(3), T(1) / T(3));
            else
                fwd(M(0, b, c), M(1, b, c), M(2, b, c), vx, vx2);
        }

    const T c13 = T(1) / T(3), c19 = T(1) / T(9), c23 = T(2) / T(3), c127 = T(1) / T(27), h = T(0.5);
    const T omega = r.omega;

    // second and third order linear combinations (K17...h:323-335)
    T mxxPyyPzz = M(2, 0, 0) + M(0, 2, 0) + M(0, 0, 2);
    T mxxMyy = M(2, 0, 0) - M(0, 2, 0);
    T mxxMzz = M(2, 0, 0) - M(0, 0, 2);
    T mxxyPyzz = M(2, 1, 0) + M(0, 1, 2);
    T mxxyMyzz = M(2, 1, 0) - M(0, 1, 2);
    T mxxzPyyz = M(2, 0, 1) + M(0, 2, 1);
    T mxxzMyyz = M(2, 0, 1) - M(0, 2, 1);
    T mxyyPxzz = M(1, 2, 0) + M(1, 0, 2);
    T mxyyMxzz = M(1, 2, 0) - M(1, 0, 2);

    // velocity gradients times rho (K17...h:347-352), OxxPyyPzz = 1
    // (the omega-only factors -3 omega, 1/2 (-omega), omega 3/2 come rounded from the host)
    const T Dxy = r.m3w * M(1, 1, 0);
    const T Dxz = r.m3w * M(1, 0, 1);
    const T Dyz = r.m3w * M(0, 1, 1);
    const T dxux = fma(M(0, 0, 0) - mxxPyyPzz, h, r.mhw * (mxxMyy + mxxMzz));
    const T dyuy = dxux + r.w32 * mxxMyy;
    const T dzuz = dxux + r.w32 * mxxMzz;

    // second order relaxation with correction (K17...h:375-387)
    mxxPyyPzz += T(1) * (M(0, 0, 0) - mxxPyyPzz) - T(3) * (T(1) - h * T(1)) * (vx2 * dxux + vy2 * dyuy + vz2 * dzuz);
    mxxMyy += omega * (-mxxMyy) - r.c3a * (vx2 * dxux - vy2 * dyuy);
    mxxMzz += omega * (-mxxMzz) - r.c3a * (vx2 * dxux - vz2 * dzuz);
    M(0, 1, 1) += omega * (-M(0, 1, 1));
    M(1, 0, 1) += omega * (-M(1, 0, 1));
    M(1, 1, 0) += omega * (-M(1, 1, 0));

    // third order with the quartic limiter (K17...h:397-410)
    T wadj;
    wadj = r.Oxyz + r.omOxyz * fabs(M(1, 1, 1)) / (fabs(M(1, 1, 1)) + r.qD);
    M(1, 1, 1) += wadj * (-M(1, 1, 1));
    wadj = r.OxyyPxzz + r.omOP * fabs(mxxyPyzz) / (fabs(mxxyPyzz) + r.qP);
    mxxyPyzz += wadj * (-mxxyPyzz);
    wadj = r.OxyyMxzz + r.omOM * fabs(mxxyMyzz) / (fabs(mxxyMyzz) + r.qM);
    mxxyMyzz += wadj * (-mxxyMyzz);
    wadj = r.OxyyPxzz + r.omOP * fabs(mxxzPyyz) / (fabs(mxxzPyyz) + r.qP);
    mxxzPyyz += wadj * (-mxxzPyyz);
    wadj = r.OxyyMxzz + r.omOM * fabs(mxxzMyyz) / (fabs(mxxzMyyz) + r.qM);
    mxxzMyyz += wadj * (-mxxzMyyz);
    wadj = r.OxyyPxzz + r.omOP * fabs(mxyyPxzz) / (fabs(mxyyPxzz) + r.qP);
    mxyyPxzz += wadj * (-mxyyPxzz);
    wadj = r.OxyyMxzz + r.omOM * fabs(mxyyMxzz) / (fabs(mxyyMxzz) + r.qM);
    mxyyMxzz += wadj * (-mxyyMxzz);

    // back from the linear combinations (K17...h:424-433)
    M(2, 0, 0) = c13 * (mxxMyy + mxxMzz + mxxPyyPzz);
    M(0, 2, 0) = c13 * (fma(T(-2), mxxMyy, mxxMzz) + mxxPyyPzz);
    M(0, 0, 2) = c13 * (fma(T(-2), mxxMzz, mxxMyy) + mxxPyyPzz);
    M(2, 1, 0) = (mxxyMyzz + mxxyPyzz) * h;
    M(0, 1, 2) = (-mxxyMyzz + mxxyPyzz) * h;
    M(2, 0, 1) = (mxxzMyyz + mxxzPyyz) * h;
    M(0, 2, 1) = (-mxxzMyyz + mxxzPyyz) * h;
    M(1, 2, 0) = (mxyyMxzz + mxyyPxzz) * h;
    M(1, 0, 2) = (-mxyyMxzz + mxyyPxzz) * h;

    // post-collision 4th order cumulants: modified equilibrium (K17...h:443-448)
    const T cm022 = r.neg_iwm * (dyuy + dzuz) * c23 * r.factorA;
    const T cm202 = r.neg_iwm * (dxux + dzuz) * c23 * r.factorA;
    const T cm220 = r.neg_iwm * (dyuy + dxux) * c23 * r.factorA;
    const T cm112 = r.neg_iwm * Dxy * c13 * r.factorB;
    const T cm121 = r.neg_iwm * Dxz * c13 * r.factorB;
    const T cm211 = r.neg_iwm * Dyz * c13 * r.factorB;
    // 5th and 6th order post-collision cumulants are zero
    const T z = T(0);

    // central moments from post-collision cumulants (K17...h:469-505)
    M(2, 1, 1) = cm211 + c13 * ((T(3) * M(2, 0, 0) + T(1)) * M(0, 1, 1) + T(6) * M(1, 1, 0) * M(1, 0, 1)) * oneOverRho;
    M(1, 2, 1) = cm121 + c13 * ((T(3) * M(0, 2, 0) + T(1)) * M(1, 0, 1) + T(6) * M(1, 1, 0) * M(0, 1, 1)) * oneOverRho;
    M(1, 1, 2) = cm112 + c13 * ((T(3) * M(0, 0, 2) + T(1)) * M(1, 1, 0) + T(6) * M(1, 0, 1) * M(0, 1, 1)) * oneOverRho;
    // products with a power of two are exact: (2 m) m = 2 (m m), and a sum with it is one fma
    const T sq110 = M(1, 1, 0) * M(1, 1, 0), sq101 = M(1, 0, 1) * M(1, 0, 1), sq011 = M(0, 1, 1) * M(0, 1, 1);
    M(2, 2, 0) = cm220 + ((fma(T(2), sq110, M(2, 0, 0) * M(0, 2, 0)) * T(9) + T(3) * (M(2, 0, 0) + M(0, 2, 0))) * oneOverRho - (drho * oneOverRho)) * c19;
    M(2, 0, 2) = cm202 + ((fma(T(2), sq101, M(2, 0, 0) * M(0, 0, 2)) * T(9) + T(3) * (M(2, 0, 0) + M(0, 0, 2))) * oneOverRho - (drho * oneOverRho)) * c19;
    M(0, 2, 2) = cm022 + ((fma(T(2), sq011, M(0, 0, 2) * M(0, 2, 0)) * T(9) + T(3) * (M(0, 0, 2) + M(0, 2, 0))) * oneOverRho - (drho * oneOverRho)) * c19;

    const T t122 = c13 * (T(3) * fma(T(2), M(1, 0, 1) * M(0, 2, 1) + M(1, 1, 0) * M(0, 1, 2), fma(T(4), M(0, 1, 1) * M(1, 1, 1), M(0, 0, 2) * M(1, 2, 0) + M(0, 2, 0) * M(1, 0, 2))) + (M(1, 2, 0) + M(1, 0, 2))) * oneOverRho;
    const T t212 = c13 * (T(3) * fma(T(2), M(0, 1, 1) * M(2, 0, 1) + M(1, 1, 0) * M(1, 0, 2), fma(T(4), M(1, 0, 1) * M(1, 1, 1), M(0, 0, 2) * M(2, 1, 0) + M(2, 0, 0) * M(0, 1, 2))) + (M(2, 1, 0) + M(0, 1, 2))) * oneOverRho;
    const T t221 = c13 * (T(3) * fma(T(2), M(1, 0, 1) * M(1, 2, 0) + M(0, 1, 1) * M(2, 1, 0), fma(T(4), M(1, 1, 0) * M(1, 1, 1), M(2, 0, 0) * M(0, 2, 1) + M(0, 2, 0) * M(2, 0, 1))) + (M(0, 2, 1) + M(2, 0, 1))) * oneOverRho;
    M(1, 2, 2) = EXACT ? z + t122 : t122;
    M(2, 1, 2) = EXACT ? z + t212 : t212;
    M(2, 2, 1) = EXACT ? z + t221 : t221;

    const T b222 = fma(T(-2), M(1, 2, 0) * M(1, 0, 2) + M(2, 1, 0) * M(0, 1, 2) + M(2, 0, 1) * M(0, 2, 1),
                       fma(T(-4), M(0, 1, 1) * M(2, 1, 1) + M(1, 0, 1) * M(1, 2, 1) + M(1, 1, 0) * M(1, 1, 2),
                           fma(T(-4), M(1, 1, 1) * M(1, 1, 1), -(M(2, 0, 0) * M(0, 2, 2) + M(0, 2, 0) * M(2, 0, 2) + M(0, 0, 2) * M(2, 2, 0))))) * oneOverRho
                 + fma(T(16), M(1, 1, 0) * M(1, 0, 1) * M(0, 1, 1),
                       fma(T(4), sq101 * M(0, 2, 0) + sq011 * M(2, 0, 0) + sq110 * M(0, 0, 2),
                           T(2) * (M(2, 0, 0) * M(0, 2, 0) * M(0, 0, 2)))) * oneOverRho * oneOverRho
                 - c13 * (M(0, 2, 2) + M(2, 0, 2) + M(2, 2, 0)) * oneOverRho - c19 * (M(2, 0, 0) + M(0, 2, 0) + M(0, 0, 2)) * oneOverRho
                 + (fma(T(2), sq101 + sq011 + sq110, M(0, 0, 2) * M(0, 2, 0) + M(0, 0, 2) * M(2, 0, 0) + M(0, 2, 0) * M(2, 0, 0))
                    + c13 * (M(0, 0, 2) + M(0, 2, 0) + M(2, 0, 0))) * oneOverRho * oneOverRho * c23
                 + c127 * ((drho * drho - drho) * oneOverRho * oneOverRho);
    M(2, 2, 2) = EXACT ? z - b222 : -b222;

    // first moments change sign (K17...h:512-514)
    M(1, 0, 0) = -M(1, 0, 0);
    M(0, 1, 0) = -M(0, 1, 0);
    M(0, 0, 1) = -M(0, 0, 1);

    const T x2mvh = (vx2 - vx) * h, x2pvh = (vx2 + vx) * h, y2mvh = (vy2 - vy) * h, y2pvh = (vy2 + vy) * h;
    const T z2mvh = (vz2 - vz) * h, z2pvh = (vz2 + vz) * h;

#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (b == 0 && c == 0)
                bwd_kx(M(0, 0, 0), M(1, 0, 0), M(2, 0, 0), vx, vx2, twovx, x2mvh, x2pvh, T(1), T(1));
            else if (b == 2 && c == 2)
                bwd_kx(M(0, 2, 2), M(1, 2, 2), M(2, 2, 2), vx, vx2, twovx, x2mvh, x2pvh, T(9), T(1) / T(9));
            else if ((b == 2 && c == 0) || (b == 0 && c == 2))
                bwd_kx(M(0, b, c), M(1, b, c), M(2, b, c), vx, vx2, twovx, x2mvh, x2pvh, T(3), T(1) / T(3));
            else
                bwdx(M(0, b, c), M(1, b, c), M(2, b, c), vx, vx2, twovx);
        }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (c == 1)
                bwdx(M(a, 0, 1), M(a, 1, 1), M(a, 2, 1), vy, vy2, twovy);
            else
                bwd_kx(M(a, 0, c), M(a, 1, c), M(a, 2, c), vy, vy2, twovy, y2mvh, y2pvh, kinv_y<T>(a, c), k_y<T>(a, c));
        }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            bwd_kx(M(a, b, 0), M(a, b, 1), M(a, b, 2), vz, vz2, twovz, z2mvh, z2pvh, kinv_z<T>(a, b), k_z<T>(a, b));
#undef M

#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = m[m3(d)];
    drho_out = drho;
    vx_out = vx;
    vy_out = vy;
    vz_out = vz;
}

// ---------------------------------------------------------------------------------------------
// The same collision, rearranged for fewer floating-point instructions (the FMA variant).
//
// Mathematically identical to k17_collide, rounded differently:
//  * the well-conditioned chimera transforms are used in their K-offset form,
//    b' = m1 - v (m0 + K), c' = m2 - 2 v m1 + v^2 (m0 + K) (forward) and the matching backward
//    form -- the reference's forwardChimeraWithK / backwardChimeraWithK
//    (src/lbm/ChimeraTransformation.h:124-150) -- since (x K^-1 + 1) K = x + K;
//  * density and momenta share the 13 pair sums and differences f_d +- f_inv(d);
//  * the eight reciprocals of a node (1/rho and the seven quartic-limiter denominators) come from
//    one division (product of the denominators, then back-substitution);
//  * omega-only products are folded into single constants.
// ---------------------------------------------------------------------------------------------
template <class T>
struct K17FastConst {
    T omega;
    T OxyyPxzz, OxyyMxzz, Oxyz;
    T kA;       // -(1/omega - 1/2) * 2/3 * factorA
    T kB;       // -(1/omega - 1/2) * 1/3 * factorB
    T qP, qM, qD;
};

template <class T>
__host__ __device__ inline K17FastConst<T> make_k17_fast_const(const K17Rates<T> &r)
{
    K17FastConst<T> c;
    c.omega = r.omega;
    c.OxyyPxzz = r.OxyyPxzz;
    c.OxyyMxzz = r.OxyyMxzz;
    c.Oxyz = r.Oxyz;
    c.kA = r.neg_iwm * (T(2) / T(3)) * r.factorA;
    c.kB = r.neg_iwm * (T(1) / T(3)) * r.factorB;
    c.qP = r.qP;
    c.qM = r.qM;
    c.qD = r.qD;
    return c;
}

namespace k17detail {
// forward transform along one line with offset K (K = 0: the plain central-moment transform);
// K is a constant of the unrolled loops, so the K = 0 lines carry no offset addition
template <class T>
__host__ __device__ __forceinline__ void fwdK(T &a, T &b, T &c, T v, T v2, T twov, T K)
{
    const T apc = a + c;
    const T m1 = c - a;
    const T m0 = apc + b;
    const T w = K == T(0) ? m0 : m0 + K;
    a = m0;
    b = fma(-v, w, m1);
    c = fma(v2, w, fma(-twov, m1, apc));
}
// backward transform with offset K: a' = ((c - b) + w (v^2 - v))/2 + b v,
// b' = (a - c) - 2 b v - w v^2, c' = ((c + b) + w (v^2 + v))/2 + b v, w = a + K
template <class T>
__host__ __device__ __forceinline__ void bwdK(T &a, T &b, T &c, T v, T v2mv, T v2pv, T twov, T v2, T K)
{
    (void)twov;
    const T w = K == T(0) ? a : a + K;
    const T bv = b * v;
    const T r0 = fma(T(0.5), fma(w, v2mv, c - b), bv);
    const T r1 = fma(-v2, w, fma(T(-2), bv, a - c));
    c = fma(T(0.5), fma(w, v2pv, c + b), bv);
    a = r0;
    b = r1;
}
// 1/x: IEEE division in double; the fast approximate division in float
template <class T>
__host__ __device__ __forceinline__ T fast_rcp(T x)
{
    return T(1) / x;
}
template <>
__host__ __device__ __forceinline__ float fast_rcp<float>(float x)
{
#ifdef __CUDA_ARCH__
    return __fdividef(1.0f, x);
#else
    return 1.0f / x;
#endif
}

// 1/rho for the velocity: correctly rounded in both precisions. u = j (1/rho) feeds the moment
// transforms, and the backward transform puts back j' = rho u + (the negated first central moment
// rho (j/rho - u)), so any error in u changes the node's momentum by twice that error times rho.
// A reciprocal that errs to one side (an approximate one) therefore makes the momentum drift step
// after step; a correctly rounded one errs both ways equally often. In float the rounded
// reciprocal flushes subnormals (rcp.rn.ftz): rho is near 1, so the bits are those of the IEEE
// reciprocal, and the form without flushing carries a slow path whose call raised the 16-bit
// pool kernel from 128 to 172 registers.
template <class T>
__host__ __device__ __forceinline__ T rho_rcp(T x)
{
    return T(1) / x;
}
template <>
__host__ __device__ __forceinline__ float rho_rcp<float>(float x)
{
#ifdef __CUDA_ARCH__
    float y;
    asm("rcp.rn.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
#else
    return 1.0f / x;
#endif
}

// the seven limiter reciprocals: in double one division and back-substitution through the
// running products (the denominators are >= the limiters, so the product stays far above the
// double range limit); in float seven fast divisions (a float product could underflow)
template <class T>
__host__ __device__ __forceinline__ void limiter_inverses(const T (&d)[7], T (&iv)[7])
{
    const T p1 = d[0] * d[1], p2 = p1 * d[2], p3 = p2 * d[3], p4 = p3 * d[4], p5 = p4 * d[5], p6 = p5 * d[6];
    T rr = T(1) / p6;
    iv[6] = rr * p5;
    rr *= d[6];
    iv[5] = rr * p4;
    rr *= d[5];
    iv[4] = rr * p3;
    rr *= d[4];
    iv[3] = rr * p2;
    rr *= d[3];
    iv[2] = rr * p1;
    rr *= d[2];
    iv[1] = rr * d[0];
    iv[0] = rr * d[1];
}
template <>
__host__ __device__ __forceinline__ void limiter_inverses<float>(const float (&d)[7], float (&iv)[7])
{
#pragma unroll
    for (int i = 0; i < 7; ++i)
        iv[i] = fast_rcp<float>(d[i]);
}
} // namespace k17detail

template <class T>
__host__ __device__ __forceinline__ void k17_collide_fast(T *f, const K17FastConst<T> &r, T fx, T fy, T fz, T &drho_out,
                                                 T &vx_out, T &vy_out, T &vz_out)
{
    using namespace k17detail;
    // pair sums / differences, canonical direction first
    const T s1 = f[1] + f[2], t1 = f[1] - f[2];       // P00
    const T s3 = f[3] + f[4], t3 = f[3] - f[4];       // 0P0
    const T s5 = f[5] + f[6], t5 = f[5] - f[6];       // 00P
    const T s7 = f[7] + f[8], t7 = f[7] - f[8];       // PP0
    const T s9 = f[9] + f[10], t9 = f[9] - f[10];     // PM0
    const T s11 = f[11] + f[12], t11 = f[11] - f[12]; // P0P
    const T s13 = f[13] + f[14], t13 = f[13] - f[14]; // P0M
    const T s15 = f[15] + f[16], t15 = f[15] - f[16]; // 0PP
    const T s17 = f[17] + f[18], t17 = f[17] - f[18]; // 0PM
    const T s19 = f[19] + f[26], t19 = f[19] - f[26]; // PPP
    const T s21 = f[21] + f[24], t21 = f[21] - f[24]; // PMP
    const T s23 = f[23] + f[22], t23 = f[23] - f[22]; // PPM
    const T s25 = f[25] + f[20], t25 = f[25] - f[20]; // PMM
    const T drho = ((((s19 + s21) + (s23 + s25)) + ((s7 + s9) + (s11 + s13))) + ((s15 + s17) + (s1 + s3))) + (s5 + f[0]);
    const T jx = (((t19 + t21) + (t23 + t25)) + ((t7 + t9) + (t11 + t13))) + t1;
    const T jy = (((t19 - t21) + (t23 - t25)) + ((t7 - t9) + (t15 + t17))) + t3;
    const T jz = (((t19 + t21) - (t23 + t25)) + ((t11 - t13) + (t15 - t17))) + t5;

    const T oneOverRho = rho_rcp(drho + T(1));
    const T vx = fma(jx, oneOverRho, fx), vy = fma(jy, oneOverRho, fy), vz = fma(jz, oneOverRho, fz);
    const T vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
    const T twovx = T(2) * vx, twovy = T(2) * vy, twovz = T(2) * vz;

    T m[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        m[m3(d)] = f[d];
#define M(a, b, c) m[(a) * 9 + (b) * 3 + (c)]
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            fwdK(M(a, b, 0), M(a, b, 1), M(a, b, 2), vz, vz2, twovz, k_z<T>(a, b));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            fwdK(M(a, 0, c), M(a, 1, c), M(a, 2, c), vy, vy2, twovy, c == 1 ? T(0) : k_y<T>(a, c));
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T K = (b == 0 && c == 0) ? T(1) : ((b == 2 || c == 2) && b != 1 && c != 1) ? T(1) / T(3) : T(0);
            fwdK(M(0, b, c), M(1, b, c), M(2, b, c), vx, vx2, twovx, K);
        }
    // K17...h:222 transforms the (2,2) x-line with K^-1 = 3 but K = 1/9: the offset is 1/K^-1 = 1/3
    // and the two higher moments come out scaled by K^-1 K = 1/3
    M(1, 2, 2) *= T(1) / T(3);
    M(2, 2, 2) *= T(1) / T(3);

    const T c13 = T(1) / T(3), c19 = T(1) / T(9), c23 = T(2) / T(3), c127 = T(1) / T(27), h = T(0.5);
    const T omega = r.omega;

    T mxxPyyPzz = M(2, 0, 0) + M(0, 2, 0) + M(0, 0, 2);
    T mxxMyy = M(2, 0, 0) - M(0, 2, 0);
    T mxxMzz = M(2, 0, 0) - M(0, 0, 2);
    T mxxyPyzz = M(2, 1, 0) + M(0, 1, 2);
    T mxxyMyzz = M(2, 1, 0) - M(0, 1, 2);
    T mxxzPyyz = M(2, 0, 1) + M(0, 2, 1);
    T mxxzMyyz = M(2, 0, 1) - M(0, 2, 1);
    T mxyyPxzz = M(1, 2, 0) + M(1, 0, 2);
    T mxyyMxzz = M(1, 2, 0) - M(1, 0, 2);

    const T m3omega = -T(3) * omega;
    const T Dxy = m3omega * M(1, 1, 0);
    const T Dxz = m3omega * M(1, 0, 1);
    const T Dyz = m3omega * M(0, 1, 1);
    const T dxux = fma(-h * omega, mxxMyy + mxxMzz, h * (M(0, 0, 0) - mxxPyyPzz));
    const T o32 = omega * T(1.5);
    const T dyuy = fma(o32, mxxMyy, dxux);
    const T dzuz = fma(o32, mxxMzz, dxux);

    const T c3h = T(3) * (T(1) - h * omega);
    mxxPyyPzz += (M(0, 0, 0) - mxxPyyPzz) - T(1.5) * (vx2 * dxux + vy2 * dyuy + vz2 * dzuz);
    mxxMyy = fma(-omega, mxxMyy, mxxMyy) - c3h * (vx2 * dxux - vy2 * dyuy);
    mxxMzz = fma(-omega, mxxMzz, mxxMzz) - c3h * (vx2 * dxux - vz2 * dzuz);
    const T omo = T(1) - omega;
    M(0, 1, 1) *= omo;
    M(1, 0, 1) *= omo;
    M(1, 1, 0) *= omo;

    // quartic limiters: seven reciprocals from one division
    const T a0 = fabs(M(1, 1, 1)), a1 = fabs(mxxyPyzz), a2 = fabs(mxxyMyzz), a3 = fabs(mxxzPyyz);
    const T a4 = fabs(mxxzMyyz), a5 = fabs(mxyyPxzz), a6 = fabs(mxyyMxzz);
    const T dd[7] = { a0 + r.qD, a1 + r.qP, a2 + r.qM, a3 + r.qP, a4 + r.qM, a5 + r.qP, a6 + r.qM };
    T iv[7];
    limiter_inverses<T>(dd, iv);
    const T i0 = iv[0], i1 = iv[1], i2 = iv[2], i3 = iv[3], i4 = iv[4], i5 = iv[5], i6 = iv[6];
    // m += (O + (1-O) |m|/(|m|+q)) (-m)
    M(1, 1, 1) -= fma(T(1) - r.Oxyz, a0 * i0, r.Oxyz) * M(1, 1, 1);
    mxxyPyzz -= fma(T(1) - r.OxyyPxzz, a1 * i1, r.OxyyPxzz) * mxxyPyzz;
    mxxyMyzz -= fma(T(1) - r.OxyyMxzz, a2 * i2, r.OxyyMxzz) * mxxyMyzz;
    mxxzPyyz -= fma(T(1) - r.OxyyPxzz, a3 * i3, r.OxyyPxzz) * mxxzPyyz;
    mxxzMyyz -= fma(T(1) - r.OxyyMxzz, a4 * i4, r.OxyyMxzz) * mxxzMyyz;
    mxyyPxzz -= fma(T(1) - r.OxyyPxzz, a5 * i5, r.OxyyPxzz) * mxyyPxzz;
    mxyyMxzz -= fma(T(1) - r.OxyyMxzz, a6 * i6, r.OxyyMxzz) * mxyyMxzz;

    M(2, 0, 0) = c13 * (mxxMyy + mxxMzz + mxxPyyPzz);
    M(0, 2, 0) = c13 * (-T(2) * mxxMyy + mxxMzz + mxxPyyPzz);
    M(0, 0, 2) = c13 * (mxxMyy - T(2) * mxxMzz + mxxPyyPzz);
    M(2, 1, 0) = (mxxyMyzz + mxxyPyzz) * h;
    M(0, 1, 2) = (mxxyPyzz - mxxyMyzz) * h;
    M(2, 0, 1) = (mxxzMyyz + mxxzPyyz) * h;
    M(0, 2, 1) = (mxxzPyyz - mxxzMyyz) * h;
    M(1, 2, 0) = (mxyyMxzz + mxyyPxzz) * h;
    M(1, 0, 2) = (mxyyPxzz - mxyyMxzz) * h;

    const T cm022 = r.kA * (dyuy + dzuz);
    const T cm202 = r.kA * (dxux + dzuz);
    const T cm220 = r.kA * (dyuy + dxux);
    const T cm112 = r.kB * Dxy;
    const T cm121 = r.kB * Dxz;
    const T cm211 = r.kB * Dyz;

    const T c13r = c13 * oneOverRho;
    const T drr = drho * oneOverRho;
    M(2, 1, 1) = fma(c13r, (T(3) * M(2, 0, 0) + T(1)) * M(0, 1, 1) + T(6) * M(1, 1, 0) * M(1, 0, 1), cm211);
    M(1, 2, 1) = fma(c13r, (T(3) * M(0, 2, 0) + T(1)) * M(1, 0, 1) + T(6) * M(1, 1, 0) * M(0, 1, 1), cm121);
    M(1, 1, 2) = fma(c13r, (T(3) * M(0, 0, 2) + T(1)) * M(1, 1, 0) + T(6) * M(1, 0, 1) * M(0, 1, 1), cm112);
    M(2, 2, 0) = cm220 + ((T(9) * (M(2, 0, 0) * M(0, 2, 0) + T(2) * M(1, 1, 0) * M(1, 1, 0)) + T(3) * (M(2, 0, 0) + M(0, 2, 0))) * oneOverRho - drr) * c19;
    M(2, 0, 2) = cm202 + ((T(9) * (M(2, 0, 0) * M(0, 0, 2) + T(2) * M(1, 0, 1) * M(1, 0, 1)) + T(3) * (M(2, 0, 0) + M(0, 0, 2))) * oneOverRho - drr) * c19;
    M(0, 2, 2) = cm022 + ((T(9) * (M(0, 0, 2) * M(0, 2, 0) + T(2) * M(0, 1, 1) * M(0, 1, 1)) + T(3) * (M(0, 0, 2) + M(0, 2, 0))) * oneOverRho - drr) * c19;
    M(1, 2, 2) = c13r * (T(3) * (M(0, 0, 2) * M(1, 2, 0) + M(0, 2, 0) * M(1, 0, 2) + T(4) * M(0, 1, 1) * M(1, 1, 1) + T(2) * (M(1, 0, 1) * M(0, 2, 1) + M(1, 1, 0) * M(0, 1, 2))) + (M(1, 2, 0) + M(1, 0, 2)));
    M(2, 1, 2) = c13r * (T(3) * (M(0, 0, 2) * M(2, 1, 0) + M(2, 0, 0) * M(0, 1, 2) + T(4) * M(1, 0, 1) * M(1, 1, 1) + T(2) * (M(0, 1, 1) * M(2, 0, 1) + M(1, 1, 0) * M(1, 0, 2))) + (M(2, 1, 0) + M(0, 1, 2)));
    M(2, 2, 1) = c13r * (T(3) * (M(2, 0, 0) * M(0, 2, 1) + M(0, 2, 0) * M(2, 0, 1) + T(4) * M(1, 1, 0) * M(1, 1, 1) + T(2) * (M(1, 0, 1) * M(1, 2, 0) + M(0, 1, 1) * M(2, 1, 0))) + (M(0, 2, 1) + M(2, 0, 1)));
    const T r2 = oneOverRho * oneOverRho;
    M(2, 2, 2) = -((-T(4) * M(1, 1, 1) * M(1, 1, 1) - (M(2, 0, 0) * M(0, 2, 2) + M(0, 2, 0) * M(2, 0, 2) + M(0, 0, 2) * M(2, 2, 0))
                    - T(4) * (M(0, 1, 1) * M(2, 1, 1) + M(1, 0, 1) * M(1, 2, 1) + M(1, 1, 0) * M(1, 1, 2))
                    - T(2) * (M(1, 2, 0) * M(1, 0, 2) + M(2, 1, 0) * M(0, 1, 2) + M(2, 0, 1) * M(0, 2, 1))) * oneOverRho
                   + (T(4) * (M(1, 0, 1) * M(1, 0, 1) * M(0, 2, 0) + M(0, 1, 1) * M(0, 1, 1) * M(2, 0, 0) + M(1, 1, 0) * M(1, 1, 0) * M(0, 0, 2))
                      + T(2) * (M(2, 0, 0) * M(0, 2, 0) * M(0, 0, 2)) + T(16) * M(1, 1, 0) * M(1, 0, 1) * M(0, 1, 1)) * r2
                   - (c13 * (M(0, 2, 2) + M(2, 0, 2) + M(2, 2, 0)) + c19 * (M(2, 0, 0) + M(0, 2, 0) + M(0, 0, 2))) * oneOverRho
                   + (T(2) * (M(1, 0, 1) * M(1, 0, 1) + M(0, 1, 1) * M(0, 1, 1) + M(1, 1, 0) * M(1, 1, 0))
                      + (M(0, 0, 2) * M(0, 2, 0) + M(0, 0, 2) * M(2, 0, 0) + M(0, 2, 0) * M(2, 0, 0)) + c13 * (M(0, 0, 2) + M(0, 2, 0) + M(2, 0, 0))) * r2 * c23
                   + c127 * ((drho * drho - drho) * r2));

    M(1, 0, 0) = -M(1, 0, 0);
    M(0, 1, 0) = -M(0, 1, 0);
    M(0, 0, 1) = -M(0, 0, 1);

    const T x2mv = vx2 - vx, x2pv = vx2 + vx, y2mv = vy2 - vy, y2pv = vy2 + vy, z2mv = vz2 - vz, z2pv = vz2 + vz;
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T K = (b == 0 && c == 0) ? T(1) : (b == 2 && c == 2) ? T(1) / T(9)
                      : ((b == 2 && c == 0) || (b == 0 && c == 2)) ? T(1) / T(3) : T(0);
            bwdK(M(0, b, c), M(1, b, c), M(2, b, c), vx, x2mv, x2pv, twovx, vx2, K);
        }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            bwdK(M(a, 0, c), M(a, 1, c), M(a, 2, c), vy, y2mv, y2pv, twovy, vy2, c == 1 ? T(0) : k_y<T>(a, c));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            bwdK(M(a, b, 0), M(a, b, 1), M(a, b, 2), vz, z2mv, z2pv, twovz, vz2, k_z<T>(a, b));
#undef M

#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = m[m3(d)];
    drho_out = drho;
    vx_out = vx;
    vy_out = vy;
    vz_out = vz;
}

} // namespace vfb

namespace vfb {
// the collision of the chosen arithmetic variant
template <class T, bool EXACT>
__host__ __device__ __forceinline__ void collide(T *f, const K17Rates<T> &r, T fx, T fy, T fz, T &drho, T &vx, T &vy, T &vz)
{
    if constexpr (EXACT)
        k17_collide<T, true>(f, r, fx, fy, fz, drho, vx, vy, vz);
    else
        k17_collide_fast<T>(f, make_k17_fast_const(r), fx, fy, fz, drho, vx, vy, vz);
}
} // namespace vfb
