// Interpolation between refinement levels: second-order moment interpolation of one cell of eight
// source nodes (src/lbm/interpolation/InterpolationCoefficients.h:74-438) and the evaluation of
// target populations from it (src/lbm/refinement/InterpolationCF.h:57, InterpolationFC.h:56).
//
// Formulation: the polynomial coefficients are written as sign-pattern sums over the cell's
// corners. Corner c = ix + 2 iy + 4 iz sits at ((ix, iy, iz) - 1/2) in cell units with signs
// s = 2 (ix, iy, iz) - 1. For every field q the trilinear coefficients are
//   q_100 = sum s_x q / 4,  q_110 = sum s_x s_y q / 2,  q_111 = sum s_x s_y s_z q, ...
// and the quadratic ones follow from the non-equilibrium second moments k_ab of the corners and
// the cross derivatives of the other velocity components (continuity), e.g.
//   a_020 = -b_110 / 2 + sum s_y k_xy / 8,   a_200 = (b_110 + c_101) / 4 + sum s_x (k_xxMyy + k_xxMzz) / 16;
// the constant term is the corner mean minus what the quadratic terms add at x^2 = 1/4. This is
// the reference's interpolation polynomial, summed in another order.
//
// On the device one cell is handled by 8 lanes of a warp, one corner each: every lane computes the
// moments of its own corner, then gathers all eight by shuffles and sums them corner by corner in
// the order c = 0..7, so every lane holds the same coefficients and evaluates its own target.
#pragma once
#include "k17.cuh"
#include "lattice.cuh"

namespace vfb {

// coefficients of one cell; u, v, w: 000 100 010 001 200 020 002 110 101 011
template <class T>
struct InterpCoef {
    T u[10], v[10], w[10];
    T d[7];      // drho: 000 100 010 001 110 101 011
    T q111[4];   // u v w drho
    T laplace;   // LaplaceRho
};

enum : int { I000 = 0, I100, I010, I001, I200, I020, I002, I110, I101, I011 };

// MomentsOnSourceNode::calculate (InterpolationCoefficients.h:74-146) of one node, f - w in
// direction order: {drho, ux, uy, uz, kxy, kyz, kxz, kxxMyy, kxxMzz} with
// k_ab = -3 omega (sum c_a c_b f / rho - u_a u_b), k_aaMbb = -3/2 omega (sum (c_a^2 - c_b^2) f / rho - (u_a^2 - u_b^2))
template <class T>
__device__ __forceinline__ void interp_node_moments(const T (&f)[27], T omega, T (&m)[9])
{
    const T drho = density_pyramid(f);
    const T inv = T(1) / (drho + T(1));
    const T vx = momentum_x(f) * inv, vy = momentum_y(f) * inv, vz = momentum_z(f) * inv;
    T sxy = T(0), syz = T(0), sxz = T(0), sxxyy = T(0), sxxzz = T(0);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        sxy += T(cx(d) * cy(d)) * f[d];
        syz += T(cy(d) * cz(d)) * f[d];
        sxz += T(cx(d) * cz(d)) * f[d];
        sxxyy += T(cx(d) * cx(d) - cy(d) * cy(d)) * f[d];
        sxxzz += T(cx(d) * cx(d) - cz(d) * cz(d)) * f[d];
    }
    m[0] = drho;
    m[1] = vx;
    m[2] = vy;
    m[3] = vz;
    m[4] = -T(3) * omega * (sxy * inv - vx * vy);
    m[5] = -T(3) * omega * (syz * inv - vy * vz);
    m[6] = -T(3) * omega * (sxz * inv - vx * vz);
    m[7] = -T(1.5) * omega * (sxxyy * inv - (vx * vx - vy * vy));
    m[8] = -T(1.5) * omega * (sxxzz * inv - (vx * vx - vz * vz));
}

// running sign-pattern sums of a cell, accumulated corner by corner
template <class T>
struct CellSums {
    T q[4][8];  // drho, u, v, w; patterns 1, x, y, z, xy, xz, yz, xyz
    T kxy[2];   // patterns x, y
    T kyz[2];   // y, z
    T kxz[2];   // x, z
    T kyy[3];   // kxxMyy: x, y, z
    T kzz[3];   // kxxMzz: x, y, z
};

template <class T>
__device__ __forceinline__ T signed_add(T acc, T v, int sign)
{
    return sign > 0 ? acc + v : acc - v;
}

template <class T>
__device__ __forceinline__ void zero_sums(CellSums<T> &S)
{
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int p = 0; p < 8; ++p)
            S.q[q][p] = T(0);
    S.kxy[0] = S.kxy[1] = S.kyz[0] = S.kyz[1] = S.kxz[0] = S.kxz[1] = T(0);
    S.kyy[0] = S.kyy[1] = S.kyy[2] = S.kzz[0] = S.kzz[1] = S.kzz[2] = T(0);
}

// add the moments m of corner c (a constant after unrolling) to the pattern sums
template <class T>
__device__ __forceinline__ void accumulate_corner(CellSums<T> &S, const T (&m)[9], int c)
{
    const int sx = (c & 1) ? 1 : -1, sy = (c & 2) ? 1 : -1, sz = (c & 4) ? 1 : -1;
    const int pat[8] = { 1, sx, sy, sz, sx * sy, sx * sz, sy * sz, sx * sy * sz };
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int p = 0; p < 8; ++p)
            S.q[q][p] = signed_add(S.q[q][p], m[q], pat[p]);
    S.kxy[0] = signed_add(S.kxy[0], m[4], sx);
    S.kxy[1] = signed_add(S.kxy[1], m[4], sy);
    S.kyz[0] = signed_add(S.kyz[0], m[5], sy);
    S.kyz[1] = signed_add(S.kyz[1], m[5], sz);
    S.kxz[0] = signed_add(S.kxz[0], m[6], sx);
    S.kxz[1] = signed_add(S.kxz[1], m[6], sz);
    S.kyy[0] = signed_add(S.kyy[0], m[7], sx);
    S.kyy[1] = signed_add(S.kyy[1], m[7], sy);
    S.kyy[2] = signed_add(S.kyy[2], m[7], sz);
    S.kzz[0] = signed_add(S.kzz[0], m[8], sx);
    S.kzz[1] = signed_add(S.kzz[1], m[8], sy);
    S.kzz[2] = signed_add(S.kzz[2], m[8], sz);
}

// sums of the cell whose eight corners are held by lanes group_base .. group_base + 7 of the warp
// (every lane of the warp calls this, with its own moments)
template <class T>
__device__ __forceinline__ void gather_cell_sums(CellSums<T> &S, const T (&mine)[9], int group_base)
{
    zero_sums(S);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        T m[9];
#pragma unroll
        for (int i = 0; i < 9; ++i)
            m[i] = __shfl_sync(0xffffffffu, mine[i], group_base + c);
        accumulate_corner(S, m, c);
    }
}

// MomentsOnSourceNodeSet::calculateCoefficients (InterpolationCoefficients.h:200-436)
template <class T>
__device__ __forceinline__ void cell_coefficients(const CellSums<T> &S, T xo, T yo, T zo, InterpCoef<T> &c)
{
    T mean[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        mean[q] = S.q[q][0] / T(8);
        const T g100 = S.q[q][1] / T(4), g010 = S.q[q][2] / T(4), g001 = S.q[q][3] / T(4);
        const T g110 = S.q[q][4] / T(2), g101 = S.q[q][5] / T(2), g011 = S.q[q][6] / T(2), g111 = S.q[q][7];
        if (q == 0) {
            c.d[0] = mean[0];
            c.d[1] = g100;
            c.d[2] = g010;
            c.d[3] = g001;
            c.d[4] = g110;
            c.d[5] = g101;
            c.d[6] = g011;
            c.q111[3] = g111;
        } else {
            T *a = q == 1 ? c.u : (q == 2 ? c.v : c.w);
            a[I100] = g100;
            a[I010] = g010;
            a[I001] = g001;
            a[I110] = g110;
            a[I101] = g101;
            a[I011] = g011;
            c.q111[q - 1] = g111;
        }
    }
    const T a110 = c.u[I110], a101 = c.u[I101], b110 = c.v[I110], b011 = c.v[I011], c101 = c.w[I101], c011 = c.w[I011];
    c.u[I200] = (b110 + c101) / T(4) + (S.kyy[0] + S.kzz[0]) / T(16);
    c.u[I020] = -b110 / T(2) + S.kxy[1] / T(8);
    c.u[I002] = -c101 / T(2) + S.kxz[1] / T(8);
    c.v[I200] = -a110 / T(2) + S.kxy[0] / T(8);
    c.v[I020] = (a110 + c011) / T(4) + (-T(2) * S.kyy[1] + S.kzz[1]) / T(16);
    c.v[I002] = -c011 / T(2) + S.kyz[1] / T(8);
    c.w[I200] = -a101 / T(2) + S.kxz[0] / T(8);
    c.w[I020] = -b011 / T(2) + S.kyz[0] / T(8);
    c.w[I002] = (a101 + b011) / T(4) + (S.kyy[2] - T(2) * S.kzz[2]) / T(16);
    c.u[I000] = mean[1] - (c.u[I200] + c.u[I020] + c.u[I002]) / T(4);
    c.v[I000] = mean[2] - (c.v[I200] + c.v[I020] + c.v[I002]) / T(4);
    c.w[I000] = mean[3] - (c.w[I200] + c.w[I020] + c.w[I002]) / T(4);
    c.laplace = (xo != T(0) || yo != T(0) || zo != T(0))
                    ? T(0)
                    : -T(3) * (c.u[I100] * c.u[I100] + c.v[I010] * c.v[I010] + c.w[I001] * c.w[I001])
                          - T(6) * (c.v[I100] * c.u[I010] + c.w[I100] * c.u[I001] + c.w[I010] * c.v[I001]);
    // move the expansion point by the offset (cells next to walls)
#pragma unroll
    for (int q = 1; q < 4; ++q) {
        T *a = q == 1 ? c.u : (q == 2 ? c.v : c.w);
        a[I000] = a[I000] + xo * a[I100] + yo * a[I010] + zo * a[I001] + xo * xo * a[I200] + yo * yo * a[I020]
                + zo * zo * a[I002] + xo * yo * a[I110] + xo * zo * a[I101] + yo * zo * a[I011];
        const T g100 = a[I100] + T(2) * xo * a[I200] + yo * a[I110] + zo * a[I101];
        const T g010 = a[I010] + T(2) * yo * a[I020] + xo * a[I110] + zo * a[I011];
        const T g001 = a[I001] + T(2) * zo * a[I002] + xo * a[I101] + yo * a[I011];
        a[I100] = g100;
        a[I010] = g010;
        a[I001] = g001;
    }
    T *d = c.d;
    d[0] = d[0] + xo * d[1] + yo * d[2] + zo * d[3] + xo * yo * d[4] + xo * zo * d[5] + yo * zo * d[6];
    const T d100 = d[1] + yo * d[4] + zo * d[5], d010 = d[2] + xo * d[4] + zo * d[6], d001 = d[3] + xo * d[5] + yo * d[6];
    d[1] = d100;
    d[2] = d010;
    d[3] = d001;
}

// interpolateCF at (x, y, z) (InterpolationCF.h:57-314) or interpolateFC at the cell centre (FC,
// InterpolationFC.h:56-269): density and velocity from the polynomials, second-order central
// moments from the strain rate scaled by -eps/omega (1 + drho), higher orders at equilibrium, then
// the backward chimera transform to f - w in direction order
template <class T, bool FC>
__device__ __forceinline__ void interp_point(const InterpCoef<T> &c, T omega, T eps, T x, T y, T z, T (&out)[27])
{
    using namespace k17detail;
    T press, u[3], g[3][3]; // g[i][j] = d u_i / d x_j
    if constexpr (FC) {
        press = c.d[0] - T(2) * c.laplace / T(8);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const T *q = i == 0 ? c.u : (i == 1 ? c.v : c.w);
            u[i] = q[I000];
            g[i][0] = q[I100];
            g[i][1] = q[I010];
            g[i][2] = q[I001];
        }
    } else {
        const T *d = c.d;
        press = d[0] + x * d[1] + y * d[2] + z * d[3] + x * y * d[4] + x * z * d[5] + y * z * d[6] + x * y * z * c.q111[3]
              + T(3) * x * x * c.laplace;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const T *q = i == 0 ? c.u : (i == 1 ? c.v : c.w);
            const T q111 = c.q111[i];
            u[i] = q[I000] + x * q[I100] + y * q[I010] + z * q[I001] + x * x * q[I200] + y * y * q[I020] + z * z * q[I002]
                 + x * y * q[I110] + x * z * q[I101] + y * z * q[I011] + x * y * z * q111;
            g[i][0] = q[I100] + T(2) * x * q[I200] + y * q[I110] + z * q[I101] + y * z * q111;
            g[i][1] = q[I010] + T(2) * y * q[I020] + x * q[I110] + z * q[I011] + x * z * q111;
            g[i][2] = q[I001] + T(2) * z * q[I002] + x * q[I101] + y * q[I011] + x * y * q111;
        }
    }
    const T s = eps / omega * (T(1) + press);
    T m[27];
#pragma unroll
    for (int i = 0; i < 27; ++i)
        m[i] = T(0);
#define VFB_M(a, b, cc) m[(a) * 9 + (b) * 3 + (cc)]
    const T mxxMyy = -T(2) / T(3) * (g[0][0] - g[1][1]) * s;
    const T mxxMzz = -T(2) / T(3) * (g[0][0] - g[2][2]) * s;
    VFB_M(0, 1, 1) = -T(1) / T(3) * (g[1][2] + g[2][1]) * s;
    VFB_M(1, 0, 1) = -T(1) / T(3) * (g[0][2] + g[2][0]) * s;
    VFB_M(1, 1, 0) = -T(1) / T(3) * (g[0][1] + g[1][0]) * s;
    VFB_M(0, 0, 0) = press;
    VFB_M(2, 0, 0) = (mxxMyy + mxxMzz + press) / T(3);
    VFB_M(0, 2, 0) = (-T(2) * mxxMyy + mxxMzz + press) / T(3);
    VFB_M(0, 0, 2) = (mxxMyy - T(2) * mxxMzz + press) / T(3);
    VFB_M(0, 2, 2) = press / T(9);
    VFB_M(2, 0, 2) = press / T(9);
    VFB_M(2, 2, 0) = press / T(9);
    VFB_M(2, 2, 2) = press / T(27);
    const T vx = u[0], vy = u[1], vz = u[2], vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
#pragma unroll
    for (int jb = 0; jb < 3; ++jb)
#pragma unroll
        for (int kc = 0; kc < 3; ++kc) {
            if (jb == 0 && kc == 0)
                bwd_k(VFB_M(0, 0, 0), VFB_M(1, 0, 0), VFB_M(2, 0, 0), vx, vx2, T(1), T(1));
            else if (jb == 2 && kc == 2)
                bwd_k(VFB_M(0, 2, 2), VFB_M(1, 2, 2), VFB_M(2, 2, 2), vx, vx2, T(9), T(1) / T(9));
            else if ((jb == 2 && kc == 0) || (jb == 0 && kc == 2))
                bwd_k(VFB_M(0, jb, kc), VFB_M(1, jb, kc), VFB_M(2, jb, kc), vx, vx2, T(3), T(1) / T(3));
            else
                bwd(VFB_M(0, jb, kc), VFB_M(1, jb, kc), VFB_M(2, jb, kc), vx, vx2);
        }
#pragma unroll
    for (int ia = 0; ia < 3; ++ia)
#pragma unroll
        for (int kc = 0; kc < 3; ++kc) {
            if (kc == 1)
                bwd(VFB_M(ia, 0, 1), VFB_M(ia, 1, 1), VFB_M(ia, 2, 1), vy, vy2);
            else
                bwd_k(VFB_M(ia, 0, kc), VFB_M(ia, 1, kc), VFB_M(ia, 2, kc), vy, vy2, kinv_y<T>(ia, kc), k_y<T>(ia, kc));
        }
#pragma unroll
    for (int ia = 0; ia < 3; ++ia)
#pragma unroll
        for (int jb = 0; jb < 3; ++jb)
            bwd_k(VFB_M(ia, jb, 0), VFB_M(ia, jb, 1), VFB_M(ia, jb, 2), vz, vz2, kinv_z<T>(ia, jb), k_z<T>(ia, jb));
#undef VFB_M
#pragma unroll
    for (int d = 0; d < 27; ++d)
        out[d] = m[m3(d)];
}

} // namespace vfb
