// D3Q27 lattice description and esoteric-twist addressing, as compile-time functions so that
// every direction loop unrolls to constant indices.
//
// Direction numbering follows src/lbm/constants/D3Q27.h:42-72 (0 = rest, 1..6 faces, 7..18
// edges, 19..26 corners). The esoteric-twist (ET) in-place streaming of
// src/gpu/core/Utilities/KernelUtilities.h:66-378 stores every population of a node either at
// the node itself or at its +1 neighbour(s): direction d is read from and written to the node
// reached by stepping +1 along each axis where d has a negative component. On even steps
// direction d lives in array plane d; on odd steps in the plane of its inverse.
#pragma once
#include <cstdint>

namespace vfb {

constexpr int kQ = 27;

// lattice velocity components
__host__ __device__ constexpr int cx(int d)
{
    // 0 P00 M00 0P0 0M0 00P 00M PP0 MM0 PM0 MP0 P0P M0M P0M M0P 0PP 0MM 0PM 0MP PPP MPP PMP MMP PPM MPM PMM MMM
    return d == 1 || d == 7 || d == 9 || d == 11 || d == 13 || d == 19 || d == 21 || d == 23 || d == 25   ? 1
         : d == 2 || d == 8 || d == 10 || d == 12 || d == 14 || d == 20 || d == 22 || d == 24 || d == 26 ? -1
                                                                                                           : 0;
}
__host__ __device__ constexpr int cy(int d)
{
    return d == 3 || d == 7 || d == 10 || d == 15 || d == 17 || d == 19 || d == 20 || d == 23 || d == 24  ? 1
         : d == 4 || d == 8 || d == 9 || d == 16 || d == 18 || d == 21 || d == 22 || d == 25 || d == 26   ? -1
                                                                                                           : 0;
}
__host__ __device__ constexpr int cz(int d)
{
    return d == 5 || d == 11 || d == 14 || d == 15 || d == 18 || d == 19 || d == 20 || d == 21 || d == 22 ? 1
         : d == 6 || d == 12 || d == 13 || d == 16 || d == 17 || d == 23 || d == 24 || d == 25 || d == 26 ? -1
                                                                                                            : 0;
}
// inverse direction (D3Q27.h:85-110)
__host__ __device__ constexpr int inv(int d) { return d == 0 ? 0 : (d <= 18 ? ((d & 1) ? d + 1 : d - 1) : 45 - d); }
// number of non-zero components: 0 rest, 1 face, 2 edge, 3 corner
__host__ __device__ constexpr int order(int d) { return (cx(d) != 0) + (cy(d) != 0) + (cz(d) != 0); }
// lattice weight w_d
__host__ __device__ constexpr double weight(int d)
{
    return order(d) == 0 ? 8.0 / 27.0 : order(d) == 1 ? 2.0 / 27.0 : order(d) == 2 ? 1.0 / 54.0 : 1.0 / 216.0;
}
// lattice weight in arithmetic type T, written as the reference's constants c8o27, c2o27,
// c1o54, c1o216 (divisions carried out in T)
template <class T>
__host__ __device__ constexpr T weight_t(int d)
{
    return order(d) == 0 ? T(8) / T(27) : order(d) == 1 ? T(2) / T(27) : order(d) == 2 ? T(1) / T(54) : T(1) / T(216);
}
// moment-space position (ix, iy, iz in 0..2) flattened
__host__ __device__ constexpr int m3(int d) { return (cx(d) + 1) * 9 + (cy(d) + 1) * 3 + (cz(d) + 1); }
// ET shift class: bit0 = +1 in x, bit1 = +1 in y, bit2 = +1 in z
__host__ __device__ constexpr int shift_class(int d) { return (cx(d) < 0) | ((cy(d) < 0) << 1) | ((cz(d) < 0) << 2); }
// array plane holding direction d on an even / odd step
template <bool EVEN>
__host__ __device__ constexpr int plane(int d)
{
    return EVEN ? d : inv(d);
}

// Directions with a given component, as bit masks (bit d): the lattice for code whose direction
// is a run-time value, e.g. a thread working on one cut link of a list.
__host__ __device__ constexpr uint32_t component_mask(int axis, int sign)
{
    uint32_t m = 0;
    for (int d = 0; d < kQ; ++d)
        if ((axis == 0 ? cx(d) : axis == 1 ? cy(d) : cz(d)) == sign)
            m |= 1u << d;
    return m;
}
constexpr uint32_t kMaskXP = component_mask(0, 1), kMaskXM = component_mask(0, -1);
constexpr uint32_t kMaskYP = component_mask(1, 1), kMaskYM = component_mask(1, -1);
constexpr uint32_t kMaskZP = component_mask(2, 1), kMaskZM = component_mask(2, -1);

__host__ __device__ __forceinline__ int shift_class_rt(int d)
{
    return (int)(((kMaskXM >> d) & 1u) | (((kMaskYM >> d) & 1u) << 1) | (((kMaskZM >> d) & 1u) << 2));
}
__host__ __device__ __forceinline__ int order_rt(int d)
{
    return (int)(((kMaskXP | kMaskXM) >> d) & 1u) + (int)(((kMaskYP | kMaskYM) >> d) & 1u) +
           (int)(((kMaskZP | kMaskZM) >> d) & 1u);
}
// weight_t<T>(d) for a run-time d: the same four constants
template <class T>
__host__ __device__ __forceinline__ T weight_rt(int d)
{
    const int o = order_rt(d);
    return o == 0 ? weight_t<T>(0) : o == 1 ? weight_t<T>(1) : o == 2 ? weight_t<T>(7) : weight_t<T>(19);
}

// c_d . u for a run-time direction, with the operations of signed_sum: x, then y, then z; a
// leading negative component negated, later ones subtracted
template <class C>
__host__ __device__ __forceinline__ C cdot_link(int d, C ux, C uy, C uz)
{
    const bool xp = (kMaskXP >> d) & 1u, xm = (kMaskXM >> d) & 1u;
    const bool yp = (kMaskYP >> d) & 1u, ym = (kMaskYM >> d) & 1u;
    const bool zp = (kMaskZP >> d) & 1u, zm = (kMaskZM >> d) & 1u;
    C s = C(0);
    bool first = true;
    if (xp || xm) { s = xp ? ux : -ux; first = false; }
    if (yp || ym) { s = first ? (yp ? uy : -uy) : (yp ? s + uy : s - uy); first = false; }
    if (zp || zm) { s = first ? (zp ? uz : -uz) : (zp ? s + uz : s - uz); }
    return s;
}

// signed sum of a velocity along direction d, spelled as the reference kernels spell it
// (x, then y, then z; a leading negative component is negated, later ones subtracted)
template <int D, class T>
__device__ __forceinline__ T signed_sum(T ux, T uy, T uz)
{
    constexpr int c0 = cx(D), c1 = cy(D), c2 = cz(D);
    T s = T(0);
    bool first = true;
    if (c0 != 0) { s = c0 > 0 ? ux : -ux; first = false; }
    if (c1 != 0) { s = first ? (c1 > 0 ? uy : -uy) : (c1 > 0 ? s + uy : s - uy); first = false; }
    if (c2 != 0) { s = first ? (c2 > 0 ? uz : -uz) : (c2 > 0 ? s + uz : s - uz); }
    return s;
}

// GEO node types of src/gpu/core/Calculation/Calculation.h:39-45
constexpr uint32_t kGeoFluid = 19, kGeoSolid = 15, kGeoVoid = 16;

} // namespace vfb
