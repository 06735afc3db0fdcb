// Structured-box addressing shared by the host launchers and the kernels.
#pragma once

#include <cstdint>

namespace vfb {

// a structured box in the addressing of the boundary, drag and init kernels: node k = x + nx (y +
// ny z); on a periodic axis (bits 0-2 of `periodic` for x, y, z) the +1 neighbour wraps
struct NodeAddr {
    int nx, ny, nz, periodic;
};

// Division by a run-time constant d in [1, 2^16) of dividends n < 2^31 with one wide multiply and a
// shift (Granlund and Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994): with l = ceil(log2 d) and m = ceil(2^(31+l) / d) < 2^32, floor(n / d) = (n m) >> (31 + l),
// because n m / 2^(31+l) exceeds n / d by less than n / 2^(31+l) < 2^-l <= 1 / d.
struct FastDiv {
    uint32_t m;
    int shift;
};

inline FastDiv make_fast_div(uint32_t d)
{
    int l = 0;
    while ((1ull << l) < d)
        ++l;
    const uint64_t num = 1ull << (31 + l);
    FastDiv f;
    f.m = (uint32_t)((num + d - 1) / d);
    f.shift = 31 + l;
    return f;
}

#ifdef __CUDACC__
__host__ __device__
#endif
inline uint32_t fast_div(uint32_t n, FastDiv f)
{
    return (uint32_t)(((uint64_t)n * f.m) >> f.shift);
}

} // namespace vfb
