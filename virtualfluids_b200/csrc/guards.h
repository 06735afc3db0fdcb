// Host-side guard tables of a post-collision BC list on a structured box.
//
// In the esoteric-twist layout the BC write of node Y for a cut direction f lands in the slot that
// the node X = Y + c_f reads as its post-collision population inv(f). When X belongs to the same
// list (a link between two BC nodes that clips the geometry, as around spheres), the write races
// with X's read inside one launch. The guard table marks, per list node X, the directions e whose
// slot another list node overwrites (bit e of mask[X]); the BC launch first saves those values and
// the BC kernel reads them from there, so every node sees the collision's values whatever the
// thread order. first[X] numbers the saved values. Layout: table[0, n) = mask, table[n, 2n) = first.
#pragma once

#include <cstdint>
#include <vector>

#include "lattice.cuh"

namespace vfb {

template <class Q>
inline uint32_t bc_guard_tables(const int32_t *k, const Q *q27, uint32_t n, int nx, int ny, int nz, int periodic,
                                std::vector<uint32_t> &table)
{
    table.assign(2 * (size_t)n, 0u);
    if (!n)
        return 0;
    const uint64_t nodes = (uint64_t)nx * ny * nz;
    std::vector<int32_t> where(nodes, -1);
    for (uint32_t i = 0; i < n; ++i)
        where[(size_t)k[i]] = (int32_t)i;
    const int ext[3] = { nx, ny, nz };
    for (uint32_t j = 0; j < n; ++j) {
        const int64_t ky = k[j];
        const int c0[3] = { (int)(ky % nx), (int)((ky / nx) % ny), (int)(ky / ((int64_t)nx * ny)) };
        for (int f = 1; f < 27; ++f) {
            const Q q = q27[(uint64_t)f * n + j];
            if (!(q >= Q(0) && q <= Q(1)))
                continue;
            const int step[3] = { cx(f), cy(f), cz(f) };
            int c[3];
            bool inside = true;
            for (int a = 0; a < 3; ++a) {
                c[a] = c0[a] + step[a];
                if (c[a] < 0 || c[a] >= ext[a]) {
                    if (!((periodic >> a) & 1))
                        inside = false;
                    c[a] = (c[a] + ext[a]) % ext[a];
                }
            }
            if (!inside)
                continue;
            const int32_t i = where[(size_t)c[0] + (size_t)ext[0] * ((size_t)c[1] + (size_t)ext[1] * c[2])];
            if (i >= 0)
                table[(size_t)i] |= 1u << inv(f);
        }
    }
    uint32_t saved = 0;
    for (uint32_t i = 0; i < n; ++i) {
        table[(size_t)n + i] = saved;
        saved += (uint32_t)__builtin_popcount(table[(size_t)i]);
    }
    return saved;
}

} // namespace vfb
