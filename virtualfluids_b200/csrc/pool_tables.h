// Host-side tables that a domain pool builds when a domain is added: the link form of its no-slip
// list and whether its collision queues fluid nodes. They are the contract between the host and
// the pool kernels (pool_noslip_kernel, k17_pool_kernel in kernels.cuh).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

namespace vfb {

// The no-slip list in the link form of pool_noslip_kernel, from q27 in the reference layout
// (q27[d n + i], double). A link is cut when q is in [0, 1] in the pool's real type (double when
// `wide`, else float), the test the kernels make.
//   cut_first: per node a mask of its cut directions (bit d), then for every 32 nodes the number
//              of links of the nodes before them;
//   q_out:     the q of the cut links in the pool's real type, per 32 nodes direction by direction
//              with the nodes ascending, the order in which a warp of the kernel lists them.
// Either output may be null; the link count is returned.
inline uint64_t noslip_link_tables(const double *q27, uint32_t n, bool wide, std::vector<uint32_t> *cut_first,
                                   std::vector<unsigned char> *q_out)
{
    auto active = [wide](double q) {
        if (wide)
            return q >= 0.0 && q <= 1.0;
        const float f = (float)q;
        return f >= 0.0f && f <= 1.0f;
    };
    auto put = [wide, q_out](double q) {
        unsigned char c[8];
        if (wide) {
            std::memcpy(c, &q, 8);
            q_out->insert(q_out->end(), c, c + 8);
        } else {
            const float f = (float)q;
            std::memcpy(c, &f, 4);
            q_out->insert(q_out->end(), c, c + 4);
        }
    };
    if (cut_first)
        cut_first->assign((size_t)n + (n + 31) / 32, 0u);
    if (q_out)
        q_out->clear();
    uint64_t links = 0;
    for (uint32_t c0 = 0; c0 < n; c0 += 32) {
        const uint32_t c1 = std::min(n, c0 + 32);
        if (cut_first)
            (*cut_first)[(size_t)n + c0 / 32] = (uint32_t)links;
        for (int d = 1; d < 27; ++d)
            for (uint32_t i = c0; i < c1; ++i) {
                const double q = q27[(size_t)d * n + i];
                if (!active(q))
                    continue;
                ++links;
                if (cut_first)
                    (*cut_first)[i] |= 1u << d;
                if (q_out)
                    put(q);
            }
    }
    return links;
}

// Whether the collision of a masked domain (m: one byte per node, nonzero = fluid) queues its
// fluid nodes per warp (k17_pool_kernel): when the lanes that 32-node segments mixing fluid and
// solid nodes would leave idle are at least 15 % of the fluid nodes. Porous blocks at porosity
// 0.75 leave 30-36 %, ducts whose solid nodes are whole wall rows 2 % (at most 14 % for the
// smallest); below the threshold the queue costs more than the idle lanes.
inline bool compact_collision(const std::vector<uint8_t> &m)
{
    uint64_t fluid = 0, idle = 0;
    for (size_t s = 0; s < m.size(); s += 32) {
        const size_t e = std::min(m.size(), s + 32);
        uint32_t f = 0;
        for (size_t k = s; k < e; ++k)
            f += m[k] != 0;
        fluid += f;
        if (f > 0 && f < 32)
            idle += 32 - f;
    }
    return fluid > 0 && idle * 100 >= fluid * 15;
}

} // namespace vfb
