// Host driver for csrc/pool_tables.h. Mode "links": reads int32 n, int32 wide, float64 q27[27 n];
// writes uint64 link count, uint32 cut_first[n + ceil(n / 32)], then the link q bytes. Mode
// "compact": reads int64 count and that many mask bytes; writes one byte, 1 when the collision
// would queue fluid nodes.
#include <cstdio>
#include <cstring>
#include <vector>

#include "pool_tables.h"

int main(int argc, char **argv)
{
    if (argc != 4)
        return 2;
    std::FILE *in = std::fopen(argv[2], "rb");
    std::FILE *out = std::fopen(argv[3], "wb");
    if (!in || !out)
        return 3;
    if (std::strcmp(argv[1], "links") == 0) {
        int32_t hdr[2];
        if (std::fread(hdr, sizeof(int32_t), 2, in) != 2)
            return 4;
        const uint32_t n = (uint32_t)hdr[0];
        std::vector<double> q(27ull * n);
        if (std::fread(q.data(), sizeof(double), q.size(), in) != q.size())
            return 5;
        std::vector<uint32_t> cut_first;
        std::vector<unsigned char> link_q;
        const uint64_t links = vfb::noslip_link_tables(q.data(), n, hdr[1] != 0, &cut_first, &link_q);
        if (vfb::noslip_link_tables(q.data(), n, hdr[1] != 0, nullptr, nullptr) != links)
            return 6;
        std::fwrite(&links, sizeof(links), 1, out);
        std::fwrite(cut_first.data(), sizeof(uint32_t), cut_first.size(), out);
        std::fwrite(link_q.data(), 1, link_q.size(), out);
    } else {
        int64_t count = 0;
        if (std::fread(&count, sizeof(count), 1, in) != 1)
            return 4;
        std::vector<uint8_t> m((size_t)count);
        if (std::fread(m.data(), 1, m.size(), in) != m.size())
            return 5;
        const unsigned char flag = vfb::compact_collision(m) ? 1 : 0;
        std::fwrite(&flag, 1, 1, out);
    }
    std::fclose(in);
    std::fclose(out);
    return 0;
}
