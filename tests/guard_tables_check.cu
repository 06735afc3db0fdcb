// Host driver for csrc/guards.h: reads a BC list from a binary file, builds its guard tables and
// writes them out, so that a test can compare them with an independent restatement of the rule.
// Input (little endian): int32 n, nx, ny, nz, periodic; int32 k[n]; float64 q27[27 n].
// Output: uint32 n_saved, then uint32 table[2 n] (mask[n], first[n]).
#include <cstdio>
#include <vector>

#include "guards.h"

int main(int argc, char **argv)
{
    if (argc != 3)
        return 2;
    std::FILE *in = std::fopen(argv[1], "rb");
    if (!in)
        return 3;
    int32_t hdr[5];
    if (std::fread(hdr, sizeof(int32_t), 5, in) != 5)
        return 4;
    const uint32_t n = (uint32_t)hdr[0];
    std::vector<int32_t> k(n);
    std::vector<double> q(27ull * n);
    if (std::fread(k.data(), sizeof(int32_t), n, in) != n || std::fread(q.data(), sizeof(double), q.size(), in) != q.size())
        return 5;
    std::fclose(in);
    std::vector<uint32_t> table;
    const uint32_t saved = vfb::bc_guard_tables(k.data(), q.data(), n, hdr[1], hdr[2], hdr[3], hdr[4], table);
    std::FILE *out = std::fopen(argv[2], "wb");
    if (!out)
        return 6;
    std::fwrite(&saved, sizeof(uint32_t), 1, out);
    std::fwrite(table.data(), sizeof(uint32_t), table.size(), out);
    std::fclose(out);
    return 0;
}
