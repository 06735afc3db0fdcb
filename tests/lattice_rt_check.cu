// Host-side check of the run-time direction helpers of csrc/lattice.cuh against the compile-time
// lattice functions, for every direction: shift class, order, weight in double and float (bit
// equal), and c_d . u with the operations of the unrolled kernels (bit equal, signed zeros
// included, on values chosen so that the sums round). Prints "ok" and exits 0 when all agree.
#include <cstdio>
#include <cstring>

#include "lattice.cuh"

using namespace vfb;

// c_d . u as the unrolled kernels spell it for a direction known at compile time
template <class C>
C cdot_reference(int d, C ux, C uy, C uz)
{
    C s = C(0);
    bool first = true;
    if (cx(d) != 0) { s = cx(d) > 0 ? ux : -ux; first = false; }
    if (cy(d) != 0) { s = first ? (cy(d) > 0 ? uy : -uy) : (cy(d) > 0 ? s + uy : s - uy); first = false; }
    if (cz(d) != 0) { s = first ? (cz(d) > 0 ? uz : -uz) : (cz(d) > 0 ? s + uz : s - uz); }
    return s;
}

template <class C>
bool same_bits(C a, C b)
{
    return std::memcmp(&a, &b, sizeof(C)) == 0;
}

template <class C>
int check_cdot()
{
    const C vals[] = { C(0), C(-0.0), C(0.1), C(-0.3), C(1e-7), C(0.0123456789), C(-2.5e-3), C(1) / C(3) };
    int bad = 0;
    for (int d = 0; d < kQ; ++d)
        for (C ux : vals)
            for (C uy : vals)
                for (C uz : vals)
                    if (!same_bits(cdot_link<C>(d, ux, uy, uz), cdot_reference<C>(d, ux, uy, uz))) {
                        if (bad < 5)
                            std::printf("cdot d=%d differs\n", d);
                        ++bad;
                    }
    return bad;
}

int main()
{
    int bad = 0;
    for (int d = 0; d < kQ; ++d) {
        if (shift_class_rt(d) != shift_class(d)) {
            std::printf("shift_class d=%d: %d vs %d\n", d, shift_class_rt(d), shift_class(d));
            ++bad;
        }
        if (order_rt(d) != order(d)) {
            std::printf("order d=%d\n", d);
            ++bad;
        }
        if (!same_bits(weight_rt<double>(d), weight_t<double>(d)) || !same_bits(weight_rt<float>(d), weight_t<float>(d))) {
            std::printf("weight d=%d\n", d);
            ++bad;
        }
        const int sx = (kMaskXP >> d & 1u) - (kMaskXM >> d & 1u), sy = (kMaskYP >> d & 1u) - (kMaskYM >> d & 1u),
                  sz = (kMaskZP >> d & 1u) - (kMaskZM >> d & 1u);
        if (sx != cx(d) || sy != cy(d) || sz != cz(d)) {
            std::printf("component masks d=%d\n", d);
            ++bad;
        }
    }
    bad += check_cdot<double>();
    bad += check_cdot<float>();
    // the esoteric-twist plane map, as the reference's KernelUtilitiesTests.cpp states it for
    // getDistributionReferences27: on even steps direction d is array plane d; on odd steps the
    // pairs below swap (M00 <-> P00, ..., MMM <-> PPP) and the rest plane stays
    {
        // D3Q27 numbering: 0 000, 1 P00, 2 M00, 3 0P0, 4 0M0, 5 00P, 6 00M, 7 PP0, 8 MM0, 9 PM0,
        // 10 MP0, 11 P0P, 12 M0M, 13 P0M, 14 M0P, 15 0PP, 16 0MM, 17 0PM, 18 0MP, 19 PPP, 20 MPP,
        // 21 PMP, 22 MMP, 23 PPM, 24 MPM, 25 PMM, 26 MMM
        const int odd_pairs[13][2] = {{2, 1}, {4, 3}, {6, 5}, {8, 7}, {10, 9}, {12, 11}, {14, 13},
                                      {16, 15}, {18, 17}, {26, 19}, {23, 22}, {24, 21}, {25, 20}};
        for (int d = 0; d < kQ; ++d)
            if (plane<true>(d) != d) {
                std::printf("even plane d=%d\n", d);
                ++bad;
            }
        if (plane<false>(0) != 0) {
            std::printf("odd rest plane\n");
            ++bad;
        }
        for (const auto &pr : odd_pairs)
            if (plane<false>(pr[0]) != pr[1] || plane<false>(pr[1]) != pr[0]) {
                std::printf("odd plane pair %d %d\n", pr[0], pr[1]);
                ++bad;
            }
        // the direction components of the numbering above
        const char *names[27] = {"000", "P00", "M00", "0P0", "0M0", "00P", "00M", "PP0", "MM0", "PM0", "MP0", "P0P", "M0M",
                                 "P0M", "M0P", "0PP", "0MM", "0PM", "0MP", "PPP", "MPP", "PMP", "MMP", "PPM", "MPM", "PMM", "MMM"};
        for (int d = 0; d < kQ; ++d) {
            const int c[3] = {cx(d), cy(d), cz(d)};
            for (int a = 0; a < 3; ++a) {
                const int want = names[d][a] == 'P' ? 1 : names[d][a] == 'M' ? -1 : 0;
                if (c[a] != want) {
                    std::printf("component %d of d=%d\n", a, d);
                    ++bad;
                }
            }
        }
    }
    if (bad) {
        std::printf("%d mismatches\n", bad);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
