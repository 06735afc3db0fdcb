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
    if (bad) {
        std::printf("%d mismatches\n", bad);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
