// The E3M12 storage codec (csrc/storage.cuh, namespace vfb::e3m12) on the host, compiled by nvcc:
//  * every bit pattern decodes to a value that encodes back to the same pattern, with no added bits
//    and with the most added bits (representable values are never moved);
//  * positive patterns decode in strictly increasing order, and a sign flip only flips the sign;
//  * stochastic rounding is unbiased: for any value, the mean of its encodings over all 2048 values
//    of the added bits decodes to the value itself (exactly, summed in double), across the normal
//    and subnormal ranges;
//  * magnitudes of 2 and more, infinities and NaN saturate to +-(2 - 2^-12).
// Prints "ok" and returns 0 when every check passes.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <random>

#include "storage.cuh"

using namespace vfb;

int main()
{
    int bad = 0;
    for (uint32_t h = 0; h < 65536; ++h) {
        const float g = e3m12::decode((uint16_t)h);
        if (e3m12::encode(g, 0) != h || e3m12::encode(g, 2047) != h) {
            if (bad < 10)
                std::printf("round trip %04x\n", h);
            ++bad;
        }
        if (h < 0x7fff && !(e3m12::decode((uint16_t)(h + 1)) > g)) {
            std::printf("not increasing at %04x\n", h);
            ++bad;
        }
        if (h < 0x8000 && e3m12::decode((uint16_t)(h | 0x8000)) != -g && h != 0) {
            std::printf("sign %04x\n", h);
            ++bad;
        }
    }
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (int i = 0; i < 20000; ++i) {
        // magnitudes from 2^-30 to 2: subnormals, every binade, and values next to 2
        const float g = (float)((u(rng) < 0.5 ? -1.0 : 1.0) * std::ldexp(1.0 + u(rng), -(int)(rng() % 31)) * 0.999);
        const double exact = (double)(g * 0x1p-120f) * 0x1p120;   // the value the codec rounds
        double sum = 0.0;
        for (uint32_t r = 0; r < 2048; ++r)
            sum += (double)e3m12::decode(e3m12::encode(g, r));
        if (sum != 2048.0 * exact) {
            if (bad < 20)
                std::printf("biased rounding of %a: mean %a\n", g, sum / 2048.0);
            ++bad;
        }
    }
    const float big[] = {2.0f, 3.5f, 1e30f, INFINITY};
    for (float v : big) {
        if (e3m12::encode(v, 0) != 0x7fff || e3m12::encode(-v, 1000) != 0xffff) {
            std::printf("saturation %g\n", v);
            ++bad;
        }
    }
    const uint16_t nan_bits = e3m12::encode(NAN, 5);
    if ((nan_bits & 0x7fff) != 0x7fff) {
        std::printf("NaN %04x\n", nan_bits);
        ++bad;
    }
    if (e3m12::decode(0x7fff) != 2.0f - 0x1p-12f || e3m12::decode(1) != 0x1p-18f || e3m12::decode(0x1000) != 0x1p-6f) {
        std::printf("range constants\n");
        ++bad;
    }
    if (bad) {
        std::printf("%d failures\n", bad);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
