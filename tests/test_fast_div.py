"""The pool kernel's division by a domain's extent (csrc/addr.h make_fast_div / fast_div): with
l = ceil(log2 d) and m = ceil(2^(31+l) / d), floor(n / d) = (n m) >> (31 + l) for every extent
d < 2^16 and dividend n < 2^31 (node indices of a domain). Checked here on the formula for all d,
at the boundaries of the quotient steps and the top of the range; the GPU tests compare the pool
kernel that uses it with the box kernel bit for bit."""
import numpy as np


def _make(d):
    lg = 0
    while (1 << lg) < d:
        lg += 1
    return (((1 << (31 + lg)) + d - 1) // d), 31 + lg


def test_fast_division_is_exact_for_every_extent():
    rng = np.random.default_rng(7)
    top = (1 << 31) - 1
    for d in range(1, 1 << 16):
        m, s = _make(d)
        assert m < (1 << 32)
        q = top // d
        ns = [0, 1, d - 1, d, d + 1, top, top - 1, q * d, q * d - 1, (q // 2) * d - 1, (q // 2) * d]
        ns += [int(v) for v in rng.integers(0, 1 << 31, 8)]
        for n in ns:
            assert (n * m) >> s == n // d, (d, n)
