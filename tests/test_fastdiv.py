"""The multiply-high division of the site decoding (lattice.cuh: make_fastdiv
and fdiv, restated here in integer arithmetic): floor(n / d) for every divisor
the geometry can produce and n over [0, 2^31), exhaustively near the multiples
of d and at random elsewhere."""
import numpy as np


def make_fastdiv(d):
    s = 0
    while (1 << s) < d:
        s += 1
    m = ((1 << (32 + s)) // d) + 1 - (1 << 32)
    assert 0 < m < (1 << 32)
    return m, s


def fdiv(n, m, s):
    hi = (n * m) >> 32
    assert hi + n < (1 << 32)
    return (hi + n) >> s


def test_fastdiv_exact():
    rng = np.random.default_rng(0)
    divisors = set(range(1, 400)) | {1 << k for k in range(31)} | {
        16 * 32 * 32 * 64, 24 * 48 * 48 * 96 // 2, 48 * 48 * 48 * 96, 12 * 24 * 24 * 48,
        8 * 8 * 8 * 8, 6 * 4 * 3 * 16, 2 ** 31 - 1, 2 ** 30 + 1, 3 ** 19, 1000003}
    for d in sorted(divisors):
        m, s = make_fastdiv(d)
        ns = set(int(v) for v in rng.integers(0, 2 ** 31, 2000))
        ns |= set(range(0, min(d * 3 + 5, 3000)))
        for k in rng.integers(0, (2 ** 31 - 1) // d + 1, 200):
            base = int(k) * d
            ns |= {base + o for o in (-1, 0, 1, d - 1) if 0 <= base + o < 2 ** 31}
        ns.add(2 ** 31 - 1)
        for n in ns:
            assert fdiv(n, m, s) == n // d, (d, n)
