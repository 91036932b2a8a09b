"""The multiply-and-shift division the batch pack/unpack kernels use for
per-instance divisors (Granlund and Montgomery 1994), restated in Python
and checked against integer division: exhaustively for small operands and
on random and boundary 32-bit operands for the divisor range of images."""
import numpy as np


def make_fastdiv(d):
    l = 0
    while l < 32 and (1 << l) < d:
        l += 1
    m = ((1 << 32) * ((1 << l) - d)) // d + 1
    assert m < (1 << 32)
    return m, min(l, 1), max(l - 1, 0)


def fdiv(f, n):
    m, s1, s2 = f
    t = (m * n) >> 32
    return (t + ((n - t) >> s1)) >> s2


def test_fastdiv_small_exhaustive():
    for d in range(1, 300):
        f = make_fastdiv(d)
        for n in range(0, 5000):
            assert fdiv(f, n) == n // d, (d, n)


def test_fastdiv_random_and_boundaries():
    rng = np.random.default_rng(5)
    divisors = list(range(1, 70)) + [96, 127, 128, 129, 1000, 2047, 2048, 2049, 32767, 65536, 1 << 20,
                                      (1 << 31) - 1, 1 << 31]
    for d in divisors:
        f = make_fastdiv(d)
        ns = [0, 1, d - 1, d, d + 1, (1 << 32) - 1, (1 << 31), (1 << 31) - 1]
        ns += [int(v) for v in rng.integers(0, 1 << 32, size=2000, dtype=np.uint64)]
        for n in ns:
            if 0 <= n < (1 << 32):
                assert fdiv(f, n) == n // d, (d, n)
