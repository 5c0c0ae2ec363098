"""The invariant-divisor division of csrc/common.cuh (FastDiv), restated: the
constructor's constants (l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
s = l - 1) and the quotient (t + ((n - t) >> 1)) >> s, t = mulhi(m, n), give
n // d exactly.  Checked for every n < 2^20 against each divisor the solver
and extraction use (every side and side - 1 of levels up to 4097), and for
random and extreme 32-bit numerators on all divisors up to 4097 and the 32-bit
extremes.  (On the GPU the extraction tests check the kernels that use it bit
for bit.)"""

import numpy as np


def constants(d):
    if d < 2:
        return 0, 0
    l = 0
    while (1 << l) < d:
        l += 1
    return ((1 << 32) * ((1 << l) - d)) // d + 1, l - 1


def quotient(n, d, m, s):
    if d == 1:
        return n
    t = (m * n) >> 32
    return (t + ((n - t) >> 1)) >> s


def test_constants_fit_32_bits():
    for d in list(range(1, 5000)) + [(1 << 31) - 1, 1 << 31, (1 << 32) - 1]:
        m, s = constants(d)
        assert 0 <= m < (1 << 32) and 0 <= s < 32


def test_exhaustive_small_numerators_on_level_sides():
    n = np.arange(1 << 20, dtype=np.uint64)
    sides = sorted({(1 << k) + 1 for k in range(1, 13)} | {(1 << k) for k in range(1, 13)} | {2, 3})
    for d in sides:
        m, s = constants(d)
        t = (np.uint64(m) * n) >> np.uint64(32)
        q = (t + ((n - t) >> np.uint64(1))) >> np.uint64(s)
        assert np.array_equal(q, n // np.uint64(d)), d


def test_random_and_extreme_numerators():
    rng = np.random.default_rng(0)
    divisors = list(range(1, 4098)) + [65535, 65536, 65537, (1 << 31) - 1, 1 << 31, (1 << 32) - 1]
    for d in divisors:
        m, s = constants(d)
        for n in [0, 1, d - 1, d, d + 1, (1 << 31), (1 << 32) - 1] + rng.integers(0, 1 << 32, 20).tolist():
            n = int(n) % (1 << 32)
            assert quotient(n, d, m, s) == n // d, (n, d)
