"""The FP64 kernels form the source's quotients a/b (a grid-spacing divisor b
with a host-tabulated reciprocal rb = RN(1/b)) by Markstein's correction:
q = RN(a rb), r = RN(a - b q) (one fused multiply-add, exact), RN(q + r rb)
(a second one).  This restates the three roundings exactly with rationals and
checks the claim the kernels rely on, RN(q + r rb) == RN(a/b), on random
operands of the solver's ranges (velocity differences and metric sums over
spacings from 1e-5 to 1e2) and on edge cases of the significands (divisors
and dividends with all-ones or power-of-two significands, and near-ties)."""
import math
import struct
from fractions import Fraction

import numpy as np


def rn(x):
    """round a rational to the nearest double (ties to even)"""
    return float(x)


def markstein(a, b):
    rb = 1.0 / b                                # the host table: RN(1/b)
    q = rn(Fraction(a) * Fraction(rb))          # __dmul_rn(a, rb)
    r = rn(Fraction(a) - Fraction(q) * Fraction(b))    # __fma_rn(-q, b, a)
    return rn(Fraction(r) * Fraction(rb) + Fraction(q))  # __fma_rn(r, rb, q)


def with_mantissa(bits, exp):
    return struct.unpack("<d", struct.pack("<Q", ((exp + 1023) << 52) | (bits & ((1 << 52) - 1))))[0]


def test_random_operands_of_the_solver():
    rng = np.random.default_rng(2024)
    n = 40000
    b = 10.0 ** rng.uniform(-5, 2, n)          # spacings
    a = rng.standard_normal(n) * 10.0 ** rng.uniform(-12, 2, n)  # differences and sums
    bad = [(x, y) for x, y in zip(a.tolist(), b.tolist()) if markstein(x, y) != x / y]
    assert not bad, bad[:5]


def test_significand_edge_cases():
    cases = []
    for eb in (-17, -3, 0, 5):
        for mb in (0, 1, (1 << 52) - 1, (1 << 51), (1 << 52) - 2, 0x5555555555555, 0xAAAAAAAAAAAAA):
            b = with_mantissa(mb, eb)
            for ea in (-40, -9, 0, 3):
                for ma in (0, 1, (1 << 52) - 1, (1 << 51) + 1, 0x123456789ABCD, mb):
                    for s in (1.0, -1.0):
                        cases.append((s * with_mantissa(ma, ea), b))
    # near-ties: a = b * (q + 1/2 ulp) rounded, for quotients of every binade edge
    rng = np.random.default_rng(7)
    for _ in range(2000):
        b = float(10.0 ** rng.uniform(-4, 1))
        q = float(rng.uniform(1, 2)) * 2.0 ** int(rng.integers(-20, 20))
        ulp = math.ulp(q)
        cases.append((rn(Fraction(b) * (Fraction(q) + Fraction(ulp) / 2)), b))
        cases.append((rn(Fraction(b) * (Fraction(q) + Fraction(ulp) / 2)) + math.ulp(b * q), b))
    bad = [(x, y) for x, y in cases if markstein(x, y) != x / y]
    assert not bad, bad[:5]
