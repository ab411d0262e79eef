"""The hierarchy build's division (tree_kernel.cuh, div_by): a / b as

    r  = RN(1 / b)                 (correctly rounded reciprocal, __frcp_rn)
    q  = RN(a r)
    e  = RN(a - b q)               (one fused multiply-add: exact residual)
    q' = RN(q + e r)               (one fused multiply-add)

P. Markstein's final step for IEEE division (IBM J. Res. Dev. 34(1), 1990).
The build relies on q' being the correctly rounded quotient RN(a / b) for
normal-range single-precision operands, so that node centres stay bit-exact
with the reference formula's IEEE division.  Here the method is carried out
in exact rational arithmetic with round-to-nearest-even to binary32 after
every operation (what the hardware's RN operations and FMAs do), on random
operands and on the usual hard cases, and compared with RN(a / b).  The GPU
side is checked on every small node of the 800k tree in
test_gpu_parity.py::test_headline_workload_tree_matches_oracle_800k.
"""
from fractions import Fraction

import numpy as np


def rn32(x: Fraction) -> Fraction:
    """Round an exact rational to the nearest binary32 value, ties to even
    (normal range; no overflow or subnormal results in these operands)."""
    if x == 0:
        return Fraction(0)
    sign = -1 if x < 0 else 1
    x = abs(x)
    e = x.numerator.bit_length() - x.denominator.bit_length()
    if Fraction(2) ** e > x:
        e -= 1
    # x in [2^e, 2^(e+1)): 24 significant bits -> unit 2^(e-23)
    scaled = x / (Fraction(2) ** (e - 23))
    m = scaled.numerator // scaled.denominator
    rem = scaled - m
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and m % 2 == 1):
        m += 1
    return sign * Fraction(m) * Fraction(2) ** (e - 23)


def div_by(a: Fraction, b: Fraction) -> Fraction:
    r = rn32(1 / b)
    q = rn32(a * r)
    e = rn32(a - b * q)
    return rn32(q + e * r)


def f32(v) -> Fraction:
    return Fraction(float(np.float32(v)))


def test_markstein_step_is_correctly_rounded_on_random_operands():
    rng = np.random.default_rng(11)
    # numerators like c m sums (signed, wide range), denominators like masses
    a = rng.standard_normal(4000) * np.exp(rng.uniform(-20.0, 20.0, 4000))
    b = np.exp(rng.uniform(-25.0, 5.0, 4000))
    bad = []
    for x, y in zip(a.astype(np.float32), b.astype(np.float32)):
        fa, fb = f32(x), f32(y)
        if div_by(fa, fb) != rn32(fa / fb):
            bad.append((float(x), float(y)))
    assert not bad, bad[:5]


def test_markstein_step_on_hard_cases():
    # all-ones significands, powers of two, quotients near halfway points,
    # and equal operands
    ones = float(np.float32(2.0) - np.float32(2.0 ** -23))
    cases = [(1.0, ones), (ones, 1.0), (ones, ones), (1.0, 3.0), (2.0, 3.0), (1.0, 2.0 ** -10),
             (5.0, 7.0), (1.0 + 2.0 ** -23, 1.0 - 2.0 ** -24), (3.0, 1.5), (-1.0, 3.0)]
    rng = np.random.default_rng(5)
    for _ in range(2000):
        # b with a long run of ones, a a small integer multiple plus a nudge
        k = int(rng.integers(1, 24))
        b = float(np.float32(2.0 - 2.0 ** (-k)))
        a = float(np.float32(rng.integers(1, 1 << 20) * 2.0 ** int(rng.integers(-30, 10))))
        cases.append((a, b))
    bad = []
    for x, y in cases:
        fa, fb = f32(x), f32(y)
        if div_by(fa, fb) != rn32(fa / fb):
            bad.append((x, y))
    assert not bad, bad[:5]


def test_rounding_helper_matches_numpy_float32():
    rng = np.random.default_rng(2)
    for v in rng.standard_normal(2000) * np.exp(rng.uniform(-30, 30, 2000)):
        assert rn32(Fraction(float(v))) == Fraction(float(np.float32(v)))
