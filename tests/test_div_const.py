"""The FP64 kernels divide by the reference's lattice constants through
div_const (csrc/lbrb_internal.cuh): q0 = RN(x * RN(1/c)), r = fma(-q0, c, x),
result = q0 if r == 0 else fma(r, RN(1/c), q0) (Markstein's correction).  This
restates those steps with exact rational arithmetic and checks that they give
the IEEE quotient RN(x / c) for every divisor the kernels use, over random
operands across 120 binades, operands whose quotients sit at binade edges,
and signed zeros.  (The GPU parity tests check the compiled kernels against
the oracle's IEEE divisions bit for bit.)"""
import math
import random
import struct
from fractions import Fraction

CS2 = 1.0 / 3.0
DIVISORS = {"2*CS2": 2.0 * CS2, "CS2": CS2, "2/9": 2.0 / 9.0, "CS2*CS2": CS2 * CS2}


def rn(q: Fraction) -> float:
    return float(q)  # CPython rounds a rational to the nearest double


def fma(a: float, b: float, c: float) -> float:
    exact = Fraction(a) * Fraction(b) + Fraction(c)
    if exact == 0:  # the sign of an exact zero sum in round-to-nearest
        return -0.0 if (math.copysign(1, a) * math.copysign(1, b) < 0 and math.copysign(1, c) < 0) else 0.0
    return rn(exact)


def div_const(x: float, c: float, rc: float) -> float:
    q0 = x * rc  # an IEEE product
    r = fma(-q0, c, x)
    return q0 if r == 0.0 else fma(r, rc, q0)


def bits(a: float) -> bytes:
    return struct.pack("<d", a)


def operands(c: float, rng: random.Random, n: int):
    xs = [rng.choice((-1.0, 1.0)) * math.ldexp(rng.random() + 0.5, rng.randint(-60, 60)) for _ in range(n)]
    for k in range(-40, 40):
        base = c * 2.0 ** k
        xs += [base + d * math.ulp(base) for d in range(-4, 5)]
    return xs + [0.0, -0.0, 1.0, -1.0, 3.0, 2.0 / 9.0, CS2, 1e-300, -1e300]


def test_div_const_is_the_ieee_quotient():
    rng = random.Random(17)
    for name, c in DIVISORS.items():
        rc = 1.0 / c
        assert rc == rn(1 / Fraction(c))  # RN(1/c)
        for x in operands(c, rng, 10000):
            want = x / c  # IEEE division of the host
            assert want == rn(Fraction(x) / Fraction(c)) or x == 0.0
            assert bits(div_const(x, c, rc)) == bits(want), (name, x)
