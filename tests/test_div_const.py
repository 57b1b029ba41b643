"""The FP64 Lagrange weights divide by 12, 24 and 120 with one FMA correction of a
product with the rounded reciprocal (div_const in csrc/dl_interp.cu).  This checks the
method against correctly rounded division (Python's float division) on the weights'
numerators over the fraction range [0, 1), on random doubles of every binade, and on
quotients that are exactly representable or lie next to a rounding boundary.  The FMA is
emulated exactly with rationals (one rounding of the exact a * b + c).  The GPU parity
tests then compare the device weights' interpolation with the oracle's bit for bit."""
from fractions import Fraction
import random
import struct

import pytest


def fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def div_const(x, d):
    inv = 1.0 / d
    q = x * inv
    r = fma(-q, float(d), x)
    return q if r == 0.0 else fma(r, inv, q)


def numerators(z):
    """The numerators of partlib.f90:317-338 in source order, with their divisors."""
    z2 = z * z
    z3 = z2 * z
    z4 = z3 * z
    z5 = z4 * z
    return [
        (6.0 * z - 5.0 * z2 - 5.0 * z3 + 5.0 * z4 - z5, 120),
        (-12.0 * z + 16.0 * z2 - z3 - 4.0 * z4 + z5, 24),
        (12.0 - 4.0 * z - 15.0 * z2 + 5.0 * z3 + 3.0 * z4 - z5, 12),
        (12.0 * z + 8.0 * z2 - 7.0 * z3 - 2.0 * z4 + z5, 12),
        (-6.0 * z - z2 + 7.0 * z3 + z4 - z5, 24),
        (4.0 * z - 5.0 * z3 + z5, 120),
    ]


def _bits(x):
    return struct.pack("<d", x)


def _next(x, s):
    b = struct.unpack("<q", struct.pack("<d", x))[0]
    b += s if x >= 0 else -s
    return struct.unpack("<d", struct.pack("<q", b))[0]


def test_weights_numerators_random_fractions():
    rng = random.Random(20240611)
    zs = [rng.random() for _ in range(4000)]
    zs += [0.0, 0.5, 0.25, 1.0 - 2.0 ** -53, 2.0 ** -52, 1.0 / 3.0]
    for z in zs:
        for x, d in numerators(z):
            assert _bits(div_const(x, d)) == _bits(x / d), (z, x, d)


@pytest.mark.parametrize("d", [12, 24, 120])
def test_random_doubles_every_binade(d):
    rng = random.Random(d)
    for _ in range(3000):
        m = rng.getrandbits(52) | (1 << 52)
        e = rng.randint(-1000, 1000)
        x = m * 2.0 ** (e - 52)
        if rng.random() < 0.5:
            x = -x
        assert _bits(div_const(x, d)) == _bits(x / d), (x, d)


@pytest.mark.parametrize("d", [12, 24, 120])
def test_exact_and_near_boundary_quotients(d):
    rng = random.Random(7 * d)
    for _ in range(2000):
        # representable quotients, and dividends next to d times a double or d times a
        # midpoint between two doubles
        q = (rng.getrandbits(52) | (1 << 52)) * 2.0 ** rng.randint(-60, 60)
        for x0 in (Fraction(q) * d, (Fraction(q) + Fraction(q) * Fraction(1, 2 ** 53)) * d):
            x = float(x0)
            for x1 in (x, _next(x, +1), _next(x, -1)):
                assert _bits(div_const(x1, d)) == _bits(x1 / d), (x1, d)
    for x in (0.0, -0.0, 2.2250738585072014e-308, -2.2250738585072014e-308):
        assert _bits(div_const(x, d)) == _bits(x / d), (x, d)
