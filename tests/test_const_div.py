"""The FP64 kernels divide by the PPM constants 3, 6 and 12 without a division
instruction (divk in flash-x_b200/csrc/fxb_device.cuh): q0 = x * RN(1/C),
r = fma(-C, q0, x), q = copysign(fma(r, RN(1/C), q0), x), Markstein's
correction step.  The oracle divides (x / C).  This restates the sequence
with exact rational fused multiply-adds and checks that it returns the
correctly rounded quotient on random and structured inputs; the device
parity tests then compare whole steps bit for bit."""
import math
import random
import struct
from fractions import Fraction

import pytest


def _fma(a, b, c):
    # one rounding of the exact a*b + c (CPython rounds int/int division correctly)
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _divk(x, C):
    y = 1.0 / C
    q0 = x * y
    r = _fma(-float(C), q0, x)
    return math.copysign(_fma(r, y, q0), x)


def _bits(v):
    return struct.unpack("<Q", struct.pack("<d", v))[0]


@pytest.mark.parametrize("C", [3, 6, 12])
def test_markstein_constant_division_is_correctly_rounded(C):
    rng = random.Random(20261203 + C)
    xs = [0.0, -0.0, 1.0, -1.0, 3.0, 6.0, 12.0, 1e-300, -1e300, 2.0 ** -1000]
    for _ in range(6000):
        mant = rng.getrandbits(52)
        exp = rng.randint(1023 - 900, 1023 + 900)
        sign = rng.getrandbits(1)
        xs.append(struct.unpack("<d", struct.pack("<Q", (sign << 63) | (exp << 52) | mant))[0])
    for k in range(2000):
        # significands near the all-ones, all-zeros and alternating patterns
        for pat in (k, 0xFFFFFFFFFFFFF ^ k, 0x5555555555555 ^ k, 0xAAAAAAAAAAAAA ^ k):
            xs.append(struct.unpack("<d", struct.pack("<Q", (1023 << 52) | (pat & 0xFFFFFFFFFFFFF)))[0])
    bad = [x for x in xs if _bits(_divk(x, C)) != _bits(x / C)]
    assert not bad, f"{len(bad)} quotients differ from x / {C}, first x = {bad[0]!r}"


def _rdiv_y(a, b):
    """rdiv_y of flash-x_b200/csrc/fxb_device.cuh: a / b from y = RN(1/b) by
    two correction steps q + (a - b q) y, the sign of a zero quotient by
    copysign."""
    y = 1.0 / b
    q = a * y
    q = _fma(_fma(-b, q, a), y, q)
    q = _fma(_fma(-b, q, a), y, q)
    return math.copysign(q, a * y)


def test_shared_reciprocal_division_is_correctly_rounded():
    rng = random.Random(20261204)

    def rnd(lo, hi):
        mant = rng.getrandbits(52)
        exp = rng.randint(1023 + lo, 1023 + hi)
        return struct.unpack("<d", struct.pack("<Q", (rng.getrandbits(1) << 63) | (exp << 52) | mant))[0]

    cases = [(0.0, 3.0), (-0.0, 3.0), (0.0, -3.0), (-0.0, -3.0), (1.0, 3.0), (2.0 - 2.0 ** -52, 2.0 - 2.0 ** -51)]
    cases += [(rnd(-300, 300), rnd(-300, 300)) for _ in range(5000)]
    for _ in range(1500):
        # significands near all ones, where RN(1/b) is least accurate relative to b
        b = struct.unpack("<d", struct.pack("<Q", (1023 << 52) | (0xFFFFFFFFFFFFF - rng.getrandbits(16))))[0]
        a = struct.unpack("<d", struct.pack("<Q", (1023 << 52) | (0xFFFFFFFFFFFFF - rng.getrandbits(20))))[0]
        cases.append((a, b))
    bad = [(a, b) for a, b in cases if _bits(_rdiv_y(a, b)) != _bits(a / b)]
    assert not bad, f"{len(bad)} quotients differ from a / b, first {bad[0]!r}"
