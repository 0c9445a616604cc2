"""The row engine divides by per-job constants (3 for the typical price, the
period for window means) without a divide instruction: div_by in
tacuda_b200/csrc/rows.cuh takes q0 = x*y with y = RN(1/d) and applies two FMA
corrections (Markstein's theorem). The GPU's DMUL and DFMA are IEEE-754
operations, so the method is checked here with exact rational arithmetic:
every product, and every FMA as one rounding of the exact value, must give the
correctly rounded quotient x / d (Python's float division)."""
from __future__ import annotations

import math
import random
from fractions import Fraction

import pytest


def rn(v: Fraction) -> float:
    return float(v)  # correctly rounded to nearest even


def fma(a: float, b: float, c: float) -> float:
    return rn(Fraction(a) * Fraction(b) + Fraction(c))


def div_by(x: float, d: float, y: float) -> float:
    q0 = x * y
    if q0 == 0.0 or not math.isfinite(q0):
        return q0  # the kernel computes the corrections too and selects q0
    q1 = fma(fma(-q0, d, x), y, q0)
    return fma(fma(-q1, d, x), y, q1)


@pytest.mark.parametrize("d", [3.0] + [float(p) for p in (1, 2, 5, 7, 9, 10, 11, 13, 14, 20, 26, 30, 49, 64, 200)])
def test_div_by_is_correctly_rounded(d):
    rng = random.Random(int(d) * 7919)
    y = 1.0 / d
    xs = [rng.uniform(-1, 1) * 2.0 ** rng.randint(-60, 60) for _ in range(3000)]
    # sums of float32 prices and their near-ties
    xs += [float(rng.randint(1, 1 << 24)) * 2.0 ** rng.randint(-30, 10) for _ in range(1000)]
    xs += [math.nextafter(k * d, math.inf) for k in range(1, 200)] + [k * d for k in range(1, 200)]
    for x in xs:
        assert div_by(x, d, y) == x / d, (x, d)


def test_div_by_special_values():
    y = 1.0 / 3.0
    assert div_by(math.inf, 3.0, y) == math.inf
    assert div_by(-math.inf, 3.0, y) == -math.inf
    assert math.isnan(div_by(math.nan, 3.0, y))
    assert div_by(0.0, 3.0, y) == 0.0
    # constant windows: three equal float32 prices give that price back
    for v in (1.0, 100.03125, 123.456787109375, 1e4 + 0.5):
        assert div_by(v + v + v, 3.0, y) == v
