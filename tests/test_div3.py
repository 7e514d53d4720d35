"""The FP64 deposition divides by 3 with Markstein's correction of a
reciprocal product (quill_b200/csrc/qp_physics.cuh, div3): q = RN(x r) with
r = RN(1/3), then RN(q + r (x - 3 q)) with the residual from one FMA.  This
restates it in exact rational arithmetic (each FMA is one rounding of the
exact value) and checks that it equals IEEE division x / 3 on random and
edge-case doubles over the whole normal range.  The GPU parity tests check the
device code against the reference's divisions bit for bit."""
from fractions import Fraction

import numpy as np

R = float.fromhex("0x1.5555555555555p-2")


def _div3(x: float) -> float:
    q = float(np.float64(x) * np.float64(R))           # RN(x r)
    e_exact = Fraction(x) - 3 * Fraction(q)            # fma(-q, 3, x) before rounding
    e = float(e_exact)
    assert Fraction(e) == e_exact, (x, "residual not exact")
    res = float(Fraction(q) + Fraction(e) * Fraction(R))  # fma(e, r, q): one rounding
    return float(np.copysign(res, x))


def test_reciprocal_is_rounded_one_third():
    assert R == 1.0 / 3.0
    assert abs(Fraction(R) - Fraction(1, 3)) == Fraction(1, 3) * Fraction(2) ** -54


def test_div3_equals_ieee_division():
    rng = np.random.default_rng(7)
    xs = []
    # random significands over the normal exponent range (results stay normal)
    m = rng.integers(0, 2 ** 52, size=20000, dtype=np.uint64)
    ex = rng.integers(-1000, 1000, size=20000)
    sg = rng.choice([-1.0, 1.0], size=20000)
    for mi, ei, si in zip(m, ex, sg):
        xs.append(si * np.ldexp(1.0 + float(mi) / 2 ** 52, int(ei)))
    # the products the deposition divides: displacement products in (-1, 1)
    xs += list(rng.uniform(-1, 1, 10000) * rng.uniform(-1, 1, 10000))
    # binade edges and multiples of 3
    for k in range(-60, 61):
        p = 2.0 ** k
        xs += [p, np.nextafter(p, 0), np.nextafter(p, np.inf), 3 * p, np.nextafter(3 * p, 0),
               np.nextafter(3 * p, np.inf), 1.5 * p, np.nextafter(1.5 * p, np.inf)]
    xs += [0.0, -0.0]
    bad = [x for x in xs if _div3(float(x)) != float(np.float64(x) / np.float64(3.0))
           or np.signbit(_div3(float(x))) != np.signbit(np.float64(x) / 3.0)]
    assert not bad, bad[:5]


def _div_fixed(x: float, y: float, r: float) -> float:
    """div_fixed (qp_physics.cuh): two FMA corrections of RN(x r), r = RN(1/y)."""
    q0 = float(np.float64(x) * np.float64(r))
    e0 = float(Fraction(x) - Fraction(q0) * Fraction(y))                 # fma(-q0, y, x)
    q1 = float(Fraction(q0) + Fraction(e0) * Fraction(r))               # fma(e0, r, q0)
    e1_exact = Fraction(x) - Fraction(q1) * Fraction(y)
    e1 = float(e1_exact)
    assert Fraction(e1) == e1_exact, (x, y, "second residual not exact")
    res = float(Fraction(q1) + Fraction(e1) * Fraction(r))
    return float(np.copysign(res, x))


def test_div_fixed_equals_ieee_division():
    """The FP64 push divides the displacement by the cell size (advance.cpp:
    281-284) with div_fixed; it must return x / y exactly."""
    rng = np.random.default_rng(11)
    ys = [2 * np.pi / 20, 2 * np.pi / 16, 2 * np.pi / 32, 2 * np.pi * np.float32(0.0625), 0.1, 3.0, 7.0]
    ys += list(np.exp(rng.uniform(np.log(1e-4), np.log(1e3), 40)))
    bad = []
    for y in ys:
        y = float(y)
        r = float(np.float64(1.0) / np.float64(y))
        xs = list(rng.uniform(-1, 1, 600) * y) + list(rng.standard_normal(300) * 10.0 ** rng.integers(-30, 30, 300))
        for k in range(-40, 41, 8):
            p = 2.0 ** k
            xs += [p * y, np.nextafter(p * y, 0), np.nextafter(p * y, np.inf), p, -p]
        xs += [0.0, -0.0]
        for x in xs:
            x = float(x)
            want = float(np.float64(x) / np.float64(y))
            got = _div_fixed(x, y, r)
            if got != want or np.signbit(got) != np.signbit(want):
                bad.append((x, y))
    assert not bad, bad[:5]
