"""Accuracy of the oracle's scalar arithmetic against mpmath (600 / 1200 bits).

The oracle restates the reference's f128 (double-double, crates/quad/src/
dd.rs:61-195) and MultiFloat<N> (multifloat/{add,mul,div,math,
transcendental}.rs) operations. Its known-answer tests (test_oracle_kat.py)
pin it to the reference's own vectors; this file checks independently that
every operation is as accurate as the algorithm it restates, so that a
slip in the restatement (a lost error term, a wrong branch) cannot hide
behind the few reference vectors.

Bounds (relative error, measured maxima over these samples in brackets):
  f128 add/sub 2^-104 [2^-105.4], mul 2^-104 [2^-104.6],
  div 2^-103.5 [2^-103.8], recip 2^-103.5 [2^-104.1], sqrt 2^-104 [2^-105.1];
  exp (|x| + 1) 2^-104.5: dd.rs:106-121 reduces by k = round(x / ln 2) with
  the double-double LN2, whose rounding error is multiplied by k [2^-96.6 at
  x = 568, 2^-100.6 for |x| <= 40]. Arguments stay above -600 so that the
  result's low limb is a normal double.
  MultiFloat<4>: add 2^-212, mul/div 2^-210, sqrt 2^-212, exp(|x| <= 40) 2^-203
  [2^-214.6, -211.9, -212.2, -213.8, -205.1]; MultiFloat<8> (the f512
  checker): add 2^-428, mul/div 2^-422, sqrt 2^-425, exp 2^-410
  [2^-431.1, -425.0, -426.3, -428.1, -413.2].
"""
import math

import mpmath as mp
import numpy as np
import pytest

import oracle as O

SAMPLES = 1500


def _dd(rng, scale_exp=30):
    hi = rng.standard_normal() * 2.0 ** int(rng.integers(-scale_exp, scale_exp))
    lo = hi * 2.0 ** -53 * rng.uniform(-1, 1)
    s = hi + lo
    return np.array([s, lo - (s - hi)])


def _val(v):
    return sum((mp.mpf(float(t)) for t in v), mp.mpf(0))


def _rel(got, exact):
    return abs((_val(got) - exact) / exact)


F128_CASES = {
    "add": (O.dd_add, lambda a, b: _val(a) + _val(b), 2, -104.0),
    "sub": (O.dd_sub, lambda a, b: _val(a) - _val(b), 2, -104.0),
    "mul": (O.dd_mul, lambda a, b: _val(a) * _val(b), 2, -104.0),
    "div": (O.dd_div, lambda a, b: _val(a) / _val(b), 2, -103.5),
    "recip": (O.dd_recip, lambda a: 1 / _val(a), 1, -103.5),
    "sqrt": (O.dd_sqrt, lambda a: mp.sqrt(_val(a)), 1, -104.0),
}


@pytest.mark.parametrize("op", sorted(F128_CASES))
def test_f128_op_accuracy(op):
    fn, exact, nargs, log2_bound = F128_CASES[op]
    rng = np.random.default_rng(100 + sorted(F128_CASES).index(op))
    worst = 0.0
    with mp.workprec(600):
        for _ in range(SAMPLES):
            args = [_dd(rng) for _ in range(nargs)]
            if op == "sqrt":
                args = [np.abs(args[0]) if args[0][0] > 0 else -args[0]]
            worst = max(worst, float(_rel(fn(*args), exact(*args))))
    assert worst <= 2.0 ** log2_bound, (op, math.log2(worst))


def test_f128_exp_accuracy():
    rng = np.random.default_rng(7)
    worst = 0.0
    with mp.workprec(600):
        for _ in range(SAMPLES):
            x = rng.uniform(-600, 700)
            lo = x * 2.0 ** -54 * rng.uniform(-1, 1)
            a = np.array([x + lo, lo - ((x + lo) - x)])
            r = float(_rel(O.dd_exp(a), mp.exp(_val(a))))
            worst = max(worst, r / (abs(x) + 1.0))
    assert worst <= 2.0 ** -104.5, math.log2(worst)


def test_f128_exp_of_zero_and_ln_roundtrip():
    assert np.array_equal(O.dd_exp(np.array([0.0, 0.0])), [1.0, 0.0])  # dd.rs:107-109
    with mp.workprec(600):
        for x in (0.5, 2.0, 10.0, 1e-3):
            y = O.dd_ln(np.array([x, 0.0]))
            assert abs(_val(y) - mp.log(x)) <= 2.0 ** -100 * max(1.0, abs(float(mp.log(x))))


def _mf(rng, N, positive=False):
    x = rng.standard_normal() * 2.0 ** int(rng.integers(-20, 20))
    if positive:
        x = abs(x)
    limbs = [x]
    for _ in range(1, N):
        limbs.append(limbs[-1] * 2.0 ** -53 * rng.uniform(-1, 1))
    return np.array(limbs)


MF_BOUNDS = {4: {"add": -212, "mul": -210, "div": -210, "sqrt": -212, "exp": -203},
             8: {"add": -428, "mul": -422, "div": -422, "sqrt": -425, "exp": -410}}


@pytest.mark.parametrize("N", [4, 8])
@pytest.mark.parametrize("op", ["add", "mul", "div", "sqrt", "exp"])
def test_multifloat_op_accuracy(N, op):
    rng = np.random.default_rng(1000 * N + len(op))
    worst = 0.0
    with mp.workprec(1200):
        for _ in range(SAMPLES // 5):
            if op in ("add", "mul", "div"):
                a, b = _mf(rng, N), _mf(rng, N)
                exact = {"add": _val(a) + _val(b), "mul": _val(a) * _val(b), "div": _val(a) / _val(b)}[op]
                got = O.mf_op(op, N, a, b)
            elif op == "sqrt":
                a = _mf(rng, N, positive=True)
                exact, got = mp.sqrt(_val(a)), O.mf_op(op, N, a)
            else:
                a = np.zeros(N)
                a[0] = rng.uniform(-40, 40)
                exact, got = mp.exp(_val(a)), O.mf_op(op, N, a)
            worst = max(worst, float(_rel(got, exact)))
    assert worst <= 2.0 ** MF_BOUNDS[N][op], (N, op, math.log2(worst))
