"""CPU check that the device arithmetic (hp_arith.cuh) reproduces the oracle.

hp_arith.cuh is compiled for the host with IEEE shims for the CUDA
intrinsics (tests/device_arith_shim.cpp) and compared bit-for-bit with the
oracle's restatement of dd.rs / multifloat/*.rs on random and adversarial
inputs: equal magnitudes of opposite sign (the stable-sort tie rule of
add.rs:43-54), exact zeros, cancellation, and limbs spanning the exponent
range. The GPU tests repeat the comparison on the device.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")


@pytest.fixture(scope="module")
def shim():
    os.makedirs(BUILD, exist_ok=True)
    so = os.path.join(BUILD, "libdevice_arith_shim.so")
    src = os.path.join(HERE, "device_arith_shim.cpp")
    hdrs = [os.path.join(HERE, "..", "quadprec_b200", "csrc", h) for h in ("hp_arith.cuh", "hp_mf.cuh")]
    if not os.path.exists(so) or os.path.getmtime(so) < max(os.path.getmtime(p) for p in [src, *hdrs]):
        subprocess.run(["/usr/bin/g++", "-O2", "-march=x86-64-v3", "-ffp-contract=off", "-fPIC", "-shared",
                        "-std=c++17", "-o", so, src], check=True)
    L = ctypes.CDLL(so)
    L.sh_batch.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long]
    return L


def run(shim, op, a, b, limbs):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b if b is not None else a, dtype=np.float64)
    o = np.zeros_like(a)
    shim.sh_batch(op, a.ctypes.data, b.ctypes.data, o.ctypes.data, a.shape[0])
    return o


def rand_dd(rng, n, spread=8):
    hi = rng.uniform(-1, 1, n) * 2.0 ** rng.integers(-spread, spread, n)
    lo = hi * 2.0 ** -53 * rng.uniform(-1, 1, n)
    s = hi + lo
    return np.stack([s, lo - (s - hi)], -1)


def rand_qd(rng, n, spread=8):
    out = np.zeros((n, 4))
    for i in range(n):
        x = rng.uniform(-1, 1) * 2.0 ** rng.integers(-spread, spread)
        limbs = [x * 2.0 ** (-53 * t) * rng.uniform(-1, 1) if t else x for t in range(4)]
        out[i] = limbs
        O.lib().or_mf_renormalize(4, O._p(out[i]))
    return out


@pytest.mark.parametrize("op,name", [(0, "add"), (1, "mul"), (2, "div"), (3, "sqrt"), (4, "recip"), (5, "exp")])
def test_dd_ops_bitexact(shim, op, name):
    rng = np.random.default_rng(op)
    a, b = rand_dd(rng, 3000), rand_dd(rng, 3000)
    if name == "sqrt":
        a[:, 0], a[:, 1] = np.abs(a[:, 0]), np.where(a[:, 0] < 0, -a[:, 1], a[:, 1])
    if name == "exp":
        a = a * 40.0
    # adversarial: exact cancellation, zeros, equal magnitudes
    a[:50] = b[:50] * np.array([-1.0, -1.0])
    a[50:60] = 0.0
    got = run(shim, op, a, b, 2)
    fn = {"add": O.dd_add, "mul": O.dd_mul, "div": O.dd_div, "sqrt": O.dd_sqrt,
          "recip": O.dd_recip, "exp": O.dd_exp}[name]
    for i in range(len(a)):
        want = fn(a[i], b[i]) if name in ("add", "mul", "div") else fn(a[i])
        assert np.array_equal(got[i], want, equal_nan=True), (name, i, a[i], b[i], got[i], want)


@pytest.mark.parametrize("op,name", [(10, "add"), (11, "mul"), (12, "div"), (13, "sqrt")])
def test_qd_ops_bitexact(shim, op, name):
    rng = np.random.default_rng(100 + op)
    n = 1500
    a, b = rand_qd(rng, n), rand_qd(rng, n)
    if name == "sqrt":
        a = np.where(a[:, :1] < 0, -a, a)
    # ties in |x| across limbs: a = -b, a = b with one limb negated, zeros
    a[:40] = -b[:40]
    a[40:80] = b[40:80]
    a[40:80, 2] = -a[40:80, 2]
    a[80:90] = 0.0
    a[90:100, 1:] = 0.0
    got = run(shim, op, a, b, 4)
    for i in range(n):
        want = O.mf_op(name, 4, a[i], b[i]) if name != "sqrt" else O.mf_op("sqrt", 4, a[i])
        assert np.array_equal(got[i], want, equal_nan=True), (name, i, a[i], b[i], got[i], want)


def rand_mf(rng, n, N, spread=8):
    out = np.zeros((n, N))
    for i in range(n):
        x = rng.uniform(-1, 1) * 2.0 ** rng.integers(-spread, spread)
        out[i] = [x * 2.0 ** (-53 * t) * rng.uniform(-1, 1) if t else x for t in range(N)]
        O.lib().or_mf_renormalize(N, O._p(out[i]))
    return out


@pytest.mark.parametrize("N", [4, 8])
@pytest.mark.parametrize("op,name", [(0, "add"), (1, "mul"), (2, "div"), (3, "sqrt")])
def test_mfn_templates_bitexact(shim, N, op, name):
    """hp_mf.cuh (the MultiFloat<N> templates behind the f512 kernels) against
    the oracle's MultiFloat<N> for N = 8, and for N = 4 (where they must also
    agree with the specialised qd_* of hp_arith.cuh)."""
    shim.sh_mfn_batch.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long]
    rng = np.random.default_rng(1000 * N + op)
    n = 600 if N == 8 else 1200
    a, b = rand_mf(rng, n, N), rand_mf(rng, n, N)
    if name == "sqrt":
        a = np.where(a[:, :1] < 0, -a, a)
    a[:30] = -b[:30]
    a[30:60] = b[30:60]
    a[30:60, 2] = -a[30:60, 2]
    a[60:70] = 0.0
    a[70:80, 1:] = 0.0
    a[80:90, N // 2:] = 0.0
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    got = np.zeros_like(a)
    shim.sh_mfn_batch((20 if N == 8 else 30) + op, a.ctypes.data, b.ctypes.data, got.ctypes.data, n)
    if N == 4:
        assert np.array_equal(got, run(shim, 10 + op, a, b, 4), equal_nan=True)
    for i in range(n):
        want = O.mf_op(name, N, a[i], b[i]) if name != "sqrt" else O.mf_op("sqrt", N, a[i])
        assert np.array_equal(got[i], want, equal_nan=True), (N, name, i, a[i], b[i], got[i], want)


def test_dd_exp_overlap_range_bitexact(shim):
    """The assembly's exp arguments -ab/(a+b) |R-R'|^2 lie in [-700, 0]: a
    dense sweep there (and near 0, where the Taylor loop runs longest) must
    reproduce the reference's bits, including its small-integer divisions."""
    rng = np.random.default_rng(2024)
    n = 100000
    hi = np.concatenate([-700.0 * rng.random(n // 2), -rng.random(n // 4) * 2.0 ** -rng.integers(0, 40, n // 4),
                         (rng.random(n - n // 2 - n // 4) - 0.5)])
    a = np.stack([hi, hi * 2.0 ** -53 * (rng.random(n) - 0.5)], -1)
    for i in range(n):  # renormalise (quick_two_sum)
        s = a[i, 0] + a[i, 1]
        a[i] = [s, a[i, 1] - (s - a[i, 0])]
    got = run(shim, 5, a, a, 2)
    want = np.array([O.dd_exp(a[i]) for i in range(n)])
    bad = np.nonzero(np.any(got != want, axis=1))[0]
    assert bad.size == 0, (bad[:5], a[bad[:5]], got[bad[:5]], want[bad[:5]])


def test_div_small_int_is_correctly_rounded(shim):
    """dd_exp divides its Taylor terms by i = 1..25 with an FMA sequence; it
    must give IEEE division's bits: 1e6 quotients per divisor 1..40,
    including values next to exact multiples and halfway points."""
    shim.sh_div_small_mismatches.restype = ctypes.c_long
    shim.sh_div_small_mismatches.argtypes = [ctypes.c_long, ctypes.c_int, ctypes.c_ulonglong]
    assert shim.sh_div_small_mismatches(1000000, 40, 2024) == 0


def test_dd_dot2_fast_error_bound(shim):
    """dd_dot2_fast (the batched Jacobi's fused rotation, c a + s b) against
    exact rational arithmetic: error below 4 2^-104 (|c a| + |s b|), on
    rotation pairs (c^2 + s^2 = 1 to f128) and operands of mixed magnitude,
    including near-total cancellation."""
    from fractions import Fraction as F

    shim.sh_dd_dot2.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_long]
    rng = np.random.default_rng(77)
    n = 4000
    th = rng.uniform(-np.pi, np.pi, n)
    c = np.stack([np.cos(th), np.zeros(n)], -1)
    s = np.stack([np.sin(th), np.zeros(n)], -1)
    c[:, 1] = c[:, 0] * 2.0 ** -53 * rng.uniform(-1, 1, n)
    s[:, 1] = s[:, 0] * 2.0 ** -53 * rng.uniform(-1, 1, n)
    a, b = rand_dd(rng, n, spread=20), rand_dd(rng, n, spread=20)
    # cancellation: b ~ -c a / s
    k = n // 4
    for i in range(k):
        ci = F(c[i, 0]) + F(c[i, 1])
        si = F(s[i, 0]) + F(s[i, 1])
        if si != 0:
            t = -ci * (F(a[i, 0]) + F(a[i, 1])) / si
            hi = float(t)
            b[i] = [hi, float(t - F(hi))]
    o = np.zeros((n, 2))
    arrs = [np.ascontiguousarray(x) for x in (c, a, s, b)]
    shim.sh_dd_dot2(*(x.ctypes.data for x in arrs), o.ctypes.data, n)
    for i in range(n):
        cv, av, sv, bv = (F(x[i, 0]) + F(x[i, 1]) for x in (c, a, s, b))
        exact = cv * av + sv * bv
        got = F(o[i, 0]) + F(o[i, 1])
        bound = F(4) * F(2) ** -104 * (abs(cv * av) + abs(sv * bv))
        assert abs(got - exact) <= bound, (i, float(abs(got - exact)), float(bound))


def test_dd_recip_fast_error_bound(shim):
    """dd_recip_fast (the batched Jacobi's rotation parameters): relative
    error below 2^-102 against exact rationals, over magnitudes 2^+-300 and
    both signs."""
    from fractions import Fraction as F

    rng = np.random.default_rng(78)
    n = 4000
    d = rand_dd(rng, n, spread=300)
    o = run(shim, 6, d, None, 2)
    for i in range(n):
        dv = F(d[i, 0]) + F(d[i, 1])
        got = F(o[i, 0]) + F(o[i, 1])
        assert abs(got * dv - 1) <= F(2) ** -102, (i, d[i], o[i])
