"""Text exchange in the reference's serde formats (host code of the library).

The expected strings are built independently here with Python's correctly
rounded formatting, rewritten to Rust's exponent style, which is what
format!("{:+.18e}") / format!("{:+.14e}") print (dd.rs:448-461,
multifloat/traits.rs:15-34): mantissa digits are the correctly rounded
decimal in both languages, Rust writes "e-5" / "e0" where printf writes
"e-05" / "e+00", and NaN as "NaN". Parsing mirrors parse_dd_string
(dd.rs:495-509) and parse_limbs_string (traits.rs:104-150), including the
exponent-sign exception and the rejection of malformed strings. No GPU is
needed: these entry points run on the host.
"""
import math

import numpy as np
import pytest

import quadprec_b200 as hp


def rust_exp(x: float, prec: int) -> str:
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "+inf" if x > 0 else "-inf"
    s = f"{x:+.{prec}e}"
    mant, ex = s.split("e")
    return f"{mant}e{int(ex)}"


def samples(n, seed):
    rng = np.random.default_rng(seed)
    hi = rng.standard_normal(n) * 10.0 ** rng.integers(-300, 300, n)
    lo = hi * 2.0 ** -53 * rng.uniform(-1, 1, n)
    return np.stack([hi, lo], -1)


def test_f128_strings_match_rust_format_and_round_trip():
    vals = samples(500, 1)
    vals[0] = [0.0, 0.0]
    vals[1] = [-0.0, 0.0]
    vals[2] = [1.0, 1e-300]
    vals[3] = [5e-324, -5e-324]
    vals[4] = [1.7976931348623157e308, -9.9e291]
    for v in vals:
        s = hp.f128_to_string(v)
        assert s == rust_exp(v[0], 18) + "+" + rust_exp(v[1], 18), s
        back = hp.f128_from_string(s)
        assert np.array_equal(back, v) and np.array_equal(np.signbit(back), np.signbit(v)), (s, back, v)


def test_f128_parse_rules():
    # the '+' inside an exponent ("e+05") is not the separator
    assert np.array_equal(hp.f128_from_string("1.5e+05+-2e-12"), [1.5e5, -2e-12])
    assert np.array_equal(hp.f128_from_string("+1e0+-0e0"), [1.0, -0.0])
    assert np.isinf(hp.f128_from_string("+inf++0e0")[0])
    assert np.isnan(hp.f128_from_string("NaN++0e0")[0])
    for bad in ["", "1.0", "1.0+", "1.0+2.0", "abc++1e0", "1.0++1e0x", "0x1p3++1e0", " 1.0++1e0"]:
        with pytest.raises(hp.HPError):
            hp.f128_from_string(bad)


@pytest.mark.parametrize("N", [2, 4, 8])
def test_multifloat_strings_match_rust_format(N):
    rng = np.random.default_rng(N)
    for _ in range(200):
        x = rng.standard_normal() * 10.0 ** rng.integers(-200, 200)
        v = np.array([x * 2.0 ** (-53 * t) * rng.uniform(-1, 1) if t else x for t in range(N)])
        s = hp.mf_to_string(v)
        assert s == "+".join(rust_exp(float(t), 14) for t in v), s
        # "{:+.14e}" keeps 15 significant digits: parsing gives each limb back
        # to 15 digits, and parsing that string again is exact
        back = hp.mf_from_string(s, N)
        assert np.allclose(back, v, rtol=1e-14, atol=0)
        assert hp.mf_to_string(back) == s
    exact = "+6.93147180559945e-1++2.31904681384630e-17"
    assert np.array_equal(hp.mf_from_string(exact, 2), [0.693147180559945, 2.3190468138463e-17])


def test_multifloat_parse_rules():
    assert np.array_equal(hp.mf_from_string("+1.0e+05+-2.0e-05++3.0e0", 3), [1e5, -2e-5, 3.0])
    for bad, n in [("+1e0++2e0", 3), ("+1e0++2e0++3e0", 2), ("+1e0++", 2), ("+1e0+ 2e0", 2), ("", 1)]:
        with pytest.raises(hp.HPError):
            hp.mf_from_string(bad, n)
