"""Pins the oracle's Obara-Saika overlaps of P, D and F shells
(crates/overlap/src/integral.rs:144-352 restated in oracle/hp_oracle.cpp).

The reference's only test of these shells checks the block size of a p-p
pair (integral.rs:428-438); the closed forms below pin the values: the
self-overlaps of primitive Cartesian Gaussians x^a y^b z^c exp(-alpha r^2)
are (pi/2alpha)^{3/2} prod (2k-1)!!/(4 alpha)^k, and an s-p overlap between
two centres is the derivative of the s-s overlap with respect to the p
centre divided by 2 alpha_p. CPU only.
"""
import math

import numpy as np

import oracle as O

# f64 tier for every pair: exponents above diffuse_threshold (screen.rs:70-75)
F64 = (0.1, 500.0, 1e-14, 12.0)
# f128 tier for every near pair: diffuse_threshold above every exponent
F128 = (1e9, 500.0, 1e-300, 1e9)


def dfact(n):
    return 1 if n <= 0 else n * dfact(n - 2)


def self_overlap(alpha, a, b, c):
    base = (math.pi / (2 * alpha)) ** 1.5
    return base * math.prod(dfact(2 * k - 1) / (4 * alpha) ** k for k in (a, b, c))


def comps(l):
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


def test_p_shell_block_size():  # integral.rs:428-438
    m, tiers = O.assemble_overlap([1], [[0.0, 0.0, 0.0]], [np.array([1.0])], [np.array([1.0])], F64)
    assert m.shape == (3, 3) and list(tiers) == [1, 0, 0]


def test_self_overlaps_closed_form_both_tiers():
    for params in (F64, F128):
        for l in (1, 2, 3):
            alpha = 0.7 + 0.3 * l
            m, _ = O.assemble_overlap([l], [[0.3, -0.2, 0.5]], [np.array([alpha])], [np.array([1.0])], params)
            for k, (a, b, c) in enumerate(comps(l)):
                assert math.isclose(m[k, k], self_overlap(alpha, a, b, c), rel_tol=1e-14), (params, l, k)


def test_s_p_overlap_is_the_centre_derivative():
    a, b = 0.8, 1.3
    A, B = np.array([0.0, 0.0, 0.0]), np.array([0.7, -0.4, 0.2])
    m, _ = O.assemble_overlap([0, 1], [A, B], [np.array([a]), np.array([b])], [np.array([1.0]), np.array([1.0])], F64)

    def ss(Bc):
        g, mu = a + b, a * b / (a + b)
        return (math.pi / g) ** 1.5 * math.exp(-mu * float(np.sum((A - Bc) ** 2)))

    h = 1e-6
    for d in range(3):
        e = np.zeros(3)
        e[d] = h
        deriv = (ss(B + e) - ss(B - e)) / (2 * h)
        # d/dB_d of exp(-b |r-B|^2) = 2 b (r-B)_d exp(..): <s_A|p_d,B> = deriv / (2 b)
        assert math.isclose(m[1 + d, 0], deriv / (2 * b), rel_tol=1e-7), (d, m[1 + d, 0], deriv / (2 * b))
        assert m[0, 1 + d] == m[1 + d, 0]


def test_f64_and_f128_tiers_agree():
    rng = np.random.default_rng(3)
    ls = [0, 1, 2, 3, 1, 2]
    cen = rng.uniform(-1.5, 1.5, (len(ls), 3))
    al = [rng.uniform(0.3, 3.0, 2) for _ in ls]
    co = [rng.uniform(0.2, 1.0, 2) for _ in ls]
    m64, t64 = O.assemble_overlap(ls, cen, al, co, F64)
    m128, t128 = O.assemble_overlap(ls, cen, al, co, F128)
    assert t64[0] == len(ls) * (len(ls) + 1) // 2 and t128[1] == t64[0]
    assert np.allclose(m64, m128, rtol=1e-12, atol=1e-14 * np.abs(m128).max())
    assert np.array_equal(m128, m128.T)
