"""Pins the CPU oracle to hyperprec's own known-answer tests.

Each test restates one #[test] of the reference (cited by file:line) against
the oracle, with the reference's tolerance. These are the golden vectors the
reference ships for this path; the oracle is trusted only because it passes
them (plus the mpmath cross-checks in test_oracle_mpmath.py).
"""
import math

import numpy as np
import pytest

import oracle as O


def f128v(vals):
    v = np.asarray(vals, dtype=np.float64)
    return np.stack([v, np.zeros_like(v)], axis=-1)


def to_f64(x):
    return x[..., 0] + x[..., 1]


def mf(vals, N):
    v = np.asarray(vals, dtype=np.float64)
    out = np.zeros(v.shape + (N,))
    out[..., 0] = v
    return out


# ---- crates/quad/src/linalg.rs tests ----
def test_dot_basic():  # linalg.rs:369-374
    r = O.dot(f128v(range(100)), f128v([1.0] * 100))
    assert abs(to_f64(r) - 4950.0) < 1e-10


def test_cholesky_3x3():  # linalg.rs:377-403
    orig = np.array([[4.0, 2, 0], [2, 5, 1], [0, 1, 6]])
    L = O.cholesky(f128v(orig.ravel()).reshape(3, 3, 2), 3)
    for i in range(3):
        for j in range(3):
            s = np.zeros(2)
            for k in range(min(i, j) + 1):
                s = O.dd_add(s, O.dd_mul(L[i, k], L[j, k]))
            assert abs(to_f64(s) - orig[i, j]) < 1e-28


def test_cholesky_parallel_200x200():  # linalg.rs:406-418
    n = 200
    i = np.arange(n, dtype=np.float64)
    a = f128v((1.0 / (np.abs(i[:, None] - i[None, :]) + 1.0)).ravel()).reshape(n, n, 2)
    for d in range(n):
        a[d, d] = O.dd_add(a[d, d], O.dd(2.0))
    O.cholesky(a, n)


def test_gemm_identity():  # linalg.rs:423-434
    eye = f128v(np.eye(3).ravel()).reshape(3, 3, 2)
    a = f128v(range(1, 10)).reshape(3, 3, 2)
    c = O.gemm(eye, a, 3, 3, 3)
    assert np.all(np.abs(to_f64(c) - to_f64(a)) < 1e-28)


def test_gemm_2x2():  # linalg.rs:437-447
    c = O.gemm(f128v([1, 2, 3, 4]).reshape(2, 2, 2), f128v([5, 6, 7, 8]).reshape(2, 2, 2), 2, 2, 2)
    assert np.all(np.abs(to_f64(c).ravel() - [19, 22, 43, 50]) < 1e-28)


def test_gemm_atb_matches_transpose():  # linalg.rs:450-462
    a = f128v([1, 2, 3, 4, 5, 6]).reshape(3, 2, 2)
    b = f128v(range(1, 13)).reshape(3, 4, 2)
    at = f128v([1, 3, 5, 2, 4, 6]).reshape(2, 3, 2)
    c1 = O.gemm(at, b, 2, 4, 3)
    c2 = O.gemm(a, b, 2, 4, 3, atb=True)
    assert np.array_equal(c1, c2)


def make_spd(n):  # linalg.rs:466-475
    i = np.arange(n, dtype=np.float64)
    a = f128v((1.0 / (np.abs(i[:, None] - i[None, :]) + 1.0)).ravel()).reshape(n, n, 2)
    for d in range(n):
        a[d, d] = O.dd_add(a[d, d], O.dd(float(n)))
    return a


def test_blocked_matches_unblocked():  # linalg.rs:478-491
    n = 20
    a = make_spd(n)
    le = O.cholesky(a, n)
    lb = O.cholesky_blocked(a, n, 8)
    for i in range(n):
        for j in range(i + 1):
            assert abs(to_f64(O.dd_sub(le[i, j], lb[i, j]))) < 1e-28


def test_jacobi_2x2():  # linalg.rs:496-509
    ev, vec, _ = O.jacobi_eigen(f128v([2, 1, 1, 2]).reshape(2, 2, 2), 2, 100)
    e = sorted(to_f64(ev))
    assert abs(e[0] - 1.0) < 1e-28 and abs(e[1] - 3.0) < 1e-28
    d = O.dd_add(O.dd_mul(vec[0, 0], vec[1, 0]), O.dd_mul(vec[0, 1], vec[1, 1]))
    assert abs(to_f64(d)) < 1e-28


def test_jacobi_3x3():  # linalg.rs:512-530
    a = f128v([4, 1, 0, 1, 3, 1, 0, 1, 2]).reshape(3, 3, 2)
    ev, vec, _ = O.jacobi_eigen(a, 3, 200)
    for i in range(3):
        av = O.matvec(a, vec[i], 3)
        for j in range(3):
            err = to_f64(O.dd_sub(av[j], O.dd_mul(ev[i], vec[i, j])))
            assert abs(err) < 1e-27
    assert abs(sum(to_f64(ev)) - 9.0) < 1e-25


def test_jacobi_identity():  # linalg.rs:533-541
    ev, _, _ = O.jacobi_eigen(f128v(np.eye(4).ravel()).reshape(4, 4, 2), 4, 10)
    assert np.all(np.abs(to_f64(ev) - 1.0) < 1e-30)


def test_solve_roundtrip():  # linalg.rs:544-563
    from quadprec_b200.workloads import shifted_hilbert

    n = 4
    a, b = shifted_hilbert(n)
    # same construction as the reference (f128 + f128 on the diagonal)
    ref = f128v((1.0 / (np.arange(n)[:, None] + np.arange(n)[None, :] + 1.0)).ravel()).reshape(n, n, 2)
    for d in range(n):
        ref[d, d] = O.dd_add(ref[d, d], O.dd(1.0))
    assert np.array_equal(a, ref)
    L = O.cholesky(a, n)
    x = O.solve_cholesky(L, b, n)
    ax = O.matvec(a, x, n)
    for i in range(n):
        assert abs(to_f64(O.dd_sub(ax[i], b[i]))) < 1e-28


def test_cholesky_not_spd_reports_pivot():  # linalg.rs:54-57
    a = f128v([1, 2, 2, 1]).reshape(2, 2, 2)
    with pytest.raises(O.CholeskyError) as ei:
        O.cholesky(a, 2)
    assert ei.value.pivot == 1 and ei.value.value == pytest.approx(-3.0)


def test_jacobi_no_converge():  # linalg.rs:361
    a = f128v([2, 1, 1, 2]).reshape(2, 2, 2)
    with pytest.raises(RuntimeError):
        O.jacobi_eigen(a, 2, 0)


# ---- crates/quad/src/multifloat/linalg.rs tests (N = 4) ----
def test_mf_dot_and_gemv():  # multifloat/linalg.rs:185-206
    eye = mf(np.eye(3).ravel(), 4).reshape(3, 3, 4)
    y = O.mf_gemv(4, eye, mf([1, 2, 3], 4), 3, 3)
    assert np.all(np.abs(y[:, 0] + y[:, 1] - [1, 2, 3]) < 1e-28)


def test_mf_gemm_2x2_and_atb():  # multifloat/linalg.rs:209-234
    c = O.mf_gemm(4, mf([1, 2, 3, 4], 4).reshape(2, 2, 4), mf([5, 6, 7, 8], 4).reshape(2, 2, 4), 2, 2, 2)
    assert np.all(np.abs(c[..., 0].ravel() - [19, 22, 43, 50]) < 1e-28)
    a = mf([1, 2, 3, 4, 5, 6], 4).reshape(3, 2, 4)
    b = mf(range(1, 13), 4).reshape(3, 4, 4)
    at = mf([1, 3, 5, 2, 4, 6], 4).reshape(2, 3, 4)
    assert np.array_equal(O.mf_gemm(4, at, b, 2, 4, 3), O.mf_gemm(4, a, b, 2, 4, 3, atb=True))


@pytest.mark.parametrize("N,eps", [(4, 1e-63), (8, 1e-127)])
def test_mf_cholesky_solve(N, eps):  # multifloat/tests.rs:618-660
    if N == 4:
        a0 = mf([4, 2, 2, 3], 4).reshape(2, 2, 4)
        n = 2
    else:
        a0 = mf([4, 2, 0, 2, 5, 1, 0, 1, 6], 8).reshape(3, 3, 8)
        n = 3
    L = O.mf_cholesky(N, a0, n)
    b = mf([1.0] * n, N)
    x = O.mf_cholesky_solve(N, L, b, n)
    ax = O.mf_gemv(N, a0, x, n, n)
    for i in range(n):
        d = O.mf_op("add", N, ax[i], -b[i])
        assert abs(d[0]) < eps


def test_mf_cholesky_3x3():  # multifloat/linalg.rs:237-263
    orig = np.array([[4.0, 2, 0], [2, 5, 1], [0, 1, 6]])
    L = O.mf_cholesky(4, mf(orig.ravel(), 4).reshape(3, 3, 4), 3)
    for i in range(3):
        for j in range(3):
            s = np.zeros(4)
            for k in range(min(i, j) + 1):
                s = O.mf_op("add", 4, s, O.mf_op("mul", 4, L[i, k], L[j, k]))
            assert abs(s[0] + s[1] - orig[i, j]) < 1e-28


# ---- crates/quad/src/multifloat/tests.rs arithmetic tests ----
@pytest.mark.parametrize("N,eps", [(4, 1e-63), (8, 1e-127)])
def test_mf_one_third_roundtrip(N, eps):  # tests.rs:48-64
    third = O.mf_op("div", N, mf(1.0, N), mf(3.0, N))
    back = O.mf_op("mul", N, third, mf(3.0, N))
    d = O.mf_op("add", N, back, -mf(1.0, N))
    assert abs(d[0]) < eps


def test_f256_one_third_golden_limbs():  # mul.rs:303-306 (1/3 limbs)
    third = O.mf_op("div", 4, mf(1.0, 4), mf(3.0, 4))
    assert third[0] == 1.0 / 3.0
    assert abs(third[1] - 1.850371707708594e-17) < 1e-31


@pytest.mark.parametrize("N,eps", [(4, 1e-63), (8, 1e-127)])
def test_mf_sqrt_two_squared(N, eps):  # tests.rs:162-176
    r = O.mf_op("sqrt", N, mf(2.0, N))
    sq = O.mf_op("mul", N, r, r)
    assert abs(O.mf_op("add", N, sq, -mf(2.0, N))[0]) < eps


@pytest.mark.parametrize("N,tol", [(4, 1e-55), (8, 1e-110)])
def test_mf_exp_times_exp_neg(N, tol):  # transcendental tests, tests.rs:226-240
    e1 = O.mf_op("exp", N, mf(1.0, N))
    em = O.mf_op("exp", N, mf(-1.0, N))
    p = O.mf_op("mul", N, e1, em)
    assert abs(O.mf_op("add", N, p, -mf(1.0, N))[0]) < tol


def test_mf_ln2_constant():  # transcendental.rs:4-9 (LN2 limbs), via exp(ln2) = 2
    ln2 = np.array([6.931471805599452862e-01, 2.319046813846299558e-17,
                    5.707708438416212066e-34, -3.582432210601811423e-50])
    e = O.mf_op("exp", 4, ln2)
    assert abs(O.mf_op("add", 4, e, -mf(2.0, 4))[0]) < 1e-55


# ---- crates/quad/src/dd.rs scalar tests ----
def test_dd_sqrt_and_exp():  # dd.rs tests: sqrt(2)^2, exp(ln2) = 2
    r = O.dd_sqrt(O.dd(2.0))
    assert abs(to_f64(O.dd_sub(O.dd_mul(r, r), O.dd(2.0)))) < 1e-30
    e = O.dd_exp(np.array([0.6931471805599453, 2.3190468138462996e-17]))
    assert abs(to_f64(O.dd_sub(e, O.dd(2.0)))) < 1e-30
    assert np.array_equal(O.dd_exp(O.dd(0.0)), [1.0, 0.0])


# ---- crates/solver/src/lib.rs tests ----
def hilbert(n):
    i = np.arange(n, dtype=np.float64)
    return 1.0 / (i[:, None] + i[None, :] + 1.0)


def test_solve_well_conditioned():  # solver/src/lib.rs:271-285
    n = 10
    a = hilbert(n) + np.eye(n)
    sol = O.solve_spd(a, np.ones(n), n)
    assert sol["strategy"] == "Float64" and sol["residual_norm"] < 1e-12


def test_solve_hilbert_13():  # solver/src/lib.rs:287-297
    sol = O.solve_spd(hilbert(13), np.ones(13), 13)
    assert sol["strategy"] in ("Float128", "MixedPrecision") and sol["kappa"] > 1e12


def test_solve_hilbert_12_mixed():  # solver/src/lib.rs:299-317
    a = hilbert(12)
    sol = O.solve_spd(a, a.sum(axis=1), 12)
    assert sol["strategy"] == "MixedPrecision" and sol["residual_norm"] < 1e-25


def test_solve_hilbert_12_f128_input():  # solver/src/lib.rs:319-340
    n = 12
    a = f128v(hilbert(n).ravel()).reshape(n, n, 2)
    b = np.zeros((n, 2))
    for i in range(n):
        for j in range(n):
            b[i] = O.dd_add(b[i], O.dd_mul(a[i, j], O.dd(1.0)))
    sol = O.solve_spd_f128(a, b, n)
    err = math.sqrt(sum(to_f64(O.dd_sub(x, O.dd(1.0))) ** 2 for x in sol["x"]))
    assert err < 1e-15


def hilbert_f128(n):  # demo/src/main.rs:93-102: f128::ONE / f128::from_f64(i+j+1)
    a = np.zeros((n, n, 2))
    for i in range(n):
        for j in range(n):
            a[i, j] = O.dd_div(O.dd(1.0), O.dd(float(i + j + 1)))
    return a


# README.md:188-195 (demo/src/main.rs:63-80): ||x-1|| and ||r|| per n.
README_HILBERT = {12: (9.89e-18, 1.18e-31), 13: (1.05e-16, 5.70e-32), 14: (5.10e-14, 5.59e-32),
                  15: (5.22e-12, 9.14e-32), 18: (5.46e-8, 1.09e-31), 20: (9.52e-5, 1.07e-31)}


@pytest.mark.parametrize("n", sorted(README_HILBERT))
def test_readme_hilbert_table(n):
    import mpmath as mp

    a = hilbert_f128(n)
    b = np.zeros((n, 2))
    for i in range(n):
        for j in range(n):
            b[i] = O.dd_add(b[i], O.dd_mul(a[i, j], O.dd(1.0)))
    sol = O.solve_spd_f128(a, b, n)
    ref_err, ref_r = README_HILBERT[n]
    # README claim: the residual stays at the f128 floor (~1e-31) for all n.
    assert sol["residual_norm"] < 2e-31
    # The README digits themselves are not reproducible: the exact solution x*
    # of this dd-stored system already differs from 1 by more than the
    # README's ||x-1|| at n = 12 (b carries dd rounding, amplified by kappa),
    # so the README was printed by another revision. What is checked instead:
    # the solve is accurate against x* (mpmath, 400 bits) to kappa * n * 2^-104,
    # and ||x-1|| has the README's order of magnitude.
    mp.mp.prec = 400
    A = mp.matrix(n, n)
    B = mp.matrix(n, 1)
    for i in range(n):
        B[i] = mp.mpf(b[i, 0]) + mp.mpf(b[i, 1])
        for j in range(n):
            A[i, j] = mp.mpf(a[i, j, 0]) + mp.mpf(a[i, j, 1])
    xs = mp.lu_solve(A, B)
    err_star = math.sqrt(sum(float((mp.mpf(sol["x"][i, 0]) + mp.mpf(sol["x"][i, 1]) - xs[i]) ** 2)
                             for i in range(n)))
    # sol["kappa"] is the reference's diagonal-ratio estimate (linalg.rs:185),
    # far below the true condition number of Hilbert matrices; bound with the
    # true kappa_inf from mpmath.
    kappa = float(mp.mnorm(A, 1) * mp.mnorm(mp.inverse(A), 1))
    assert err_star <= kappa * n * 2.0 ** -104
    err = math.sqrt(sum(to_f64(O.dd_sub(x, O.dd(1.0))) ** 2 for x in sol["x"]))
    assert ref_err / 30 < err < ref_err * 30


# ---- crates/overlap tests ----
def _norm(alpha):
    return (2.0 * alpha / math.pi) ** 0.75


def h2_basis():  # assemble.rs:92-114
    al = [3.42525, 0.62391, 0.16886]
    co = [0.15433 * _norm(3.42525), 0.53533 * _norm(0.62391), 0.44463 * _norm(0.16886)]
    return np.array([[0.0, 0, 0], [1.4, 0, 0]]), [al, al], [co, co]


def test_h2_overlap_symmetric():  # assemble.rs:116-130
    c, al, co = h2_basis()
    s, tiers = O.assemble_overlap_s(c, al, co)
    assert abs(s[0, 1] - s[1, 0]) < 1e-15
    assert abs(s[0, 0] - 1.0) < 0.02 and abs(s[1, 1] - 1.0) < 0.02
    assert 0.5 < s[0, 1] < 0.8


def test_all_tight_uses_f64():  # assemble.rs:132-139
    c, al, co = h2_basis()
    _, tiers = O.assemble_overlap_s(c, al, co)
    assert tiers["f128_pairs"] == 0 and tiers["f64_pairs"] > 0


def test_diffuse_triggers_f128():  # assemble.rs:141-164
    al = [50.0, 0.04]
    co = [0.3 * _norm(50.0), 0.7 * _norm(0.04)]
    _, tiers = O.assemble_overlap_s(np.array([[0.0, 0, 0], [2.0, 0, 0]]), [al, al], [co, co])
    assert tiers["f128_pairs"] > 0


def test_self_overlap_normalized():  # integral.rs:367-383
    s = O.overlap_primitive_f64(1.0, np.zeros(3), 1.0, np.zeros(3)) * _norm(1.0) ** 2
    assert abs(s - 1.0) < 1e-14


def test_f64_f128_agree_tight():  # integral.rs:385-408
    ca, cb = np.zeros(3), np.array([1.0, 0, 0])
    pa = [(10.0, 0.5), (5.0, 0.5)]
    pb = [(8.0, 0.6), (3.0, 0.4)]
    s64 = sum(x[1] * y[1] * O.overlap_primitive_f64(x[0], ca, y[0], cb) for x in pa for y in pb)
    s128 = np.zeros(2)
    for x in pa:
        for y in pb:
            sp = O.overlap_primitive_f128(x[0], ca, y[0], cb)
            s128 = O.dd_add(s128, O.dd_mul(O.dd_mul(O.dd(x[1]), O.dd(y[1])), sp))
    assert abs(s64 - to_f64(s128)) < 1e-14


def test_overlap_norm_dd_diagonal_and_symmetry():
    cen = np.array([[0.0, 0, 0], [1.4, 0.1, -0.2], [0.3, 2.0, 0.5]])
    al = np.array([0.5, 2.0, 0.03])
    s = O.overlap_norm_dd(cen, al)
    assert np.array_equal(s[np.arange(3), np.arange(3)], [[1.0, 0.0]] * 3)
    assert np.array_equal(s, s.transpose(1, 0, 2))


def _gen_eigen_residual(f, s, ev, c, n, m):
    """max_i |(F c_k)_i - eps_k (S c_k)_i| over k, in f128 (the reference
    tests' dd loops, ortho.rs:316-340)."""
    worst = 0.0
    for k in range(m):
        ck = c[:, k]
        fc = O.gemm(f, np.ascontiguousarray(ck.reshape(n, 1, 2)), n, 1, n).reshape(n, 2)
        sc = O.gemm(s, np.ascontiguousarray(ck.reshape(n, 1, 2)), n, 1, n).reshape(n, 2)
        for i in range(n):
            esc = O.dd_mul(ev[k], sc[i])
            d = O.dd_sub(fc[i], esc)
            worst = max(worst, abs(d[0] + d[1]))
    return worst


def test_solve_gen_eigen_2x2():  # solver/src/ortho.rs:303-343
    n = 2
    f = f128v([[2.0, 1.0], [1.0, 3.0]])
    s = f128v([[1.0, 0.2], [0.2, 1.0]])
    ev, c, m = O.solve_gen_eigen(f, s, n, 1e-8)
    assert m == 2
    assert _gen_eigen_residual(f, s, ev, c, n, m) < 1e-25
    assert ev[0, 0] + ev[0, 1] < ev[1, 0] + ev[1, 1]


def test_solve_gen_eigen_identity_overlap():  # solver/src/ortho.rs:346-377
    n = 3
    f = f128v([[3.0, 1.0, 0.0], [1.0, 2.0, 1.0], [0.0, 1.0, 4.0]])
    s = f128v(np.eye(n))
    ev, c, m = O.solve_gen_eigen(f, s, n, 1e-8)
    assert m == 3
    assert _gen_eigen_residual(f, s, ev, c, n, m) < 1e-25
