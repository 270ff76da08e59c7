"""GPU parity for Cholesky, triangular solves, matvec and the SPD solver.

Bit-identical to the oracle: cholesky (any internal block size),
cholesky_blocked (same nb), forward_solve, matvec, cond_estimate.
Within the normwise bound: backward_solve / solve_cholesky (summation order
differs) and hence solve_spd's refined x; its strategy and kappa must match.
"""
import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import shifted_hilbert, dense_dd

pytestmark = pytest.mark.gpu


def spd_dd(n, seed, shift=None):
    """Symmetric positive definite f128 matrix: B B^T / n + shift I."""
    b = dense_dd(n, n, seed=seed)
    bh = b[..., 0] + b[..., 1]
    a = bh @ bh.T / n + (shift if shift is not None else 1.0) * np.eye(n)
    out = np.zeros((n, n, 2))
    out[..., 0] = a
    out[..., 1] = dense_dd(n, n, seed=seed + 1)[..., 1] * 1e-3
    out[..., 1] = (out[..., 1] + out[..., 1].transpose()) * 0.5 * np.abs(a) * 2.0 ** -50
    return out


def lower(x):
    n = x.shape[0]
    return x * np.tril(np.ones((n, n)))[..., None]


def nwerr(x, ref):
    d = (x[..., 0] - ref[..., 0]) + (x[..., 1] - ref[..., 1])
    return np.linalg.norm(d) / max(np.linalg.norm(ref[..., 0]), 1e-300)


@pytest.mark.parametrize("n", [1, 2, 3, 17, 64, 65, 130, 257])
def test_cholesky_bitexact(gpu, n):
    a = spd_dd(n, seed=n)
    L = gpu.f128_cholesky(a, n)
    ref = O.cholesky(a, n)
    assert np.array_equal(lower(L), lower(ref))
    # strict upper triangle untouched
    iu = np.triu_indices(n, 1)
    assert np.array_equal(L[iu], a[iu])


def test_cholesky_reference_kats(gpu):
    f = lambda v: np.stack([np.asarray(v, float), np.zeros(len(v))], -1)
    L = gpu.f128_cholesky(f([4, 2, 0, 2, 5, 1, 0, 1, 6]).reshape(3, 3, 2), 3)  # linalg.rs:377
    assert np.array_equal(lower(L), lower(O.cholesky(f([4, 2, 0, 2, 5, 1, 0, 1, 6]).reshape(3, 3, 2), 3)))
    n = 200  # linalg.rs:406-418
    i = np.arange(n, dtype=np.float64)
    a = f((1.0 / (np.abs(i[:, None] - i[None, :]) + 1.0)).ravel()).reshape(n, n, 2)
    for d in range(n):
        a[d, d] = O.dd_add(a[d, d], O.dd(2.0))
    assert np.array_equal(lower(gpu.f128_cholesky(a, n)), lower(O.cholesky(a, n)))


@pytest.mark.parametrize("n,nb", [(20, 8), (130, 64), (100, 7), (257, 32), (64, 64)])
def test_cholesky_blocked_bitexact(gpu, n, nb):
    a = spd_dd(n, seed=3 * n + nb)
    L = gpu.f128_cholesky_blocked(a, n, nb)
    ref = O.cholesky_blocked(a, n, nb)
    assert np.array_equal(lower(L), lower(ref))


def test_cholesky_not_spd(gpu):
    n = 70
    a = spd_dd(n, seed=5)
    a[40, 40] = [-1.0, 0.0]
    with pytest.raises(gpu.CholeskyError) as ei:
        gpu.f128_cholesky(a, n)
    with pytest.raises(O.CholeskyError) as eo:
        O.cholesky(a, n)
    assert ei.value.pivot == eo.value.pivot == 40
    assert ei.value.value == eo.value.value
    with pytest.raises(gpu.CholeskyError) as eb:
        gpu.f128_cholesky_blocked(a, n, 16)
    assert eb.value.pivot == 40


@pytest.mark.parametrize("n", [1, 5, 64, 300, 1100])
def test_solves_and_matvec(gpu, n):
    a = spd_dd(n, seed=11 + n)
    L = O.cholesky(a, n)
    b = dense_dd(n, 1, seed=7)[:, 0]
    assert np.array_equal(gpu.f128_forward_solve(L, b, n), O.forward_solve(L, b, n))
    assert np.array_equal(gpu.f128_matvec(a, b, n), O.matvec(a, b, n))
    tol = 4 * n * 2.0 ** -104 * 1e3
    assert nwerr(gpu.f128_backward_solve(L, b, n), O.backward_solve(L, b, n)) <= tol
    assert nwerr(gpu.f128_solve_cholesky(L, b, n), O.solve_cholesky(L, b, n)) <= tol
    assert gpu.f128_cond_estimate(L, n) == O.cond_estimate(L, n)


def test_solve_roundtrip_readme_matrix(gpu):  # linalg.rs:544-563 at n=4 and the n=512 workload
    for n in (4, 512):
        a, b = shifted_hilbert(n)
        L = gpu.f128_cholesky(a, n)
        assert np.array_equal(lower(L), lower(O.cholesky(a, n)))
        x = gpu.f128_solve_cholesky(L, b, n)
        ax = O.matvec(a, x, n)
        r = (ax[:, 0] - b[:, 0]) + (ax[:, 1] - b[:, 1])
        assert np.max(np.abs(r)) < 1e-28


def hilbert(n):
    i = np.arange(n, dtype=np.float64)
    return 1.0 / (i[:, None] + i[None, :] + 1.0)


@pytest.mark.parametrize("case", ["well", "hilbert12", "hilbert13", "shifted200"])
def test_solve_spd_matches_reference(gpu, case):  # solver/src/lib.rs:271-340
    if case == "well":
        n = 10
        a = hilbert(n) + np.eye(n)
        b = np.ones(n)
    elif case == "hilbert12":
        n = 12
        a = hilbert(n)
        b = a.sum(axis=1)
    elif case == "hilbert13":
        n = 13
        a = hilbert(n)
        b = np.ones(n)
    else:
        n = 200
        a = hilbert(n) + 5.0 * np.eye(n)
        b = a.sum(axis=1)
    g = gpu.solve_spd(a, b, n)
    r = O.solve_spd(a, b, n)
    assert g["strategy"] == r["strategy"]
    assert g["kappa"] == r["kappa"]
    if case == "well":
        assert g["residual_norm"] < 1e-12
    if case == "hilbert12":
        assert g["residual_norm"] < 1e-25
    # x differs from the oracle's only through summation order in the
    # backward solves (f64 and f128); both are within kappa * n * u of x*.
    # (Float64 strategy: x is the promoted f64 solution, so the unit is 2^-53.)
    unit = 2.0 ** -50 if g["strategy"] == "Float64" else 2.0 ** -100
    xe = nwerr(g["x"], r["x"])
    assert xe <= max(np.linalg.cond(a), 1.0) * n * unit


def test_solve_spd_f128_hilbert12(gpu):  # solver/src/lib.rs:319-340
    n = 12
    a = np.zeros((n, n, 2))
    a[..., 0] = hilbert(n)
    b = np.zeros((n, 2))
    for i in range(n):
        for j in range(n):
            b[i] = O.dd_add(b[i], O.dd_mul(a[i, j], O.dd(1.0)))
    g = gpu.solve_spd_f128(a, b, n)
    r = O.solve_spd_f128(a, b, n)
    err = np.sqrt(np.sum(((g["x"][:, 0] - 1.0) + g["x"][:, 1]) ** 2))
    assert err < 1e-15 and g["strategy"] == "Float128" and g["kappa"] == r["kappa"]
    assert abs(g["residual_norm"]) < 1e-30


@pytest.mark.parametrize("length", [0, 1, 7, 1023, 1024, 1025, 5000])
def test_dot_bitexact(gpu, length):
    """linalg.rs:7-26: serial below 1024 entries, chunk sums folded above."""
    a = dense_dd(1, max(length, 1), seed=300 + length)[0][:length]
    b = dense_dd(1, max(length, 1), seed=400 + length)[0][:length]
    got = gpu.f128_dot(a, b)
    ref = O.dot(a, b) if length else np.zeros(2)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("rows,cols", [(1, 1), (3, 70), (70, 3), (129, 257), (1000, 17)])
def test_gemv_bitexact(gpu, rows, cols):
    """linalg.rs:29-38: every row summed in column order."""
    a = dense_dd(rows, cols, seed=rows * 7 + cols)
    x = dense_dd(1, cols, seed=cols + 11)[0]
    assert np.array_equal(gpu.f128_gemv(a, rows, cols, x), O.gemv(a, rows, cols, x))


def test_solve_cholesky_dev_matches_host_form(gpu):
    import torch

    n = 300
    a = spd_dd(n, 21)
    L = gpu.f128_cholesky(a, n)
    b = dense_dd(1, n, seed=5)[0]
    x_host = gpu.f128_solve_cholesky(L, b, n)
    dL = torch.from_numpy(np.ascontiguousarray(L)).cuda()
    dx = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    gpu.check(gpu.lib().hp_f128_solve_cholesky_dev(dL.data_ptr(), dx.data_ptr(), n, 0))
    torch.cuda.synchronize()
    assert np.array_equal(dx.cpu().numpy(), x_host)
