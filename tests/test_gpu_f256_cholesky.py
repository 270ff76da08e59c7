"""GPU parity for the f256 (MultiFloat<4>) Cholesky and solve (C ABI).

hp_f256_cholesky must equal the oracle's mf_cholesky::<4> (the reference's
crates/quad/src/multifloat/linalg.rs:88-139) bit for bit on the lower
triangle and leave the upper triangle untouched. hp_f256_cholesky_solve
(linalg.rs:141-172) is compared with the oracle's solve within
||x - x_ref|| <= 1e-55 ||x_ref||: its backward sweep orders each row's
subtractions differently (f256 rounding 2^-208 per operation).
"""
import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import uniform

pytestmark = pytest.mark.gpu


def f256_spd(n, seed):
    """Symmetric, diagonally dominant (n, n, 4) matrix with four
    non-overlapping limbs per entry (|x_{k+1}| < ulp(x_k) / 2)."""
    u = uniform(n * n * 4, seed=seed).reshape(n, n, 4)
    a = np.zeros((n, n, 4))
    a[..., 0] = 2.0 * u[..., 0] - 1.0
    for k in range(1, 4):
        a[..., k] = a[..., k - 1] * 2.0 ** -54 * (2.0 * u[..., k] - 1.0)
    a = np.where(np.tril(np.ones((n, n), bool))[..., None], a, np.swapaxes(a, 0, 1))
    for i in range(n):
        a[i, i, 0] = n + 1.0 + abs(a[i, i, 0])
    return a


@pytest.mark.parametrize("n", [1, 2, 5, 31, 33, 64, 65, 130])
def test_f256_cholesky_bitexact(gpu, n):
    a = f256_spd(n, seed=1000 + n)
    got = gpu.f256_cholesky(a, n)
    ref = O.mf_cholesky(4, a, n)
    low = np.tril(np.ones((n, n), bool))
    assert np.array_equal(got[low], ref[low])
    assert np.array_equal(got[~low], a[~low])  # upper triangle untouched


def test_f256_cholesky_not_spd(gpu):
    n = 40
    a = f256_spd(n, seed=7)
    a[23, 23] = (-1.0, 0.0, 0.0, 0.0)
    with pytest.raises(gpu.CholeskyError) as ei:
        gpu.f256_cholesky(a, n)
    assert ei.value.pivot == 23
    with pytest.raises(RuntimeError):
        O.mf_cholesky(4, a, n)


@pytest.mark.parametrize("n", [1, 3, 40, 97])
def test_f256_cholesky_solve(gpu, n):
    a = f256_spd(n, seed=77 + n)
    l = O.mf_cholesky(4, a, n)
    u = uniform(2 * n, seed=5 + n).reshape(2, n)
    b = np.zeros((n, 4))
    b[:, 0] = 2.0 * u[0] - 1.0
    b[:, 1] = b[:, 0] * 2.0 ** -54 * (2.0 * u[1] - 1.0)
    x = gpu.f256_cholesky_solve(l, b, n)
    xr = O.mf_cholesky_solve(4, l, b, n)
    d = (x[:, 0] - xr[:, 0]) + (x[:, 1] - xr[:, 1]) + (x[:, 2] - xr[:, 2]) + (x[:, 3] - xr[:, 3])
    assert np.linalg.norm(d) <= 1e-55 * np.linalg.norm(xr[:, 0])


@pytest.mark.parametrize("n,m", [(1, 1), (3, 7), (33, 130), (200, 65)])
def test_f256_gemv_bitexact(gpu, n, m):
    """hp_f256_gemv / hp_f256_dot equal mf_gemv::<4> / mf_dot::<4> bit for bit."""
    u = uniform(n * m * 4 + m * 4, seed=900 + n + m)
    a = np.zeros((n, m, 4))
    a[..., 0] = 2.0 * u[: n * m].reshape(n, m) - 1.0
    for k in range(1, 4):
        a[..., k] = a[..., k - 1] * 2.0 ** -54 * (2.0 * u[k * n * m : (k + 1) * n * m].reshape(n, m) - 1.0)
    x = np.zeros((m, 4))
    x[:, 0] = 2.0 * u[4 * n * m : 4 * n * m + m] - 1.0
    x[:, 1] = x[:, 0] * 2.0 ** -54
    assert np.array_equal(gpu.f256_gemv(a, x, n, m), O.mf_gemv(4, a, x, n, m))
    assert np.array_equal(gpu.f256_dot(a[0], x), O.mf_gemv(4, a[:1], x, 1, m)[0])
