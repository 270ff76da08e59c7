"""f512 (MultiFloat<8>) GEMM, Cholesky and solve on the GPU against the oracle.

hp_f512_gemm[_atb] and hp_f512_cholesky must be bit-identical to the oracle's
mf_gemm::<8> / mf_cholesky::<8> (crates/quad/src/multifloat/linalg.rs:39-139);
hp_f512_cholesky_solve's forward sweep is bit-identical and its backward
sweep reorders each row's subtractions, so x agrees to f512 accuracy. On the
overlap SPD workloads the GPU's f512 factor + solve reproduces the committed
oracle solutions (tests/golden/overlap_*.npz, computed by the oracle's
mf_cholesky<8> + mf_cholesky_solve<8>) to the 4 limbs they keep.
"""
import os

import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import dense_dd

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def to_mf(x, N, seed):
    """f128 entries (..., 2) widened to N renormalised limbs with random low limbs."""
    rng = np.random.default_rng(seed)
    flat = x.reshape(-1, 2)
    out = np.zeros((flat.shape[0], N))
    out[:, :2] = flat
    for t in range(2, N):
        out[:, t] = out[:, t - 1] * 2.0 ** -53 * rng.uniform(-1, 1, flat.shape[0])
    for i in range(out.shape[0]):
        O.lib().or_mf_renormalize(N, O._p(out[i]))
    return out.reshape(x.shape[:-1] + (N,))


@pytest.mark.parametrize("atb", [False, True])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (3, 5, 7), (17, 13, 29), (40, 31, 37)])
def test_f512_gemm_bitexact(gpu, m, n, k, atb):
    a = to_mf(dense_dd(k, m, seed=m + k) if atb else dense_dd(m, k, seed=m + k), 8, 1)
    b = to_mf(dense_dd(k, n, seed=n + k + 1), 8, 2)
    assert np.array_equal(gpu.f512_gemm(a, b, m, n, k, atb), O.mf_gemm(8, a, b, m, n, k, atb=atb))


def spd8(n, seed):
    b = dense_dd(n, n, seed=seed)
    bh = b[..., 0] + b[..., 1]
    a = np.zeros((n, n, 2))
    a[..., 0] = bh @ bh.T / n + np.eye(n)
    a8 = to_mf(a, 8, seed)
    return (a8 + a8.transpose(1, 0, 2)) / 2.0


@pytest.mark.parametrize("n", [1, 2, 3, 17, 40, 65])
def test_f512_cholesky_bitexact(gpu, n):
    a = spd8(n, 300 + n)
    got = gpu.f512_cholesky(a, n)
    ref = O.mf_cholesky(8, a, n)
    low = np.tril(np.ones((n, n), dtype=bool))
    assert np.array_equal(got[low], ref[low])
    assert np.array_equal(got[~low], a[~low])  # strict upper triangle untouched


def test_f512_cholesky_not_spd(gpu):
    """A first limb <= 0 on the diagonal (multifloat/linalg.rs:105-107) fails
    at the same pivot as the oracle."""
    a = spd8(5, 9)
    a[3, 3] = 0.0
    a[3, :3] = a[:3, 3] = 10.0
    with pytest.raises(gpu.CholeskyError) as ei:
        gpu.f512_cholesky(a, 5)
    assert ei.value.pivot == 3
    assert O.lib().or_mf_cholesky(8, O._p(np.ascontiguousarray(a.copy())), 5) != 0


def rel8(x, ref):
    d = np.zeros(len(x))
    for t in range(8):
        d = d + (x[:, t] - ref[:, t])
    return np.linalg.norm(d) / np.linalg.norm(ref[:, 0])


@pytest.mark.parametrize("n", [1, 7, 64, 130])
def test_f512_solve_vs_oracle(gpu, n):
    a = spd8(n, 500 + n)
    L = O.mf_cholesky(8, a, n)
    b = to_mf(dense_dd(1, n, seed=n)[0], 8, 3)
    assert rel8(gpu.f512_cholesky_solve(L, b, n), O.mf_cholesky_solve(8, L, b, n)) <= 1e-120


@pytest.mark.parametrize("name", ["overlap_2x2x2", "overlap_3x4x5"])
def test_f512_reproduces_overlap_fixtures(gpu, name):
    from quadprec_b200.workloads import overlap_spd_problem

    lat = {"overlap_2x2x2": (2, 2, 2), "overlap_3x4x5": (3, 4, 5)}[name]
    cen, alpha, b = overlap_spd_problem(*lat, seed=0)
    n = len(alpha)
    S8 = np.zeros((n, n, 8))
    S8[..., :2] = gpu.overlap_norm_dd(cen, alpha)
    b8 = np.zeros((n, 8))
    b8[:, 0] = b
    x = gpu.f512_cholesky_solve(gpu.f512_cholesky(S8, n), b8, n)
    xs = np.load(os.path.join(GOLDEN, name + ".npz"))["x_star"]
    d = (x[:, 0] - xs[:, 0]) + (x[:, 1] - xs[:, 1]) + (x[:, 2] - xs[:, 2]) + (x[:, 3] - xs[:, 3]) + x[:, 4]
    assert np.linalg.norm(d) / np.linalg.norm(xs[:, 0]) <= 1e-60
