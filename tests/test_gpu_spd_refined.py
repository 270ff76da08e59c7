"""GPU SPD solves of the overlap workloads to <= 1e-25 against the f512 oracle.

The problem matrix is the f128 overlap matrix of normalised s Gaussians on a
jittered lattice (bit-identical between GPU and oracle); x* comes from the
oracle's MultiFloat<8> Cholesky solve (tests/golden/make_overlap_fixtures.py).
Both modes must reach the target: HP_MODE_PLAIN (the reference's f128
cholesky + f256 residual refinement) and HP_MODE_OZAKI (residue-domain
Cholesky on the int8 tensor cores + accurate residual refinement).
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import overlap_spd_problem

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"fixture {name} not generated")
    z = np.load(path)
    return z["x_star"], z["b"], json.loads(str(z["meta"]))


def rel_err(x, xs):
    d = (xs[:, 0] - x[:, 0]) + (xs[:, 1] - x[:, 1]) + xs[:, 2] + xs[:, 3]
    return np.linalg.norm(d) / np.linalg.norm(xs[:, 0])


@pytest.mark.parametrize("name", ["overlap_2x2x2", "overlap_3x4x5", "overlap_5x10x10"])
@pytest.mark.parametrize("mode", [0, 1])
def test_overlap_solve_1e25(gpu, name, mode):
    xs, b_fix, meta = load(name)
    cen, alpha, b = overlap_spd_problem(*meta["lattice"], seed=meta["seed"])
    assert np.array_equal(b, b_fix), "workload generator drifted from the fixture"
    S = gpu.overlap_norm_dd(cen, alpha)
    n = len(alpha)
    x, info = gpu.spd_solve_refined(S, b, n, mode=mode)
    assert info["converged"] == 1, info
    err = rel_err(x, xs)
    assert err <= 1e-25, (err, info)


def test_refined_not_spd(gpu):
    n = 40
    a = np.zeros((n, n, 2))
    a[..., 0] = np.eye(n)
    a[17, 17, 0] = -2.0
    for mode in (0, 1):
        with pytest.raises(gpu.HPError) as ei:
            gpu.spd_solve_refined(a, np.ones(n), n, mode=mode)
        assert ei.value.code == gpu.HP_ERR_NOT_SPD
        assert "pivot 17" in str(ei.value), (mode, str(ei.value))


def test_refined_small_hilbert_exact(gpu):
    """kappa(H_12) ~ 1e16: both modes reproduce the f256 oracle solve to 1e-25."""
    n = 12
    i = np.arange(n, dtype=np.float64)
    a = np.zeros((n, n, 2))
    for r in range(n):
        for c in range(n):
            a[r, c] = O.dd_div(O.dd(1.0), O.dd(float(r + c + 1)))
    b = np.ones(n)
    a4 = np.zeros((n, n, 4))
    a4[..., :2] = a
    L4 = O.mf_cholesky(4, a4, n)
    b4 = np.zeros((n, 4))
    b4[:, 0] = b
    xs = O.mf_cholesky_solve(4, L4, b4, n)
    for mode in (0, 1):
        x, info = gpu.spd_solve_refined(a, b, n, mode=mode)
        assert rel_err(x, xs) <= 1e-25


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 130])
def test_refined_ragged_sizes(gpu, n):
    """Partial last blocks of the wavefront solves (64-row blocks) and of the
    residue-domain panels: both modes leave a residual |b - A x| below 1e-30
    |A| |x| row by row, computed exactly in rationals."""
    from fractions import Fraction as F

    rng = np.random.default_rng(1000 + n)
    B = rng.standard_normal((n, n))
    A = B @ B.T / n + np.eye(n)
    A = (A + A.T) / 2  # exactly symmetric
    a = np.zeros((n, n, 2))
    a[..., 0] = A
    b = rng.standard_normal(n)
    for mode in (0, 1):
        x, info = gpu.spd_solve_refined(a, b, n, mode=mode)
        assert info["converged"] == 1, (mode, info)
        xs = [F(float(x[i, 0])) + F(float(x[i, 1])) for i in range(n)]
        worst = 0
        for i in range(n):
            row = [F(float(A[i, j])) for j in range(n)]
            r = F(float(b[i])) - sum(row[j] * xs[j] for j in range(n))
            scale = sum(abs(row[j]) * abs(xs[j]) for j in range(n))
            worst = max(worst, abs(r) / scale)
        assert worst <= F(1, 10**30), (mode, float(worst))
