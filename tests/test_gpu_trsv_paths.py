"""The blocked f128 triangular solves of the refinement loop against the oracle.

hp_spd_solve_refined with max_iter = 0 in HP_MODE_PLAIN returns the first
solve x = L^-T L^-1 b, where L is the reference-order f128 Cholesky factor and
both sweeps run the wavefront kernel of trsv_blocked.cu (64-row blocks,
precomputed diagonal-block inverses, exchange buffers polled for sentinels).
It must agree with the oracle's solve_cholesky (linalg.rs:99-126 order) to
f128 accuracy on a well-conditioned system, including ragged last blocks, a
single row and a single block.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def system(n):
    rng = np.random.default_rng(7000 + n)
    B = rng.standard_normal((n, n))
    A = B @ B.T / n + np.eye(n)
    A = (A + A.T) / 2
    a = np.zeros((n, n, 2))
    a[..., 0] = A
    return a, rng.standard_normal(n)


def oracle_solve(a, b, n):
    L = O.cholesky(a, n)
    bb = np.zeros((n, 2))
    bb[:, 0] = b
    return O.solve_cholesky(L, bb, n)


def rel(x, xs):
    d = (x[:, 0] - xs[:, 0]) + (x[:, 1] - xs[:, 1])
    return np.linalg.norm(d) / np.linalg.norm(xs[:, 0])


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 130, 1000])
def test_wavefront_solve_matches_oracle(gpu, n):
    a, b = system(n)
    x, info = gpu.spd_solve_refined(a, b, n, mode=0, max_iter=0)
    assert rel(x, oracle_solve(a, b, n)) <= 1e-28
