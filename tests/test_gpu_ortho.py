"""GPU canonical orthogonalisation (hp_canonical_orthogonalize) against the
oracle's canonical_orthogonalize (the reference's crates/solver/src/ortho.rs:
147-183). The GPU takes its eigenpairs from the parallel round-robin Jacobi,
so X agrees with the oracle's column by column up to sign and f128 rounding:
same kept count, max | |X| - |X_ref| | <= 1e-22 max |X_ref| (well separated
eigenvalues) and X^T S X = I to 1e-24.
"""
import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import overlap_lattice

pytestmark = pytest.mark.gpu


def overlap_f128(nx, ny, nz, seed):
    cen, alpha = overlap_lattice(nx, ny, nz, seed=seed)
    n = len(alpha)
    return np.ascontiguousarray(O.overlap_norm_dd(cen, alpha)), n


@pytest.mark.parametrize("shape,threshold", [((1, 2, 2), 1e-6), ((2, 2, 3), 1e-4), ((2, 3, 4), 1e-3)])
def test_canonical_orthogonalize(gpu, shape, threshold):
    s, n = overlap_f128(*shape, seed=sum(shape))
    x = gpu.canonical_orthogonalize(s, n, threshold)
    xr = O.canonical_orthogonalize(s, n, threshold)
    assert x.shape == xr.shape
    m = x.shape[1]
    assert 0 < m <= n
    xa, xra = x[..., 0] + x[..., 1], xr[..., 0] + xr[..., 1]
    assert np.max(np.abs(np.abs(xa) - np.abs(xra))) <= 1e-22 * np.max(np.abs(xra))
    xtsx = O.gemm(O.gemm(np.ascontiguousarray(np.swapaxes(x, 0, 1)), s, m, n, n), x, m, m, n)
    err = np.max(np.abs((xtsx[..., 0] + xtsx[..., 1]) - np.eye(m)))
    assert err <= 1e-24, err


def _gen_eigen_residual(f, s, ev, c, n, m):
    """max over k, i of |(F c_k)_i - eps_k (S c_k)_i| relative to |F| |c_k|,
    evaluated with the oracle's f128 GEMM."""
    fc = O.gemm(f, c, n, m, n)
    sc = O.gemm(s, c, n, m, n)
    fa = np.abs(f[..., 0]) @ np.abs(c[..., 0])
    worst = 0.0
    for k in range(m):
        for i in range(n):
            d = O.dd_sub(fc[i, k], O.dd_mul(ev[k], sc[i, k]))
            worst = max(worst, abs(d[0] + d[1]) / max(fa[i, k], 1e-300))
    return worst


@pytest.mark.parametrize("case", ["2x2", "identity3"])
def test_solve_gen_eigen_reference_cases(gpu, case):
    """The reference's own tests (ortho.rs:303-377): F c = eps S c to 1e-25,
    eigenvalues ascending, against the oracle's eigenvalues."""
    if case == "2x2":
        n = 2
        f = np.zeros((n, n, 2)); f[..., 0] = [[2.0, 1.0], [1.0, 3.0]]
        s = np.zeros((n, n, 2)); s[..., 0] = [[1.0, 0.2], [0.2, 1.0]]
    else:
        n = 3
        f = np.zeros((n, n, 2)); f[..., 0] = [[3.0, 1.0, 0.0], [1.0, 2.0, 1.0], [0.0, 1.0, 4.0]]
        s = np.zeros((n, n, 2)); s[..., 0] = np.eye(n)
    ev, c, m = gpu.solve_gen_eigen(f, s, n, 1e-8)
    evr, cr, mr = O.solve_gen_eigen(f, s, n, 1e-8)
    assert m == mr == n
    assert np.all(np.diff(ev[:, 0] + ev[:, 1]) > 0)
    assert np.max(np.abs((ev[:, 0] - evr[:, 0]) + (ev[:, 1] - evr[:, 1]))) <= 1e-30 * np.max(np.abs(evr[:, 0]))
    assert _gen_eigen_residual(f, s, ev, c, n, m) < 1e-25


@pytest.mark.parametrize("shape,threshold", [((1, 2, 2), 1e-6), ((2, 2, 3), 1e-4), ((2, 3, 4), 1e-3)])
def test_solve_gen_eigen_overlap(gpu, shape, threshold):
    """Roothaan-Hall form on an overlap matrix with a symmetric F: same basis
    size and eigenvalues as the oracle (f128 rounding), each eigenvector
    column equal up to sign, and, in the retained basis (the problem is
    projected onto span X when eigenvalues of S are dropped),
    C^T F C = diag(eps) and C^T S C = I."""
    s, n = overlap_f128(*shape, seed=sum(shape) + 7)
    rng = np.random.default_rng(n)
    fm = rng.standard_normal((n, n))
    fm = (fm + fm.T) / 2
    f = np.zeros((n, n, 2))
    f[..., 0] = fm
    ev, c, m = gpu.solve_gen_eigen(f, s, n, threshold)
    evr, cr, mr = O.solve_gen_eigen(f, s, n, threshold)
    assert m == mr and 0 < m <= n
    e, er = ev[:, 0] + ev[:, 1], evr[:, 0] + evr[:, 1]
    assert np.max(np.abs(e - er)) <= 1e-24 * np.max(np.abs(er)), np.max(np.abs(e - er))
    ca, cra = c[..., 0] + c[..., 1], cr[..., 0] + cr[..., 1]
    assert np.max(np.abs(np.abs(ca) - np.abs(cra))) <= 1e-20 * np.max(np.abs(cra))
    ct = np.ascontiguousarray(np.swapaxes(c, 0, 1))
    ctfc = O.gemm(O.gemm(ct, f, m, n, n), c, m, m, n)
    assert np.max(np.abs((ctfc[..., 0] + ctfc[..., 1]) - np.diag(e))) <= 1e-24 * np.max(np.abs(e))
    ctsc = O.gemm(O.gemm(ct, s, m, n, n), c, m, m, n)
    assert np.max(np.abs((ctsc[..., 0] + ctsc[..., 1]) - np.eye(m))) <= 1e-24
