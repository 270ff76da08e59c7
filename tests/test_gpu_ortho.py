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
