"""GPU adjoint of overlap assembly + solve, checked against f256 central
finite differences (h = 1e-20) and the reference-primitive gradient."""
import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import overlap_lattice, normal

pytestmark = pytest.mark.gpu


def problem(nx, ny, nz, seed=0):
    cen, alpha = overlap_lattice(nx, ny, nz, seed=seed)
    n = len(alpha)
    b = normal(n, seed, offset=10 ** 9)
    center_of = np.arange(n) // 4
    return cen, alpha, b, center_of, n // 4


def f64_to_f256(x):
    out = np.zeros(np.shape(x) + (4,))
    out[..., 0] = x
    return out


def two_prod(a, b):
    p = a * b
    # exact error of the product (Dekker split), numpy has no fma
    c = 134217729.0
    def split(v):
        t = c * v
        hi = t - (t - v)
        return hi, v - hi
    ah, al = split(a)
    bh, bl = split(b)
    e = ((ah * bh - p) + ah * bl + al * bh) + al * bl
    return p, e


def fd_param(cen, alpha, b, kind, idx, comp, h=1e-20):
    """f256 central difference of L wrt one parameter."""
    vals = []
    for sgn in (1.0, -1.0):
        c4 = f64_to_f256(cen)
        a4 = f64_to_f256(alpha)
        if kind == "R":  # all basis functions on centre idx move together
            for u in range(4 * idx, 4 * idx + 4):
                c4[u, comp, 1] = sgn * h
        else:  # alpha_u (1 +- h): ln alpha moves by ln(1 +- h)
            p, e = two_prod(alpha[idx], sgn * h)
            a4[idx, 1], a4[idx, 2] = p, e
        vals.append(O.loss_f256(c4, a4, b))
    d = O.mf_op("add", 4, vals[0], -vals[1])
    return O.mf_op("div", 4, d, f64_to_f256(2 * h))  # f256 quotient


@pytest.mark.parametrize("mode", [0, 1])
def test_adjoint_vs_f256_finite_differences(gpu, mode):
    cen, alpha, b, co, nc = problem(2, 2, 2)
    loss, gR, ga, info = gpu.overlap_adjoint(cen, alpha, b, co, nc, mode=mode)
    gmax = max(np.abs(gR[..., 0]).max(), np.abs(ga[..., 0]).max())
    for (kind, idx, comp) in [("R", 0, 0), ("R", 3, 2), ("R", 7, 1), ("a", 0, 0), ("a", 13, 0), ("a", 31, 0)]:
        fd = fd_param(cen, alpha, b, kind, idx, comp)
        g = gR[idx, comp] if kind == "R" else ga[idx]
        err = abs(((g[0] - fd[0]) + (g[1] - fd[1])) - fd[2])
        assert err <= 1e-25 * gmax, (kind, idx, comp, g, fd, err)


def test_adjoint_vs_reference_primitives(gpu):
    cen, alpha, b, co, nc = problem(3, 3, 3)
    loss, gR, ga, info = gpu.overlap_adjoint(cen, alpha, b, co, nc)
    lo, gRo, gao = O.adjoint_f128(cen, alpha, b, co, nc)
    # the reference-primitive gradient uses an f128-only solve: agreement to
    # its own accuracy (kappa * 2^-104 relative)
    rel = lambda x, y: np.abs((x[..., 0] - y[..., 0]) + (x[..., 1] - y[..., 1])).max() / np.abs(y[..., 0]).max()
    assert rel(gR, gRo) < 1e-12 and rel(ga, gao) < 1e-12
    assert abs((loss[0] - lo[0]) + (loss[1] - lo[1])) < 1e-12 * abs(lo[0])
