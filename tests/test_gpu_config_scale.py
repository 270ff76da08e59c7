"""Parity at the benchmark configurations' own sizes (through the C ABI).

The small-size parity tests elsewhere pin every kernel bit for bit or to the
stated tolerance; this file checks the benchmarked workloads themselves
against f512 / f256 references computed by the oracle and committed as
fixtures (tests/golden/make_*.py):

* f128 GEMM and GEMM_atb at m = n = k = 2048, f256 GEMM at 1024, both
  modes: 4096 sampled entries plus two full rows against the oracle's f512
  dot products; normwise ||C - C*||_F / || |A| |B| ||_F over the sample
  <= 4 k 2^-104 (f128) and 4 k 2^-208 (f256).
* The 4096-system batch (n in [16, 384]): 64 sampled systems (48 spread over
  the sizes, the 16 largest cond_estimate) against mf_cholesky<8> solves:
  ||x - x*|| / ||x*|| <= 1e-25 each.
* Batched Jacobi on overlap matrices of that batch (n up to 128) against the
  oracle's jacobi_eigen (linalg.rs:299-362), at f128 level: eigenvalues within
  1e-26 ||A||, eigenvectors (up to sign) within 1e-24 where the eigenvalue is
  separated from its neighbours by at least 1e-6 ||A||, V V^T = I within
  1e-28 in f128 arithmetic.
* The adjoint at n = 1000: 56 parameters against f256 central differences
  (h = 1e-20), each within 2^-88 of the sum of its terms' magnitudes (the
  contraction -lambda^T dS lambda runs in f128 and cancels: lambda = S^-1 b
  reaches 3e10 while the gradient is ~1e10), and the full gradient against
  the reference-primitive gradient (f128 Cholesky solve, to that solve's own
  accuracy).
"""
import os

import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import (batched_overlap_systems, dd_to_qd, gemm_operands, overlap_spd_problem,
                                     sample_abs_products, sample_index, sampled_error)

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gemm_fixture():
    return np.load(os.path.join(GOLDEN, "gemm_f512_sample.npz"))


@pytest.mark.parametrize("atb", [False, True])
@pytest.mark.parametrize("mode", ["plain", "ozaki"])
def test_f128_gemm_2048_vs_f512(gpu, gemm_fixture, atb, mode):
    s = 2048
    name = "f128_gemm_atb_2048" if atb else "f128_gemm_2048"
    a, b = gemm_operands(s, s, s, seed=0, atb=atb)
    c = gpu.f128_gemm(a, b, s, s, s, gpu.PLAIN if mode == "plain" else gpu.OZAKI, atb)
    idx = sample_index(s, s)
    err, err_rel = sampled_error(c, gemm_fixture[name], sample_abs_products(a, b, idx, atb), idx)
    assert len(idx) >= 4096 + 2 * s
    assert err <= 4 * s * 2.0 ** -104, (name, mode, err, err_rel)
    if mode == "ozaki":  # exact products, one rounding of the 106-bit inputs
        assert err <= 2.0 ** -104, (name, err)


@pytest.mark.parametrize("mode", ["plain", "ozaki"])
def test_f256_gemm_1024_vs_f512(gpu, gemm_fixture, mode):
    s = 1024
    a, b = gemm_operands(s, s, s, seed=0)
    a, b = dd_to_qd(a), dd_to_qd(b)
    c = gpu.f256_gemm(a, b, s, s, s, gpu.PLAIN if mode == "plain" else gpu.OZAKI)
    idx = sample_index(s, s)
    err, err_rel = sampled_error(c, gemm_fixture["f256_gemm_1024"], sample_abs_products(a, b, idx), idx)
    assert err <= 4 * s * 2.0 ** -208, (mode, err, err_rel)


@pytest.fixture(scope="module")
def batch4096():
    return batched_overlap_systems(4096, seed=0)


def test_batched_4096_sample_vs_f512(gpu, batch4096):
    B = batch4096
    fx = np.load(os.path.join(GOLDEN, "batched_4096_sample.npz"))
    x, st, it = gpu.spd_solve_batched(B)
    assert np.all(st == 0), np.nonzero(st)[0][:10]
    off, xo, xs = B["offsets"], fx["x_offsets"], fx["x_star"]
    errs = []
    for t, s in enumerate(fx["index"]):
        xg = x[off[s]:off[s + 1]]
        xr = xs[xo[t]:xo[t + 1]]
        assert len(xg) == len(xr) == fx["n"][t]
        d = (xg[:, 0] - xr[:, 0]) + (xg[:, 1] - xr[:, 1]) - xr[:, 2] - xr[:, 3]
        errs.append(np.linalg.norm(d) / np.linalg.norm(xr[:, 0]))
    errs = np.array(errs)
    assert len(errs) >= 64 and fx["n"].min() == 16 and fx["n"].max() == 384
    assert errs.max() <= 1e-25, (errs.max(), fx["index"][errs.argmax()], fx["n"][errs.argmax()])


def _f64(x):
    return x[..., 0] + x[..., 1]


def _jacobi_cases(B, targets=(16, 40, 64, 96, 112, 128)):
    ns = np.diff(B["offsets"])
    picks = []
    for t in targets:
        cand = np.nonzero(ns == t)[0]
        if len(cand) == 0:
            cand = np.nonzero(ns == ns[ns <= t].max())[0]
        picks.append(int(cand[0]))
    return picks


def test_batched_jacobi_f128_level_vs_oracle(gpu, batch4096):
    import torch

    B = batch4096
    picks = _jacobi_cases(B)
    off = B["offsets"]
    mats, ns = [], []
    for s in picks:
        o, e = off[s], off[s + 1]
        mats.append(O.overlap_norm_dd(B["centers"][o:e], B["alpha"][o:e]))
        ns.append(e - o)
    noff = np.zeros(len(picks) + 1, dtype=np.int64)
    noff[1:] = np.cumsum(ns)
    A = torch.from_numpy(np.concatenate([m.reshape(-1, 2) for m in mats])).cuda()
    ev = torch.empty((int(noff[-1]), 2), dtype=torch.float64, device="cuda")
    vec = torch.empty_like(A)
    sw = torch.zeros(len(picks), dtype=torch.int32, device="cuda")
    st = torch.zeros(len(picks), dtype=torch.int32, device="cuda")
    gpu.check(gpu.lib().hp_f128_jacobi_eigen_batched_dev(len(picks), noff.ctypes.data, A.data_ptr(), 200,
                                                         ev.data_ptr(), vec.data_ptr(), sw.data_ptr(),
                                                         st.data_ptr(), 0))
    torch.cuda.synchronize()
    assert int(st.abs().sum()) == 0
    evh, vh = ev.cpu().numpy(), vec.cpu().numpy()
    m0 = 0
    for t, (n, S) in enumerate(zip(ns, mats)):
        lam = evh[noff[t]:noff[t + 1]]
        V = vh[m0:m0 + n * n].reshape(n, n, 2)
        m0 += n * n
        lr, Vr, _ = O.jacobi_eigen(S, n, 200)
        norm = np.abs(_f64(lr)).max()
        og, orr = np.argsort(_f64(lam)), np.argsort(_f64(lr))
        dl = (lam[og, 0] - lr[orr, 0]) + (lam[og, 1] - lr[orr, 1])
        assert np.abs(dl).max() <= 1e-26 * norm, (n, np.abs(dl).max() / norm)
        # eigenvectors (rows), up to sign, where the eigenvalue is separated
        ls = _f64(lr)[orr]
        gap = np.full(n, np.inf)
        if n > 1:
            dif = np.diff(ls)
            gap[:-1] = dif
            gap[1:] = np.minimum(gap[1:], dif)
        checked = 0
        for q in range(n):
            if gap[q] < 1e-6 * norm:
                continue
            vg, vr = V[og[q]], Vr[orr[q]]
            sg = 1.0 if np.dot(_f64(vg), _f64(vr)) > 0 else -1.0
            dv = (sg * vg[:, 0] - vr[:, 0]) + (sg * vg[:, 1] - vr[:, 1])
            assert np.abs(dv).max() <= 1e-24, (n, q, np.abs(dv).max(), gap[q] / norm)
            checked += 1
        assert checked >= n // 2, (n, checked)
        # V V^T = I in f128 arithmetic (the oracle's gemm with B = V^T)
        VVt = O.gemm(V, np.ascontiguousarray(V.transpose(1, 0, 2)), n, n, n)
        I = np.zeros((n, n, 2))
        I[np.arange(n), np.arange(n), 0] = 1.0
        dI = (VVt[..., 0] - I[..., 0]) + VVt[..., 1]
        assert np.abs(dI).max() <= 1e-28, (n, np.abs(dI).max())


ADJ = (5, 5, 10)


@pytest.fixture(scope="module")
def adjoint_problem():
    cen, alpha, b = overlap_spd_problem(*ADJ, seed=0)
    n = len(alpha)
    return cen, alpha, b, np.arange(n, dtype=np.int32) // 4, n // 4


def _term_scales(cen, alpha, lam, centres, funcs):
    """sum over v of |each term| of the f128 contraction behind each checked
    component (float64): g_R(c) = sum_{u in c} 4 l_u sum_v l_v S_uv p_uv (R_u - R_v),
    g_lna(u) = -2 l_u sum_v l_v S_uv f_uv. The contraction is accurate to a
    small multiple of 2^-104 times this sum, which is much larger than the
    component itself when lambda = S^-1 b is large (kappa(S) ~ 1e13 here)."""
    S = O.overlap_norm_dd(cen, alpha)[..., 0]
    l = np.abs(lam[:, 0])
    a = alpha
    p = a[:, None] * a[None, :] / (a[:, None] + a[None, :])
    W = l[:, None] * l[None, :] * np.abs(S)
    np.fill_diagonal(W, 0.0)
    sR = []
    for c in centres:
        us = np.arange(4 * c, 4 * c + 4)
        d = np.abs(cen[us][:, None, :] - cen[None, :, :])
        sR.append((4 * W[us][:, :, None] * p[us][:, :, None] * d).sum(axis=(0, 1)))
    r2 = ((cen[:, None, :] - cen[None, :, :]) ** 2).sum(-1)
    f = np.abs(0.75 * (a[None, :] - a[:, None]) / (a[:, None] + a[None, :])) + \
        r2 * a[:, None] * a[None, :] ** 2 / (a[:, None] + a[None, :]) ** 2
    sa = [(2 * W[u] * f[u]).sum() for u in funcs]
    return np.array(sR), np.array(sa)


@pytest.mark.parametrize("mode", [0, 1])
def test_adjoint_1000_vs_f256_finite_differences(gpu, adjoint_problem, mode):
    """56 components against f256 central differences (converged: h = 1e-16,
    1e-20 and 1e-24 agree to the stored digits). Each component must be
    within 2^-88 of the sum of the magnitudes of its terms, and within 1e-20
    of the largest component. The host restatement of the same computation
    (oracle.adjoint_f128_refined: lambda refined to 1e-28, f128 contraction)
    reaches 2^-90.8 of the term sum at worst and 1e-23 of the largest
    component: lambda's own relative error and the f128 rounding of each term
    are both multiplied by the cancellation."""
    cen, alpha, b, co, nc = adjoint_problem
    loss, gR, ga, info = gpu.overlap_adjoint(cen, alpha, b, co, nc, mode=mode)
    assert info["converged"]
    fx = np.load(os.path.join(GOLDEN, "adjoint_fd_1000.npz"))
    lam, _ = O.spd_solve_refined(O.overlap_norm_dd(cen, alpha), b, len(alpha))
    sR, sa = _term_scales(cen, alpha, lam, fx["centres"], fx["funcs"])
    gmax = max(np.abs(gR[..., 0]).max(), np.abs(ga[..., 0]).max())
    worst, checked = 0.0, 0
    for ci, c in enumerate(fx["centres"]):
        for comp in range(3):
            fd, g = fx["gR"][ci, comp], gR[c, comp]
            err = abs(((g[0] - fd[0]) + (g[1] - fd[1])) - fd[2] - fd[3])
            assert err <= 2.0 ** -88 * sR[ci, comp], (c, comp, err, sR[ci, comp])
            worst = max(worst, err)
            checked += 1
    for qi, u in enumerate(fx["funcs"]):
        fd, g = fx["ga"][qi], ga[u]
        err = abs(((g[0] - fd[0]) + (g[1] - fd[1])) - fd[2] - fd[3])
        assert err <= 2.0 ** -88 * sa[qi], (u, err, sa[qi])
        worst = max(worst, err)
        checked += 1
    assert checked >= 32
    assert worst <= 1e-20 * gmax, worst / gmax


def test_adjoint_1000_vs_reference_primitives(gpu, adjoint_problem):
    cen, alpha, b, co, nc = adjoint_problem
    loss, gR, ga, info = gpu.overlap_adjoint(cen, alpha, b, co, nc)
    lo, gRo, gao = O.adjoint_f128(cen, alpha, b, co, nc)
    # the reference-primitive gradient solves with an unrefined f128 Cholesky,
    # accurate to about kappa(S) 2^-104 relative; the GPU gradient is refined
    rel = lambda x, y: np.abs((x[..., 0] - y[..., 0]) + (x[..., 1] - y[..., 1])).max() / np.abs(y[..., 0]).max()
    assert rel(gR, gRo) < 1e-12 and rel(ga, gao) < 1e-12, (rel(gR, gRo), rel(ga, gao))
    assert abs((loss[0] - lo[0]) + (loss[1] - lo[1])) < 1e-12 * abs(lo[0])
