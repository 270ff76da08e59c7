"""CPU oracle for the extended-precision linear-algebra path.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the timed CPU
baseline in ``bench.py``. It is a C++ restatement of hyperprec's Rust code
(m0at/quadprec: crates/quad/src/dd.rs, linalg.rs, multifloat/*.rs,
crates/solver/src/lib.rs, ortho.rs, crates/overlap/src/*.rs), compiled from
``hp_oracle.cpp`` by ``Makefile``. The product (``quadprec_b200``) never
imports this package.

Arrays follow the reference's memory layout: an f128 value is two float64
(hi, lo); a MultiFloat<N> value is N float64, most significant first; matrices
are row-major with no padding. Python-side arrays are numpy float64 with a
trailing limb axis, e.g. an n x n f128 matrix has shape (n, n, 2).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libhp_oracle.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_sz = ctypes.c_size_t


def build() -> str:
    """Compile libhp_oracle.so with the committed Makefile (needs g++)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        sigs = {
            "or_num_threads": ([], ctypes.c_int),
            "or_set_num_threads": ([ctypes.c_int], None),
            "or_dd_add": ([_d, _d, _d], None),
            "or_dd_sub": ([_d, _d, _d], None),
            "or_dd_mul": ([_d, _d, _d], None),
            "or_dd_div": ([_d, _d, _d], None),
            "or_dd_sqrt": ([_d, _d], None),
            "or_dd_recip": ([_d, _d], None),
            "or_dd_exp": ([_d, _d], None),
            "or_dd_ln": ([_d, _d], None),
            "or_mf_add": ([ctypes.c_int, _d, _d, _d], ctypes.c_int),
            "or_mf_mul": ([ctypes.c_int, _d, _d, _d], ctypes.c_int),
            "or_mf_div": ([ctypes.c_int, _d, _d, _d], ctypes.c_int),
            "or_mf_sqrt": ([ctypes.c_int, _d, _d], ctypes.c_int),
            "or_mf_exp": ([ctypes.c_int, _d, _d], ctypes.c_int),
            "or_mf_renormalize": ([ctypes.c_int, _d], ctypes.c_int),
            "or_f128_gemm_rows": ([_d, _d, _d, _sz, _sz, _sz, ctypes.c_int, _sz, _sz], None),
            "or_f128_gemm": ([_d, _d, _d, _sz, _sz, _sz], None),
            "or_f128_gemm_atb": ([_d, _d, _d, _sz, _sz, _sz], None),
            "or_f128_gemm_entries": ([_d, _d, _d, _sz, _sz, _sz, ctypes.c_int, _i64, _sz], None),
            "or_f128_dot": ([_d, _d, _sz, _d], None),
            "or_f128_gemv": ([_d, _sz, _sz, _d, _d], None),
            "or_f128_matvec": ([_d, _d, _d, _sz], None),
            "or_f128_cholesky": ([_d, _sz, _i64, _d], ctypes.c_int),
            "or_f128_cholesky_blocked": ([_d, _sz, _sz, _i64, _d], ctypes.c_int),
            "or_f128_forward_solve": ([_d, _d, _d, _sz], None),
            "or_f128_backward_solve": ([_d, _d, _d, _sz], None),
            "or_f128_solve_cholesky": ([_d, _d, _d, _sz], None),
            "or_f128_cond_estimate": ([_d, _sz], ctypes.c_double),
            "or_f128_jacobi_eigen": ([_d, _sz, _sz, _d, _d, ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
            "or_mf_gemm_rows": ([ctypes.c_int, _d, _d, _d, _sz, _sz, _sz, ctypes.c_int, _sz, _sz], ctypes.c_int),
            "or_mf_gemm": ([ctypes.c_int, _d, _d, _d, _sz, _sz, _sz], ctypes.c_int),
            "or_mf_gemm_atb": ([ctypes.c_int, _d, _d, _d, _sz, _sz, _sz], ctypes.c_int),
            "or_mf_gemm_entries": ([ctypes.c_int, _d, _d, _d, _sz, _sz, _sz, ctypes.c_int, _i64, _sz], ctypes.c_int),
            "or_mf_gemv": ([ctypes.c_int, _d, _d, _d, _sz, _sz], ctypes.c_int),
            "or_mf_cholesky": ([ctypes.c_int, _d, _sz], ctypes.c_int),
            "or_mf_cholesky_solve": ([ctypes.c_int, _d, _d, _d, _sz], ctypes.c_int),
            "or_solve_spd": ([_d, _d, _sz, _d, _d, _d, _i64], ctypes.c_int),
            "or_solve_spd_f128": ([_d, _d, _sz, _d, _d, _d, _i64], ctypes.c_int),
            "or_canonical_orthogonalize": ([_d, _sz, ctypes.c_double, _d], ctypes.c_size_t),
            "or_solve_gen_eigen": ([_d, _d, _sz, ctypes.c_double, _d, _d], ctypes.c_size_t),
            "or_overlap_primitive_f64": ([ctypes.c_double, _d, ctypes.c_double, _d], ctypes.c_double),
            "or_overlap_primitive_f128": ([ctypes.c_double, _d, ctypes.c_double, _d, _d], None),
            "or_assemble_overlap_s": ([_sz, _d, _i64, _d, _d, _d, _d, _i64], None),
            "or_assemble_overlap": ([_sz, ctypes.POINTER(ctypes.c_int32), _d, _i64, _d, _d, _d, _d, _i64],
                                    ctypes.c_int),
            "or_overlap_norm_dd": ([_sz, _d, _d, _d], None),
            "or_adjoint_f128": ([_sz, _d, _d, _d, ctypes.POINTER(ctypes.c_int32), _sz, _d, _d, _d], ctypes.c_int),
            "or_loss_f256": ([_sz, _d, _d, _d, _d], ctypes.c_int),
            "or_adjoint_f128_lambda": ([_sz, _d, _d, _d, _d, ctypes.POINTER(ctypes.c_int32), _sz, _d, _d, _d],
                                       ctypes.c_int),
            "or_spd_solve_refined": ([_d, _d, _sz, ctypes.c_double, ctypes.c_int, _d], ctypes.c_int),
            "or_batched_refined": ([ctypes.c_int, _i64, _d, _d, _d, ctypes.c_double, ctypes.c_int, _d,
                                    ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
            "or_gemm_entries_f512": ([ctypes.c_int, _d, _d, _d, _d, _sz, _sz, _sz, ctypes.c_int, _i64, _sz],
                                     ctypes.c_int),
            "or_fd_grad_f256": ([_sz, _d, _d, _d, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                 _sz, ctypes.c_double, _d, _d], ctypes.c_int),
        }
        for name, (args, res) in sigs.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "need C-contiguous float64"
    return a.ctypes.data_as(_d)


def _f(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(t: int) -> None:
    lib().or_set_num_threads(int(t))


def num_threads() -> int:
    return int(lib().or_num_threads())


# ---------------- f128 scalars ----------------
def dd(hi, lo=0.0) -> np.ndarray:
    return np.array([hi, lo], dtype=np.float64)


def _dd2(name, a, b):
    o = np.zeros(2)
    getattr(lib(), name)(_p(_f(a)), _p(_f(b)), _p(o))
    return o


def dd_add(a, b): return _dd2("or_dd_add", a, b)
def dd_sub(a, b): return _dd2("or_dd_sub", a, b)
def dd_mul(a, b): return _dd2("or_dd_mul", a, b)
def dd_div(a, b): return _dd2("or_dd_div", a, b)


def _dd1(name, a):
    o = np.zeros(2)
    getattr(lib(), name)(_p(_f(a)), _p(o))
    return o


def dd_sqrt(a): return _dd1("or_dd_sqrt", a)
def dd_recip(a): return _dd1("or_dd_recip", a)
def dd_exp(a): return _dd1("or_dd_exp", a)
def dd_ln(a): return _dd1("or_dd_ln", a)


def mf_op(name: str, N: int, *args) -> np.ndarray:
    o = np.zeros(N)
    rc = getattr(lib(), "or_mf_" + name)(N, *[_p(_f(a)) for a in args], _p(o))
    assert rc == 0
    return o


# ---------------- f128 linalg ----------------
def gemm(a, b, m, n, k, atb=False, rows=None) -> np.ndarray:
    """linalg.rs:150 gemm / :168 gemm_atb. a: (m,k,2) or (k,m,2) if atb."""
    a, b = _f(a), _f(b)
    c = np.zeros((m, n, 2))
    r0, r1 = (0, m) if rows is None else rows
    lib().or_f128_gemm_rows(_p(a), _p(b), _p(c), m, n, k, int(atb), r0, r1)
    return c


def gemm_entries(a, b, m, n, k, idx, atb=False) -> np.ndarray:
    a, b = _f(a), _f(b)
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    out = np.zeros((len(idx), 2))
    lib().or_f128_gemm_entries(_p(a), _p(b), _p(out), m, n, k, int(atb),
                               idx.ctypes.data_as(_i64), len(idx))
    return out


def dot(a, b) -> np.ndarray:
    a, b = _f(a), _f(b)
    o = np.zeros(2)
    lib().or_f128_dot(_p(a), _p(b), a.shape[0], _p(o))
    return o


def matvec(a, x, n) -> np.ndarray:
    a, x = _f(a), _f(x)
    y = np.zeros((n, 2))
    lib().or_f128_matvec(_p(a), _p(x), _p(y), n)
    return y


def gemv(a, rows, cols, x) -> np.ndarray:
    a, x = _f(a), _f(x)
    y = np.zeros((rows, 2))
    lib().or_f128_gemv(_p(a), rows, cols, _p(x), _p(y))
    return y


class CholeskyError(Exception):
    """linalg.rs:197-200: failure pivot and the non-positive diagonal value."""

    def __init__(self, pivot: int, value: float):
        super().__init__(f"Cholesky failed at pivot {pivot} (value={value:.4e})")
        self.pivot, self.value = pivot, value


def cholesky(a, n) -> np.ndarray:
    """linalg.rs:42. Returns a new array holding L in its lower triangle."""
    a = _f(a).copy()
    pv, val = ctypes.c_int64(0), ctypes.c_double(0)
    rc = lib().or_f128_cholesky(_p(a), n, ctypes.byref(pv), ctypes.byref(val))
    if rc != 0:
        raise CholeskyError(pv.value, val.value)
    return a


def cholesky_blocked(a, n, nb) -> np.ndarray:
    a = _f(a).copy()
    pv, val = ctypes.c_int64(0), ctypes.c_double(0)
    rc = lib().or_f128_cholesky_blocked(_p(a), n, nb, ctypes.byref(pv), ctypes.byref(val))
    if rc != 0:
        raise CholeskyError(pv.value, val.value)
    return a


def forward_solve(l, b, n):
    y = np.zeros((n, 2))
    lib().or_f128_forward_solve(_p(_f(l)), _p(_f(b)), _p(y), n)
    return y


def backward_solve(l, y, n):
    x = np.zeros((n, 2))
    lib().or_f128_backward_solve(_p(_f(l)), _p(_f(y)), _p(x), n)
    return x


def solve_cholesky(l, b, n):
    x = np.zeros((n, 2))
    lib().or_f128_solve_cholesky(_p(_f(l)), _p(_f(b)), _p(x), n)
    return x


def cond_estimate(l, n) -> float:
    return float(lib().or_f128_cond_estimate(_p(_f(l)), n))


def jacobi_eigen(a, n, max_iter):
    """linalg.rs:299. Returns (evals (n,2), evecs as rows (n,n,2), sweeps)."""
    ev = np.zeros((n, 2))
    vec = np.zeros((n, n, 2))
    sw = ctypes.c_size_t(0)
    rc = lib().or_f128_jacobi_eigen(_p(_f(a)), n, max_iter, _p(ev), _p(vec), ctypes.byref(sw))
    if rc != 0:
        raise RuntimeError("Jacobi eigenvalue solver did not converge within max iterations")
    return ev, vec, sw.value


# ---------------- MultiFloat<N> linalg ----------------
def mf_gemm(N, a, b, m, n, k, atb=False, rows=None):
    a, b = _f(a), _f(b)
    c = np.zeros((m, n, N))
    r0, r1 = (0, m) if rows is None else rows
    assert lib().or_mf_gemm_rows(N, _p(a), _p(b), _p(c), m, n, k, int(atb), r0, r1) == 0
    return c


def mf_gemm_entries(N, a, b, m, n, k, idx, atb=False):
    a, b = _f(a), _f(b)
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    out = np.zeros((len(idx), N))
    assert lib().or_mf_gemm_entries(N, _p(a), _p(b), _p(out), m, n, k, int(atb),
                                    idx.ctypes.data_as(_i64), len(idx)) == 0
    return out


def gemm_entries_f512(a, b, m, n, k, idx, atb=False):
    """f512 entries C[i, j] of op(A) B for f128 (..., 2) or f256 (..., 4) inputs:
    (count x 4 leading limbs, count sums of |a||b|) -- the GEMMs' f512 checker."""
    a, b = _f(a), _f(b)
    limbs = a.shape[-1]
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    out = np.zeros((len(idx), 4))
    ab = np.zeros(len(idx))
    assert lib().or_gemm_entries_f512(limbs, _p(a), _p(b), _p(out), _p(ab), m, n, k, int(atb),
                                      idx.ctypes.data_as(_i64), len(idx)) == 0
    return out, ab


def mf_gemv(N, a, x, n, m):
    y = np.zeros((n, N))
    assert lib().or_mf_gemv(N, _p(_f(a)), _p(_f(x)), _p(y), n, m) == 0
    return y


def mf_cholesky(N, a, n):
    a = _f(a).copy()
    if lib().or_mf_cholesky(N, _p(a), n) != 0:
        raise RuntimeError("Cholesky failed: matrix is not positive definite")
    return a


def mf_cholesky_solve(N, l, b, n):
    x = np.zeros((n, N))
    assert lib().or_mf_cholesky_solve(N, _p(_f(l)), _p(_f(b)), _p(x), n) == 0
    return x


# ---------------- solver ----------------
STRATEGIES = ("Float64", "MixedPrecision", "Float128")


def _solution(rc, x, xf, info, pv):
    if rc != 0:
        raise RuntimeError(f"Matrix is not positive definite (failed at pivot {pv.value})")
    return {"x": x, "x_f64": xf, "kappa": info[0], "residual_norm": info[1],
            "strategy": STRATEGIES[int(info[2])], "refinement_iters": int(info[3])}


def solve_spd(a_f64, b_f64, n):
    """solver/src/lib.rs:38."""
    x, xf, info = np.zeros((n, 2)), np.zeros(n), np.zeros(4)
    pv = ctypes.c_int64(0)
    rc = lib().or_solve_spd(_p(_f(a_f64)), _p(_f(b_f64)), n, _p(x), _p(xf), _p(info), ctypes.byref(pv))
    return _solution(rc, x, xf, info, pv)


def spd_solve_refined(S, b, n, tol=1e-28, max_iter=10):
    """f128 cholesky + solve_cholesky refined with f256 residuals (the host
    counterpart of the GPU's plain refined solve). Returns (x (n, 2), steps)."""
    S, b = _f(S), _f(b)
    if b.ndim == 1:
        b = np.stack([b, np.zeros_like(b)], -1)
    x = np.zeros((n, 2))
    it = lib().or_spd_solve_refined(_p(S), _p(b), n, tol, max_iter, _p(x))
    if it < 0:
        raise CholeskyError(-1, float("nan"))
    return x, int(it)


def batched_refined(batch, tol=1e-28, max_iter=10):
    """Host counterpart of the GPU batched solver (or_batched_refined): every
    system assembled in f128 and solved by spd_solve_refined, OpenMP over
    systems. Returns (x (N, 2), iters (count,))."""
    off = np.ascontiguousarray(batch["offsets"], dtype=np.int64)
    count = len(off) - 1
    x = np.zeros((int(off[-1]), 2))
    it = np.zeros(count, dtype=np.int32)
    lib().or_batched_refined(count, off.ctypes.data_as(_i64), _p(_f(batch["centers"])), _p(_f(batch["alpha"])),
                             _p(_f(batch["b"])), tol, max_iter, _p(x), it.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    return x, it


def solve_spd_f128(a, b, n):
    """solver/src/lib.rs:71."""
    x, xf, info = np.zeros((n, 2)), np.zeros(n), np.zeros(4)
    pv = ctypes.c_int64(0)
    rc = lib().or_solve_spd_f128(_p(_f(a)), _p(_f(b)), n, _p(x), _p(xf), _p(info), ctypes.byref(pv))
    return _solution(rc, x, xf, info, pv)


def canonical_orthogonalize(s, n, threshold):
    """solver/src/ortho.rs:151. Returns X (n, n_orth, 2)."""
    x = np.zeros((n, n, 2))
    m = lib().or_canonical_orthogonalize(_p(_f(s)), n, threshold, _p(x))
    return np.ascontiguousarray(x.reshape(-1)[: n * m * 2].reshape(n, m, 2))


def solve_gen_eigen(f, s, n, threshold):
    """solver/src/ortho.rs:191. Returns (eigenvalues (m, 2), C (n, m, 2), m)."""
    ev = np.zeros((n, 2))
    c = np.zeros((n, n, 2))
    m = lib().or_solve_gen_eigen(_p(_f(f)), _p(_f(s)), n, threshold, _p(ev), _p(c))
    return ev[:m].copy(), np.ascontiguousarray(c.reshape(-1)[: n * m * 2].reshape(n, m, 2)), m


# ---------------- overlap ----------------
def overlap_primitive_f64(ai, ci, aj, cj) -> float:
    return float(lib().or_overlap_primitive_f64(ai, _p(_f(ci)), aj, _p(_f(cj))))


def overlap_primitive_f128(ai, ci, aj, cj) -> np.ndarray:
    o = np.zeros(2)
    lib().or_overlap_primitive_f128(ai, _p(_f(ci)), aj, _p(_f(cj)), _p(o))
    return o


DEFAULT_SCREEN = (0.1, 500.0, 1e-14, 12.0)  # screen.rs:36-45


def assemble_overlap_s(centers, prim_alpha, prim_coeff, params=DEFAULT_SCREEN):
    """assemble.rs:35 for s shells. prim_alpha/prim_coeff: list of per-shell lists."""
    n = len(centers)
    off = np.zeros(n + 1, dtype=np.int64)
    for i, al in enumerate(prim_alpha):
        off[i + 1] = off[i] + len(al)
    al = _f(np.concatenate([np.asarray(x, dtype=np.float64) for x in prim_alpha]))
    co = _f(np.concatenate([np.asarray(x, dtype=np.float64) for x in prim_coeff]))
    mat = np.zeros((n, n))
    tc = np.zeros(3, dtype=np.int64)
    lib().or_assemble_overlap_s(n, _p(_f(centers)), off.ctypes.data_as(_i64), _p(al), _p(co),
                                _p(_f(params)), _p(mat), tc.ctypes.data_as(_i64))
    return mat, {"f64_pairs": int(tc[0]), "f128_pairs": int(tc[1]), "skipped_pairs": int(tc[2])}


def assemble_overlap(shell_l, centers, prim_alpha, prim_coeff, params=DEFAULT_SCREEN):
    """assemble.rs:35-85 for shells of kinds S/P/D/F (shell_l = 0..3) with the
    Obara-Saika blocks of integral.rs:144-352: (matrix (n_ao, n_ao), tier_counts)."""
    shell_l = np.ascontiguousarray(shell_l, dtype=np.int32)
    n = len(shell_l)
    off = np.zeros(n + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(a) for a in prim_alpha])
    al = _f(np.concatenate(prim_alpha))
    co = _f(np.concatenate(prim_coeff))
    n_ao = int(sum((l + 1) * (l + 2) // 2 for l in shell_l))
    mat = np.zeros((n_ao, n_ao))
    tiers = np.zeros(3, dtype=np.int64)
    rc = lib().or_assemble_overlap(n, shell_l.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _p(_f(centers)),
                                   off.ctypes.data_as(_i64), _p(al), _p(co), _p(_f(params)), _p(mat),
                                   tiers.ctypes.data_as(_i64))
    assert rc == 0
    return mat, tiers


def overlap_norm_dd(centers, alpha) -> np.ndarray:
    n = len(alpha)
    s = np.zeros((n, n, 2))
    lib().or_overlap_norm_dd(n, _p(_f(centers)), _p(_f(alpha)), _p(s))
    return s


# ---------------- adjoint ----------------
def adjoint_f128(centers, alpha, b, center_of, n_centers):
    """Gradient of L = b^T S^-1 b from the reference's f128 primitives.

    Returns (loss (2,), grad wrt centre coordinates (n_centers,3,2),
    grad wrt log-exponents (n,2))."""
    n = len(alpha)
    co = np.ascontiguousarray(center_of, dtype=np.int32)
    loss = np.zeros(2)
    gR = np.zeros((n_centers, 3, 2))
    ga = np.zeros((n, 2))
    rc = lib().or_adjoint_f128(n, _p(_f(centers)), _p(_f(alpha)), _p(_f(b)),
                               co.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), n_centers, _p(loss), _p(gR), _p(ga))
    if rc != 0:
        raise RuntimeError("not positive definite")
    return loss, gR, ga


def adjoint_f128_refined(centers, alpha, b, center_of, n_centers):
    """The host counterpart of the GPU adjoint: lambda from the refined host
    solve (spd_solve_refined: f128 factor, f256 residuals, to ~1e-25), then
    the same f128 contraction. Returns (loss, gR (n_centers,3,2), ga (n,2))."""
    n = len(alpha)
    S = overlap_norm_dd(centers, alpha)
    lam, _ = spd_solve_refined(S, np.asarray(b, dtype=np.float64), n)
    co = np.ascontiguousarray(center_of, dtype=np.int32)
    loss, gR, ga = np.zeros(2), np.zeros((n_centers, 3, 2)), np.zeros((n, 2))
    rc = lib().or_adjoint_f128_lambda(n, _p(_f(centers)), _p(_f(alpha)), _p(_f(b)), _p(_f(lam)),
                                      co.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), n_centers, _p(loss),
                                      _p(gR), _p(ga))
    assert rc == 0
    return loss, gR, ga


def loss_f256(centers4, alpha4, b):
    """L = b^T S^-1 b in MultiFloat<4> from f256 centres (n,3,4) and exponents (n,4)."""
    n = len(alpha4)
    out = np.zeros(4)
    rc = lib().or_loss_f256(n, _p(_f(centers4)), _p(_f(alpha4)), _p(_f(b)), _p(out))
    if rc != 0:
        raise RuntimeError("not positive definite")
    return out


def fd_grad_f256(centers, alpha, b, center_of, cen_list, h=1e-20):
    """f256 central differences of L = b^T S^-1 b wrt the coordinates of the
    centres in cen_list and the log-exponents of their basis functions
    (or_fd_grad_f256). Returns (gR (len(cen_list), 3, 4), funcs, ga (len(funcs), 4))."""
    centers, alpha, b = _f(centers), _f(alpha), _f(b)
    co = np.ascontiguousarray(center_of, dtype=np.int32)
    cl = np.ascontiguousarray(cen_list, dtype=np.int32)
    funcs = np.nonzero(np.isin(co, cl))[0]
    gR = np.zeros((len(cl), 3, 4))
    ga = np.zeros((len(funcs), 4))
    i32 = ctypes.POINTER(ctypes.c_int32)
    rc = lib().or_fd_grad_f256(len(alpha), _p(centers), _p(alpha), _p(b), co.ctypes.data_as(i32),
                               cl.ctypes.data_as(i32), len(cl), h, _p(gR), _p(ga))
    assert rc == 0, "f256 factorisation failed"
    return gR, funcs, ga
