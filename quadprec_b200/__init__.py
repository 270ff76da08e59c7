"""quadprec_b200: ctypes binding of the B200 extended-precision library.

The product is the C ABI in ``include/hyperprec_gpu.h`` implemented by
``libhyperprec_gpu.so`` (hand-written sm_100a CUDA). This module only loads
that library and converts numpy/torch buffers to pointers for the test suite
and ``bench.py``. There is no CPU fallback: if the library or a CUDA device is
missing, calls raise.

Arrays use the reference's layout: an f128 matrix is float64 of shape
(rows, cols, 2) (hi, lo); an f256 matrix is (rows, cols, 4).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhyperprec_gpu.so")

HP_OK = 0
HP_ERR_INVALID_ARG = -1
HP_ERR_NOT_SPD = -2
HP_ERR_NO_CONVERGE = -3
HP_ERR_CUDA = -4
HP_ERR_TIMEOUT = -5
HP_ERR_UNSUPPORTED = -6

PLAIN = 0
OZAKI = 1

_lib = None
_d = ctypes.POINTER(ctypes.c_double)
_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_i64p = ctypes.POINTER(ctypes.c_int64)


class HPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hyperprec error {code}: {msg}")
        self.code = code


# name -> (argtypes, restype); kept in step with include/hyperprec_gpu.h
SIGNATURES = {
    "hp_last_error": ([], ctypes.c_char_p),
    "hp_version": ([], ctypes.c_char_p),
    "hp_device_ok": ([], ctypes.c_int),
    "hp_device_status": ([_vp, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int], ctypes.c_int),
    "hp_measure_peaks": ([ctypes.c_int, _d, _d, _d, _d], ctypes.c_int),
    "hp_f128_to_string": ([_vp, ctypes.c_char_p, _sz], ctypes.c_int),
    "hp_f128_from_string": ([ctypes.c_char_p, _vp], ctypes.c_int),
    "hp_mf_to_string": ([ctypes.c_int, _vp, ctypes.c_char_p, _sz], ctypes.c_int),
    "hp_mf_from_string": ([ctypes.c_int, ctypes.c_char_p, _vp], ctypes.c_int),
    "hp_debug_trsv_wavefront": ([_vp, _vp, _vp, _sz, ctypes.c_int, ctypes.c_uint64, ctypes.c_int], ctypes.c_int),
    "hp_profile_enable": ([ctypes.c_int], None),
    "hp_profile_read": ([_d, ctypes.c_int, ctypes.c_char_p, _sz], ctypes.c_int),
    "hp_f128_gemm": ([_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int], ctypes.c_int),
    "hp_f128_gemm_atb": ([_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int], ctypes.c_int),
    "hp_f128_gemm_dev": ([_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int, _vp], ctypes.c_int),
    "hp_f128_gemm_atb_dev": ([_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int, _vp], ctypes.c_int),
    "hp_f128_gemm_noalloc_dev": ([_vp, _vp, _vp, _sz, _sz, _sz, _vp], ctypes.c_int),
    "hp_f256_gemm": ([_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int], ctypes.c_int),
    "hp_f256_gemm_atb": ([_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int], ctypes.c_int),
    "hp_f256_gemm_dev": ([_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int, _vp], ctypes.c_int),
    "hp_f256_gemm_atb_dev": ([_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int, _vp], ctypes.c_int),
    "hp_f512_gemm": ([_vp, _vp, _vp, _sz, _sz, _sz], ctypes.c_int),
    "hp_f512_gemm_atb": ([_vp, _vp, _vp, _sz, _sz, _sz], ctypes.c_int),
    "hp_f512_gemm_dev": ([_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int, _vp], ctypes.c_int),
    "hp_f512_cholesky": ([_vp, _sz, _i64p], ctypes.c_int),
    "hp_f512_cholesky_solve": ([_vp, _vp, _vp, _sz], ctypes.c_int),
    "hp_f128_cholesky": ([_vp, _sz, _i64p, _d], ctypes.c_int),
    "hp_f128_cholesky_blocked": ([_vp, _sz, _sz, _i64p, _d], ctypes.c_int),
    "hp_f128_cholesky_dev": ([_vp, _sz, _i64p, _d, _vp], ctypes.c_int),
    "hp_f128_forward_solve": ([_vp, _vp, _vp, _sz], ctypes.c_int),
    "hp_f128_backward_solve": ([_vp, _vp, _vp, _sz], ctypes.c_int),
    "hp_f128_solve_cholesky": ([_vp, _vp, _vp, _sz], ctypes.c_int),
    "hp_f128_matvec": ([_vp, _vp, _vp, _sz], ctypes.c_int),
    "hp_f128_solve_cholesky_dev": ([_vp, _vp, _sz, _vp], ctypes.c_int),
    "hp_f128_dot": ([_vp, _vp, _sz, _vp], ctypes.c_int),
    "hp_f128_gemv": ([_vp, _sz, _sz, _vp, _vp], ctypes.c_int),
    "hp_f128_cond_estimate": ([_vp, _sz, _d], ctypes.c_int),
    "hp_f256_cholesky": ([_vp, _sz, _i64p], ctypes.c_int),
    "hp_f256_cholesky_dev": ([_vp, _sz, _i64p, _vp], ctypes.c_int),
    "hp_f256_cholesky_solve": ([_vp, _vp, _vp, _sz], ctypes.c_int),
    "hp_f256_gemv": ([_vp, _vp, _vp, _sz, _sz], ctypes.c_int),
    "hp_f256_dot": ([_vp, _vp, _sz, _vp], ctypes.c_int),
    "hp_canonical_orthogonalize": ([_vp, _sz, ctypes.c_double, _vp, ctypes.POINTER(_sz)], ctypes.c_int),
    "hp_solve_gen_eigen": ([_vp, _vp, _sz, ctypes.c_double, _vp, _vp, ctypes.POINTER(_sz)], ctypes.c_int),
    "hp_solve_spd": ([_vp, _vp, _sz, _vp, _vp, _vp, _i64p], ctypes.c_int),
    "hp_solve_spd_f128": ([_vp, _vp, _sz, _vp, _vp, _vp, _i64p], ctypes.c_int),
    "hp_spd_solve_refined": ([_vp, _vp, _sz, ctypes.c_int, ctypes.c_double, ctypes.c_int, _vp, _vp, _i64p],
                             ctypes.c_int),
    "hp_spd_solve_refined_dev": ([_vp, _vp, _sz, ctypes.c_int, ctypes.c_double, ctypes.c_int, _vp, _vp, _i64p,
                                  _vp], ctypes.c_int),
    "hp_batched_config": ([_vp, _vp], ctypes.c_int),
    "hp_spd_solve_batched": ([ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_int],
                             ctypes.c_int),
    "hp_spd_solve_batched_dev": ([ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_int,
                                  _vp], ctypes.c_int),
    "hp_overlap_norm_dd_batched_dev": ([ctypes.c_int, _vp, _vp, _vp, _vp, _vp], ctypes.c_int),
    "hp_f128_jacobi_eigen": ([_vp, _sz, _sz, _vp, _vp, ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "hp_f128_jacobi_eigen_batched_dev": ([ctypes.c_int, _vp, _vp, _sz, _vp, _vp, _vp, _vp, _vp], ctypes.c_int),
    "hp_overlap_adjoint": ([_sz, _vp, _vp, _vp, _vp, _sz, ctypes.c_int, _vp, _vp, _vp, _vp], ctypes.c_int),
    "hp_overlap_adjoint_dev": ([_sz, _vp, _vp, _vp, _vp, _sz, ctypes.c_int, _vp, _vp, _vp, _vp, _vp], ctypes.c_int),
    "hp_assemble_overlap_s": ([_sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp], ctypes.c_int),
    "hp_assemble_overlap": ([_sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_sz)], ctypes.c_int),
    "hp_overlap_norm_dd": ([_sz, _vp, _vp, _vp], ctypes.c_int),
    "hp_overlap_norm_dd_dev": ([_sz, _vp, _vp, _vp, _vp], ctypes.c_int),
}


class Solution(ctypes.Structure):
    """hp_solution_t (crates/solver/src/lib.rs:10-23 Solution, without vectors)."""
    _fields_ = [("kappa", ctypes.c_double), ("residual_norm", ctypes.c_double),
                ("strategy", ctypes.c_int32), ("refinement_iters", ctypes.c_int32)]


STRATEGIES = ("Float64", "MixedPrecision", "Float128")


class RefineInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("last_correction", ctypes.c_double), ("factor_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double)]


def lib():
    """Load libhyperprec_gpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: run quadprec_b200.build.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != HP_OK:
        raise HPError(rc, (lib().hp_last_error() or b"").decode())


def _ptr(a) -> int:
    if isinstance(a, np.ndarray):
        assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return int(a.data_ptr())  # torch tensor (host pinned or device)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def device_ok() -> bool:
    return bool(lib().hp_device_ok())


def profile_enable(on: bool = True) -> None:
    lib().hp_profile_enable(1 if on else 0)


def profile_read() -> dict:
    """Phase durations (ms) recorded since profile_enable(); waits for them."""
    ms = (ctypes.c_double * 32)()
    names = ctypes.create_string_buffer(1024)
    n = lib().hp_profile_read(ms, 32, names, 1024)
    keys = names.value.decode().split(",") if n else []
    return {k: ms[i] for i, k in enumerate(keys)}


# ---------------- GEMM ----------------
def f128_gemm(a, b, m, n, k, mode=PLAIN, atb=False) -> np.ndarray:
    """linalg.rs:150 gemm / :168 gemm_atb through the host-pointer C ABI."""
    a, b = _c(a), _c(b)
    c = np.empty((m, n, 2))
    fn = lib().hp_f128_gemm_atb if atb else lib().hp_f128_gemm
    check(fn(_ptr(a), _ptr(b), _ptr(c), m, n, k, mode))
    return c


def f256_gemm(a, b, m, n, k, mode=PLAIN, atb=False) -> np.ndarray:
    """multifloat/linalg.rs:39 mf_gemm / :64 mf_gemm_atb with N = 4."""
    a, b = _c(a), _c(b)
    c = np.empty((m, n, 4))
    fn = lib().hp_f256_gemm_atb if atb else lib().hp_f256_gemm
    check(fn(_ptr(a), _ptr(b), _ptr(c), m, n, k, mode))
    return c


def f128_gemm_dev(a, b, c, m, n, k, mode=PLAIN, atb=False, stream=0) -> None:
    """Device-pointer form; a, b, c are CUDA tensors (float64, AoS)."""
    fn = lib().hp_f128_gemm_atb_dev if atb else lib().hp_f128_gemm_dev
    check(fn(_ptr(a), _ptr(b), _ptr(c), m, n, k, mode, stream))


def f256_gemm_dev(a, b, c, m, n, k, mode=PLAIN, atb=False, stream=0) -> None:
    fn = lib().hp_f256_gemm_atb_dev if atb else lib().hp_f256_gemm_dev
    check(fn(_ptr(a), _ptr(b), _ptr(c), m, n, k, mode, stream))


# ---------------- Cholesky / solves / SPD ----------------
class CholeskyError(HPError):
    """linalg.rs:197-200 CholeskyError { pivot, value }."""

    def __init__(self, pivot: int, value: float):
        RuntimeError.__init__(self, f"Cholesky failed at pivot {pivot} (value={value:.4e})")
        self.code, self.pivot, self.value = HP_ERR_NOT_SPD, pivot, value


def _chol_call(fn, a, *args):
    a = _c(a).copy()
    pv, val = ctypes.c_int64(-1), ctypes.c_double(0.0)
    rc = fn(_ptr(a), *args, ctypes.byref(pv), ctypes.byref(val))
    if rc == HP_ERR_NOT_SPD:
        raise CholeskyError(pv.value, val.value)
    check(rc)
    return a


def f128_cholesky(a, n):
    """linalg.rs:42 cholesky; returns a copy with L in the lower triangle."""
    return _chol_call(lib().hp_f128_cholesky, a, n)


def f128_cholesky_blocked(a, n, nb):
    """linalg.rs:238 cholesky_blocked."""
    return _chol_call(lib().hp_f128_cholesky_blocked, a, n, nb)


def f256_cholesky(a, n):
    """multifloat/linalg.rs:88 mf_cholesky::<4>; a is (n, n, 4); returns a copy
    with L in the lower triangle (bit-identical to the reference)."""
    a = _c(a).copy()
    pv = ctypes.c_int64(-1)
    rc = lib().hp_f256_cholesky(_ptr(a), n, ctypes.byref(pv))
    if rc == HP_ERR_NOT_SPD:
        raise CholeskyError(pv.value, float("nan"))
    check(rc)
    return a


def f512_gemm(a, b, m, n, k, atb=False) -> np.ndarray:
    """multifloat/linalg.rs:39 mf_gemm::<8> / :64 mf_gemm_atb::<8> (bit-identical)."""
    a, b = _c(a), _c(b)
    c = np.empty((m, n, 8))
    fn = lib().hp_f512_gemm_atb if atb else lib().hp_f512_gemm
    check(fn(_ptr(a), _ptr(b), _ptr(c), m, n, k))
    return c


def f512_cholesky(a, n):
    """multifloat/linalg.rs:89 mf_cholesky::<8>; returns a copy with L in the lower triangle."""
    a = _c(a).copy()
    pv = ctypes.c_int64(-1)
    rc = lib().hp_f512_cholesky(_ptr(a), n, ctypes.byref(pv))
    if rc == HP_ERR_NOT_SPD:
        raise CholeskyError(pv.value, float("nan"))
    check(rc)
    return a


def f512_cholesky_solve(l, b, n):
    """multifloat/linalg.rs:145 mf_cholesky_solve::<8>: x (n, 8)."""
    l, b = _c(l), _c(b)
    x = np.empty((n, 8))
    check(lib().hp_f512_cholesky_solve(_ptr(l), _ptr(b), _ptr(x), n))
    return x


def f256_cholesky_solve(l, b, n):
    """multifloat/linalg.rs:141 mf_cholesky_solve::<4>; l (n, n, 4), b (n, 4)."""
    l, b = _c(l), _c(b)
    out = np.empty((n, 4))
    check(lib().hp_f256_cholesky_solve(_ptr(l), _ptr(b), _ptr(out), n))
    return out


def canonical_orthogonalize(s, n, threshold):
    """solver/src/ortho.rs:151 canonical_orthogonalize; s is (n, n, 2).
    Returns X as (n, n_orth, 2)."""
    s = _c(s)
    x = np.zeros((n, n, 2))
    m = _sz(0)
    check(lib().hp_canonical_orthogonalize(_ptr(s), n, threshold, _ptr(x), ctypes.byref(m)))
    return np.ascontiguousarray(x.reshape(-1)[: n * m.value * 2].reshape(n, m.value, 2))


def solve_gen_eigen(f, s, n, threshold):
    """solver/src/ortho.rs:191 solve_gen_eigen; f, s are (n, n, 2).
    Returns (eigenvalues (m, 2) ascending, eigenvectors C (n, m, 2), m)."""
    f, s = _c(f), _c(s)
    ev = np.zeros((n, 2))
    c = np.zeros((n, n, 2))
    m = _sz(0)
    check(lib().hp_solve_gen_eigen(_ptr(f), _ptr(s), n, threshold, _ptr(ev), _ptr(c), ctypes.byref(m)))
    mm = m.value
    return ev[:mm].copy(), np.ascontiguousarray(c.reshape(-1)[: n * mm * 2].reshape(n, mm, 2)), mm


def f256_gemv(a, x, n, m):
    """multifloat/linalg.rs:17 mf_gemv::<4>; a (n, m, 4), x (m, 4) -> (n, 4)."""
    a, x = _c(a), _c(x)
    y = np.empty((n, 4))
    check(lib().hp_f256_gemv(_ptr(a), _ptr(x), _ptr(y), n, m))
    return y


def f256_dot(a, b):
    """multifloat/linalg.rs:7 mf_dot::<4>; a, b (len, 4) -> (4,)."""
    a, b = _c(a), _c(b)
    out = np.empty(4)
    check(lib().hp_f256_dot(_ptr(a), _ptr(b), len(a), _ptr(out)))
    return out


def _solve(name, l, b, n):
    l, b = _c(l), _c(b)
    out = np.empty((n, 2))
    check(getattr(lib(), name)(_ptr(l), _ptr(b), _ptr(out), n))
    return out


def f128_forward_solve(l, b, n): return _solve("hp_f128_forward_solve", l, b, n)
def f128_backward_solve(l, y, n): return _solve("hp_f128_backward_solve", l, y, n)
def f128_solve_cholesky(l, b, n): return _solve("hp_f128_solve_cholesky", l, b, n)
def f128_matvec(a, x, n): return _solve("hp_f128_matvec", a, x, n)


def measure_peaks(reps=5) -> dict:
    """Measured FP64 (TFLOP/s) and int8 tensor (TOP/s) rates of this device."""
    v = [ctypes.c_double(0.0) for _ in range(4)]
    check(lib().hp_measure_peaks(reps, *[ctypes.byref(x) for x in v]))
    return {"fp64_tflops": v[0].value, "i8_tops": v[1].value, "fp64_ms": v[2].value, "i8_ms": v[3].value}


def f128_to_string(v) -> str:
    """dd.rs:448-461 human-readable serde form of one f128 (hi, lo)."""
    v = _c(v)
    buf = ctypes.create_string_buffer(64)
    check(lib().hp_f128_to_string(_ptr(v), buf, 64))
    return buf.value.decode()


def f128_from_string(s: str) -> np.ndarray:
    """dd.rs:495-509 parse_dd_string."""
    out = np.zeros(2)
    check(lib().hp_f128_from_string(s.encode(), _ptr(out)))
    return out


def mf_to_string(v) -> str:
    """multifloat/traits.rs:15-34 human-readable serde form of one MultiFloat<N>."""
    v = _c(v)
    cap = 24 * len(v) + 8
    buf = ctypes.create_string_buffer(cap)
    check(lib().hp_mf_to_string(len(v), _ptr(v), buf, cap))
    return buf.value.decode()


def mf_from_string(s: str, n_limbs: int) -> np.ndarray:
    """multifloat/traits.rs:104-150 parse_limbs_string."""
    out = np.zeros(n_limbs)
    check(lib().hp_mf_from_string(n_limbs, s.encode(), _ptr(out)))
    return out


def device_status(stream=0, clear=True) -> tuple[int, int]:
    """(return code, status bits) of the *_dev calls enqueued on `stream`."""
    bits = ctypes.c_uint32(0)
    rc = lib().hp_device_status(stream, ctypes.byref(bits), int(clear))
    return rc, int(bits.value)


def debug_trsv_wavefront(l, b, n, upper_t=False, wait_ns=0, withheld_block=-1):
    """(return code, x) of the wavefront solve L x = b (or L^T x = b)."""
    l, b = _c(l), _c(b)
    x = np.zeros((n, 2))
    rc = lib().hp_debug_trsv_wavefront(_ptr(l), _ptr(b), _ptr(x), n, int(upper_t), int(wait_ns),
                                       int(withheld_block))
    return rc, x


def f128_dot(a, b) -> np.ndarray:
    """linalg.rs:7 dot: one f128 (2,)."""
    a, b = _c(a), _c(b)
    out = np.zeros(2)
    check(lib().hp_f128_dot(_ptr(a), _ptr(b), len(a), _ptr(out)))
    return out


def f128_gemv(a, rows, cols, x) -> np.ndarray:
    """linalg.rs:29 gemv: y (rows, 2) = A (rows x cols) x."""
    a, x = _c(a), _c(x)
    y = np.zeros((rows, 2))
    check(lib().hp_f128_gemv(_ptr(a), rows, cols, _ptr(x), _ptr(y)))
    return y


def f128_cond_estimate(l, n) -> float:
    out = ctypes.c_double(0)
    check(lib().hp_f128_cond_estimate(_ptr(_c(l)), n, ctypes.byref(out)))
    return out.value


def _spd(fn, a, b, n):
    a, b = _c(a), _c(b)
    x, xf = np.empty((n, 2)), np.empty(n)
    sol = Solution()
    pv = ctypes.c_int64(-1)
    rc = fn(_ptr(a), _ptr(b), n, _ptr(x), _ptr(xf), ctypes.byref(sol), ctypes.byref(pv))
    if rc == HP_ERR_NOT_SPD:
        raise HPError(rc, f"Matrix is not positive definite (failed at pivot {pv.value})")
    check(rc)
    return {"x": x, "x_f64": xf, "kappa": sol.kappa, "residual_norm": sol.residual_norm,
            "strategy": STRATEGIES[sol.strategy], "refinement_iters": sol.refinement_iters}


def solve_spd(a_f64, b_f64, n):
    """crates/solver/src/lib.rs:38 solve_spd."""
    return _spd(lib().hp_solve_spd, a_f64, b_f64, n)


def solve_spd_f128(a, b, n):
    """crates/solver/src/lib.rs:71 solve_spd_f128."""
    return _spd(lib().hp_solve_spd_f128, a, b, n)


# ---------------- overlap ----------------
DEFAULT_SCREEN = (0.1, 500.0, 1e-14, 12.0)  # crates/overlap/src/screen.rs:36-45


def assemble_overlap_s(centers, prim_alpha, prim_coeff, params=DEFAULT_SCREEN):
    """assemble.rs:35 assemble_overlap_mixed for a basis of s shells."""
    n = len(centers)
    off = np.zeros(n + 1, dtype=np.int64)
    for i, al in enumerate(prim_alpha):
        off[i + 1] = off[i] + len(al)
    al = _c(np.concatenate([np.asarray(x, dtype=np.float64) for x in prim_alpha]))
    co = _c(np.concatenate([np.asarray(x, dtype=np.float64) for x in prim_coeff]))
    mat = np.zeros((n, n))
    tc = np.zeros(3, dtype=np.int64)
    pr = _c(params)
    check(lib().hp_assemble_overlap_s(n, _ptr(_c(centers)), off.ctypes.data, _ptr(al), _ptr(co), _ptr(pr),
                                      _ptr(mat), tc.ctypes.data))
    return mat, {"f64_pairs": int(tc[0]), "f128_pairs": int(tc[1]), "skipped_pairs": int(tc[2])}


def assemble_overlap(shell_l, centers, prim_alpha, prim_coeff, params=DEFAULT_SCREEN):
    """assemble.rs:35 for shells of kinds S/P/D/F: (matrix (n_ao, n_ao), tier_counts)."""
    shell_l = np.ascontiguousarray(shell_l, dtype=np.int32)
    centers = _c(centers)
    n = len(shell_l)
    off = np.zeros(n + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(a) for a in prim_alpha])
    al = _c(np.concatenate(prim_alpha))
    co = _c(np.concatenate(prim_coeff))
    n_ao = int(sum((l + 1) * (l + 2) // 2 for l in shell_l))
    mat = np.zeros((n_ao, n_ao))
    tiers = np.zeros(3, dtype=np.int64)
    got = ctypes.c_size_t(0)
    check(lib().hp_assemble_overlap(n, shell_l.ctypes.data, _ptr(centers), off.ctypes.data, _ptr(al), _ptr(co),
                                    _ptr(_c(params)), _ptr(mat), tiers.ctypes.data, ctypes.byref(got)))
    assert got.value == n_ao
    return mat, tiers


def overlap_norm_dd(centers, alpha) -> np.ndarray:
    """f128 overlap matrix of normalised s Gaussians (n x n x 2)."""
    centers, alpha = _c(centers), _c(alpha)
    n = len(alpha)
    s = np.empty((n, n, 2))
    check(lib().hp_overlap_norm_dd(n, _ptr(centers), _ptr(alpha), _ptr(s)))
    return s


def spd_solve_refined(S, b, n, mode=OZAKI, tol=1e-28, max_iter=10):
    """Refined SPD solve to 1e-25 (see hp_spd_solve_refined). b may be f64 (n,) or f128 (n,2)."""
    S = _c(S)
    b = _c(b)
    if b.ndim == 1:
        b = np.stack([b, np.zeros_like(b)], -1)
    x = np.empty((n, 2))
    info = RefineInfo()
    pv = ctypes.c_int64(-1)
    rc = lib().hp_spd_solve_refined(_ptr(S), _ptr(b), n, mode, tol, max_iter, _ptr(x), ctypes.byref(info),
                                    ctypes.byref(pv))
    if rc == HP_ERR_NOT_SPD:
        raise HPError(rc, f"Matrix is not positive definite (failed at pivot {pv.value})")
    check(rc)
    return x, {f: getattr(info, f) for f, _ in RefineInfo._fields_}


# ---------------- batched solves / Jacobi ----------------
def spd_solve_batched(batch, tol=1e-28, max_iter=10):
    """Solve every system of workloads.batched_overlap_systems() (host arrays)."""
    off = np.ascontiguousarray(batch["offsets"], dtype=np.int64)
    count = len(off) - 1
    b = _c(batch["b"])
    if b.ndim == 1:
        b = np.stack([b, np.zeros_like(b)], -1)
    x = np.empty((int(off[-1]), 2))
    st = np.zeros(count, dtype=np.int32)
    it = np.zeros(count, dtype=np.int32)
    check(lib().hp_spd_solve_batched(count, off.ctypes.data, _ptr(_c(batch["centers"])), _ptr(_c(batch["alpha"])),
                                      _ptr(b), _ptr(x), st.ctypes.data, it.ctypes.data, tol, max_iter))
    return x, st, it


def batched_config():
    """(threads per CTA, CTAs per SM) the autotuner chose for the latest batched solve."""
    t = np.zeros(1, dtype=np.int32)
    c = np.zeros(1, dtype=np.int32)
    check(lib().hp_batched_config(t.ctypes.data, c.ctypes.data))
    return int(t[0]), int(c[0])


def f128_jacobi_eigen(a, n, max_iter):
    """linalg.rs:299 jacobi_eigen: (evals (n,2), eigenvectors as rows (n,n,2), sweeps)."""
    ev = np.empty((n, 2))
    vec = np.empty((n, n, 2))
    sw = ctypes.c_size_t(0)
    rc = lib().hp_f128_jacobi_eigen(_ptr(_c(a)), n, max_iter, _ptr(ev), _ptr(vec), ctypes.byref(sw))
    if rc == HP_ERR_NO_CONVERGE:
        raise HPError(rc, "Jacobi eigenvalue solver did not converge within max iterations")
    check(rc)
    return ev, vec, sw.value


# ---------------- adjoint ----------------
def overlap_adjoint(centers, alpha, b, center_of, n_centers, mode=OZAKI):
    """Gradient of L = b^T S^-1 b: (loss (2,), grad_R (n_centers,3,2), grad_lnalpha (n,2), info)."""
    n = len(alpha)
    co = np.ascontiguousarray(center_of, dtype=np.int32)
    loss = np.empty(2)
    gR = np.empty((n_centers, 3, 2))
    ga = np.empty((n, 2))
    info = RefineInfo()
    check(lib().hp_overlap_adjoint(n, _ptr(_c(centers)), _ptr(_c(alpha)), _ptr(_c(b)), co.ctypes.data, n_centers,
                                   mode, _ptr(loss), _ptr(gR), _ptr(ga), ctypes.byref(info)))
    return loss, gR, ga, {f: getattr(info, f) for f, _ in RefineInfo._fields_}
