"""GPU parity for the GEMM entry points (through the C ABI).

HP_MODE_PLAIN must be bit-identical to the oracle (the reference's gemm /
mf_gemm). HP_MODE_OZAKI must satisfy the normwise tolerance
||C - C_ref||_F / || |A| |B| ||_F <= 4 k 2^-104 (f128) stated for this path.
Sizes cover ragged edges of every tile shape (1, 2, 3, 17, 63, 65, 127, 129,
255, 257) plus zeros, cancellation and wide exponent ranges.
"""
import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import dense_dd, dd_to_qd, gemm_operands

pytestmark = pytest.mark.gpu


def normwise_err(c, cref, a_abs_b_abs):
    d = (c[..., 0] - cref[..., 0]) + (c[..., 1] - cref[..., 1])
    return np.linalg.norm(d) / max(np.linalg.norm(a_abs_b_abs), 1e-300)


def abs_prod(a, b, atb):
    A = np.abs(a[..., 0] + a[..., 1])
    B = np.abs(b[..., 0] + b[..., 1])
    return (A.T if atb else A) @ B


SHAPES = [(1, 1, 1), (2, 2, 2), (3, 5, 7), (17, 63, 65), (65, 17, 129), (127, 129, 63), (130, 257, 255),
          (64, 64, 16), (257, 65, 300)]


@pytest.mark.parametrize("atb", [False, True])
@pytest.mark.parametrize("m,n,k", SHAPES)
def test_f128_plain_bitexact(gpu, m, n, k, atb):
    a, b = gemm_operands(m, n, k, seed=m * 1000 + n * 10 + k, atb=atb)
    c = gpu.f128_gemm(a, b, m, n, k, gpu.PLAIN, atb)
    ref = O.gemm(a, b, m, n, k, atb=atb)
    assert np.array_equal(c, ref)


def test_f128_plain_reference_kats(gpu):
    f = lambda v: np.stack([np.asarray(v, float), np.zeros(len(v))], -1)
    c = gpu.f128_gemm(f([1, 2, 3, 4]).reshape(2, 2, 2), f([5, 6, 7, 8]).reshape(2, 2, 2), 2, 2, 2)
    assert np.array_equal(c[..., 0].ravel(), [19, 22, 43, 50])  # linalg.rs:437-447
    a = f([1, 2, 3, 4, 5, 6]).reshape(3, 2, 2)
    b = f(range(1, 13)).reshape(3, 4, 2)
    at = f([1, 3, 5, 2, 4, 6]).reshape(2, 3, 2)
    assert np.array_equal(gpu.f128_gemm(at, b, 2, 4, 3), gpu.f128_gemm(a, b, 2, 4, 3, atb=True))


@pytest.mark.parametrize("atb", [False, True])
@pytest.mark.parametrize("m,n,k", SHAPES + [(300, 520, 1030)])
def test_f128_ozaki_tolerance(gpu, m, n, k, atb):
    a, b = gemm_operands(m, n, k, seed=7 + m + n + k, atb=atb)
    c = gpu.f128_gemm(a, b, m, n, k, gpu.OZAKI, atb)
    ref = O.gemm(a, b, m, n, k, atb=atb)
    err = normwise_err(c, ref, abs_prod(a, b, atb))
    assert err <= 4 * k * 2.0 ** -104, err


def test_f128_ozaki_wide_exponents_and_zeros(gpu):
    rng = np.random.default_rng(3)
    m, n, k = 70, 90, 150
    a = dense_dd(m, k, seed=11)
    b = dense_dd(k, n, seed=12)
    a *= (2.0 ** rng.integers(-300, 300, size=(m, 1)))[..., None]  # per-row scales
    b *= (2.0 ** rng.integers(-300, 300, size=(1, n)))[..., None]  # per-column scales
    a[5] = 0.0          # an all-zero row
    b[:, 7] = 0.0       # an all-zero column
    a[9, :] = a[10, :]  # two equal rows
    c = gpu.f128_gemm(a, b, m, n, k, gpu.OZAKI)
    ref = O.gemm(a, b, m, n, k)
    assert np.all(c[5] == 0.0) and np.all(c[:, 7] == 0.0)
    # row/column scaling makes the error bound entrywise in |A||B|
    ab = abs_prod(a, b, False)
    d = np.abs((c[..., 0] - ref[..., 0]) + (c[..., 1] - ref[..., 1]))
    assert np.all(d <= 4 * k * 2.0 ** -104 * ab + 1e-300)


@pytest.mark.parametrize("atb", [False, True])
@pytest.mark.parametrize("m", [70, 600])
def test_f128_ozaki_nonfinite_rows_and_columns(gpu, m, atb):
    """An inf or NaN limb in a row of op(A) or a column of B makes that row or
    column of C NaN (the chosen path's scaling has no finite exponent for it);
    every other entry is the finite product, within the entrywise bound. m = 600
    takes the host-pointer path's streamed A panels."""
    n, k = 90, 150
    a = dense_dd(k, m, seed=31) if atb else dense_dd(m, k, seed=31)
    b = dense_dd(k, n, seed=32)
    bad_rows, bad_cols = [3, 5, 7], [2, 6]
    at = (lambda r, p: (p, r)) if atb else (lambda r, p: (r, p))
    a[at(3, 10)][0] = np.nan        # NaN high limb
    a[at(5, 0)][0] = np.inf         # inf high limb
    a[at(7, 20)][1] = -np.inf       # non-finite low limb only
    b[4, 2, 0] = np.inf
    b[8, 6, 1] = np.nan
    c = gpu.f128_gemm(a, b, m, n, k, gpu.OZAKI, atb)
    assert np.all(np.isnan(c[bad_rows, :, 0])) and np.all(np.isnan(c[:, bad_cols, 0]))
    # the other entries against the oracle on the inputs with the bad rows and columns cleared
    a0, b0 = a.copy(), b.copy()
    for r in bad_rows:
        if atb:
            a0[:, r] = 0.0
        else:
            a0[r] = 0.0
    b0[:, bad_cols] = 0.0
    ref = O.gemm(a0, b0, m, n, k, atb=atb)
    good_r = np.setdiff1d(np.arange(m), bad_rows)
    good_c = np.setdiff1d(np.arange(n), bad_cols)
    cg, rg = c[np.ix_(good_r, good_c)], ref[np.ix_(good_r, good_c)]
    assert np.all(np.isfinite(cg))
    ab = abs_prod(a0, b0, atb)[np.ix_(good_r, good_c)]
    d = np.abs((cg[..., 0] - rg[..., 0]) + (cg[..., 1] - rg[..., 1]))
    assert np.all(d <= 4 * k * 2.0 ** -104 * ab + 1e-300)


@pytest.mark.parametrize("k", [128, 129, 600000])
def test_f128_ozaki_moduli_count_boundaries(gpu, k):
    """k = 128 / 129 straddle the step from 29 to 30 moduli; k = 600000 needs 32
    (and 19 k-chunks of the unsigned residue GEMM): every moduli count the
    tensor-core residue and CRT kernels are built for with k up to 2^20."""
    m = n = 16
    a, b = gemm_operands(m, n, k, seed=41 + k)
    c = gpu.f128_gemm(a, b, m, n, k, gpu.OZAKI)
    ref = O.gemm(a, b, m, n, k)
    err = normwise_err(c, ref, abs_prod(a, b, False))
    assert err <= 4 * k * 2.0 ** -104, err


def test_f128_ozaki_cancellation(gpu):
    """C = A B with B = [x, -x]: the two halves must cancel to (near) zero."""
    m, k = 40, 200
    a = dense_dd(m, k, seed=21)
    x = dense_dd(k, 8, seed=22)
    b = np.concatenate([x, -x], axis=1)
    c = gpu.f128_gemm(a, b, m, 16, k, gpu.OZAKI)
    s = (c[:, :8, 0] + c[:, 8:, 0]) + (c[:, :8, 1] + c[:, 8:, 1])
    assert np.all(s == 0.0)


@pytest.mark.parametrize("atb", [False, True])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (3, 5, 7), (17, 33, 20), (40, 31, 37)])
def test_f256_plain_bitexact(gpu, m, n, k, atb):
    a, b = gemm_operands(m, n, k, seed=5 + m, atb=atb)
    a4, b4 = dd_to_qd(a), dd_to_qd(b)
    a4[..., 2] = a4[..., 1] * 2.0 ** -60  # fill the low limbs too
    c = gpu.f256_gemm(a4, b4, m, n, k, gpu.PLAIN, atb)
    ref = O.mf_gemm(4, a4, b4, m, n, k, atb=atb)
    assert np.array_equal(c, ref)


def test_zero_sizes_and_nulls(gpu):
    e = np.zeros((0, 0, 2))
    assert gpu.f128_gemm(e, e, 0, 0, 0).shape == (0, 0, 2)
    c = gpu.f128_gemm(np.zeros((3, 0, 2)), np.zeros((0, 4, 2)), 3, 4, 0)
    assert np.all(c == 0.0)
    with pytest.raises(gpu.HPError) as ei:
        gpu.check(gpu.lib().hp_f128_gemm(None, None, None, 2, 2, 2, 0))
    assert ei.value.code == gpu.HP_ERR_INVALID_ARG
    with pytest.raises(gpu.HPError):
        gpu.f128_gemm(np.zeros((2, 2, 2)), np.zeros((2, 2, 2)), 2, 2, 2, mode=7)


def test_device_pointer_form(gpu):
    import torch

    m, n, k = 96, 80, 70
    a, b = gemm_operands(m, n, k, seed=99)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    dc = torch.empty((m, n, 2), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    gpu.f128_gemm_dev(da, db, dc, m, n, k, gpu.PLAIN, stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(dc.cpu().numpy(), O.gemm(a, b, m, n, k))


def qd_operand(rows, cols, seed):
    """Full 4-limb f256 entries: a dd entry plus two lower limbs."""
    x = dense_dd(rows, cols, seed=seed)
    y = dense_dd(rows, cols, seed=seed + 1000)
    q = np.zeros((rows, cols, 4))
    q[..., :2] = x
    q[..., 2] = y[..., 0] * np.abs(x[..., 1]) * 2.0 ** -53
    q[..., 3] = y[..., 1] * np.abs(x[..., 1]) * 2.0 ** -53
    return q


def qd_normwise_err(c, ref, a, b, atb):
    d = ((c[..., 0] - ref[..., 0]) + (c[..., 1] - ref[..., 1])) + ((c[..., 2] - ref[..., 2]) + (c[..., 3] - ref[..., 3]))
    A = np.abs(a[..., 0])
    B = np.abs(b[..., 0])
    return np.linalg.norm(d) / np.linalg.norm((A.T if atb else A) @ B)


@pytest.mark.parametrize("atb", [False, True])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (3, 5, 7), (17, 33, 20), (70, 40, 130)])
def test_f256_ozaki_tolerance(gpu, m, n, k, atb):
    a = qd_operand(k, m, 31) if atb else qd_operand(m, k, 31)
    b = qd_operand(k, n, 37)
    c = gpu.f256_gemm(a, b, m, n, k, gpu.OZAKI, atb)
    ref = O.mf_gemm(4, a, b, m, n, k, atb=atb)
    err = qd_normwise_err(c, ref, a, b, atb)
    assert err <= 4 * k * 2.0 ** -208, err


def test_f256_ozaki_exact_small_integers(gpu):
    """Integer matrices: the f256 Ozaki product is exact."""
    rng = np.random.default_rng(9)
    m, n, k = 20, 30, 40
    A = np.zeros((m, k, 4))
    B = np.zeros((k, n, 4))
    A[..., 0] = rng.integers(-1000, 1000, (m, k))
    B[..., 0] = rng.integers(-1000, 1000, (k, n))
    c = gpu.f256_gemm(A, B, m, n, k, gpu.OZAKI)
    assert np.array_equal(c[..., 0], A[..., 0] @ B[..., 0]) and np.all(c[..., 1:] == 0)


def qd_abs_prod(a, b, atb):
    A = np.abs(a[..., 0])
    return (A.T if atb else A) @ np.abs(b[..., 0])


def qd_entry_err(c, ref):
    return np.abs(((c[..., 0] - ref[..., 0]) + (c[..., 1] - ref[..., 1])) + ((c[..., 2] - ref[..., 2]) + (c[..., 3] - ref[..., 3])))


@pytest.mark.parametrize("atb", [False, True])
def test_f256_ozaki_ragged_tiles(gpu, atb):
    """Rows and columns over several 128-entry CRT tiles and 128-row residue
    tiles, none a multiple of the tile sizes: every entry within the
    entrywise bound 4 k 2^-208 |A| |B|."""
    m, n, k = 140, 300, 150
    a = qd_operand(k, m, 41) if atb else qd_operand(m, k, 41)
    b = qd_operand(k, n, 43)
    c = gpu.f256_gemm(a, b, m, n, k, gpu.OZAKI, atb)
    ref = O.mf_gemm(4, a, b, m, n, k, atb=atb)
    assert np.all(qd_entry_err(c, ref) <= 4 * k * 2.0 ** -208 * qd_abs_prod(a, b, atb) + 1e-300)


@pytest.mark.parametrize("k", [1, 128, 129, 16384])
def test_f256_ozaki_moduli_count_boundaries(gpu, k):
    """The f256 GEMM needs 28 moduli at k = 1, 29 up to k = 128, 30 from 129
    (to 8192) and 31 from 16384 (to 2^20): each count its tensor-core
    residue and CRT kernels are built for."""
    m, n = 8, 12
    a = qd_operand(m, k, 51)
    b = qd_operand(k, n, 53)
    c = gpu.f256_gemm(a, b, m, n, k, gpu.OZAKI)
    ref = O.mf_gemm(4, a, b, m, n, k)
    assert np.all(qd_entry_err(c, ref) <= 4 * k * 2.0 ** -208 * qd_abs_prod(a, b, False) + 1e-300)


@pytest.mark.parametrize("atb", [False, True])
def test_f256_ozaki_nonfinite_rows_and_columns(gpu, atb):
    """An inf or NaN limb in a row of op(A) or a column of B makes that row or
    column of the f256 product NaN; the other entries are the finite product."""
    m, n, k = 70, 140, 60
    a = qd_operand(k, m, 61) if atb else qd_operand(m, k, 61)
    b = qd_operand(k, n, 63)
    bad_rows, bad_cols = [3, 5, 69], [2, 130]
    at = (lambda r, p: (p, r)) if atb else (lambda r, p: (r, p))
    a[at(3, 10)][0] = np.nan
    a[at(5, 0)][2] = np.inf        # a lower limb only
    a[at(69, 59)][0] = -np.inf
    b[4, 2, 3] = np.nan
    b[8, 130, 0] = np.inf
    c = gpu.f256_gemm(a, b, m, n, k, gpu.OZAKI, atb)
    assert np.all(np.isnan(c[bad_rows, :, 0])) and np.all(np.isnan(c[:, bad_cols, 0]))
    a0, b0 = a.copy(), b.copy()
    for r in bad_rows:
        if atb:
            a0[:, r] = 0.0
        else:
            a0[r] = 0.0
    b0[:, bad_cols] = 0.0
    ref = O.mf_gemm(4, a0, b0, m, n, k, atb=atb)
    good_r = np.setdiff1d(np.arange(m), bad_rows)
    good_c = np.setdiff1d(np.arange(n), bad_cols)
    cg, rg = c[np.ix_(good_r, good_c)], ref[np.ix_(good_r, good_c)]
    assert np.all(np.isfinite(cg))
    ab = qd_abs_prod(a0, b0, atb)[np.ix_(good_r, good_c)]
    assert np.all(qd_entry_err(cg, rg) <= 4 * k * 2.0 ** -208 * ab + 1e-300)


@pytest.mark.parametrize("atb", [False, True])
def test_f128_ozaki_long_k_chunks(gpu, atb):
    """k beyond one accumulation chunk of the unsigned residue GEMM (32768):
    the second chunk adds into the first's residues modulo m."""
    m, n, k = 5, 9, 40000
    a, b = gemm_operands(m, n, k, seed=99, atb=atb)
    c = gpu.f128_gemm(a, b, m, n, k, gpu.OZAKI, atb)
    ref = O.gemm(a, b, m, n, k, atb=atb)
    err = normwise_err(c, ref, abs_prod(a, b, atb))
    assert err <= 4 * k * 2.0 ** -104, err


@pytest.mark.parametrize("atb", [False, True])
@pytest.mark.parametrize("m,n,k", [(512, 130, 200), (700, 257, 129), (1100, 64, 300), (2050, 33, 65),
                                   (600, 1100, 70), (1024, 2048, 130), (530, 1024, 129)])
def test_f128_ozaki_host_pipeline_matches_device(gpu, m, n, k, atb):
    """Host-pointer chosen GEMMs with m >= 512 run op(A) in row panels (with
    atb, A's column panels copied into compact k x rows matrices) and, for
    n >= 1024, B and C in two column panels (copies overlapped with the
    blocks' kernels); every entry must carry the bits of the one-shot
    device-pointer path, ragged last panels included, and the normwise
    tolerance against the oracle."""
    import torch

    a, b = gemm_operands(m, n, k, seed=7 + m, atb=atb)
    c_host = gpu.f128_gemm(a, b, m, n, k, gpu.OZAKI, atb)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    dc = torch.empty((m, n, 2), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    gpu.f128_gemm_dev(da, db, dc, m, n, k, gpu.OZAKI, atb=atb, stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(c_host, dc.cpu().numpy())
    if m in (700, 600):
        err = normwise_err(c_host, O.gemm(a, b, m, n, k, atb=atb), abs_prod(a, b, atb))
        assert err <= 4 * k * 2.0 ** -104, err


def test_f128_ozaki_host_column_panels_nonfinite(gpu):
    """The host pipeline's second column panel carries its own column
    exponents: a NaN column there, an inf row, and every other entry equal bit
    for bit to the one-shot device-pointer path."""
    import torch

    m, n, k = 600, 1100, 60
    a, b = gemm_operands(m, n, k, seed=77)
    a[11, 5, 0] = np.inf
    b[7, 1050, 1] = np.nan
    c_host = gpu.f128_gemm(a, b, m, n, k, gpu.OZAKI)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    dc = torch.empty((m, n, 2), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    gpu.f128_gemm_dev(da, db, dc, m, n, k, gpu.OZAKI, stream=s.cuda_stream)
    s.synchronize()
    assert np.all(np.isnan(c_host[11, :, 0])) and np.all(np.isnan(c_host[:, 1050, 0]))
    assert np.array_equal(c_host, dc.cpu().numpy(), equal_nan=True)


@pytest.mark.parametrize("atb", [False, True])
@pytest.mark.parametrize("m,n,k", [(512, 130, 60), (600, 1100, 70), (1024, 1024, 129), (530, 257, 200)])
def test_f256_ozaki_host_pipeline_matches_device(gpu, m, n, k, atb):
    """Host-pointer chosen f256 GEMMs with m >= 512 stream op(A) in row panels
    and, for n >= 1024, B and C in two column panels; every entry must carry
    the bits of the one-shot device-pointer path, and one shape is checked
    against the oracle's mf_gemm at the entrywise bound 4 k 2^-208 |A||B|."""
    import torch

    a = qd_operand(k, m, 71 + m) if atb else qd_operand(m, k, 71 + m)
    b = qd_operand(k, n, 73 + n)
    c_host = gpu.f256_gemm(a, b, m, n, k, gpu.OZAKI, atb)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    dc = torch.empty((m, n, 4), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    gpu.f256_gemm_dev(da, db, dc, m, n, k, gpu.OZAKI, atb=atb, stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(c_host, dc.cpu().numpy())
    if (m, n) == (600, 1100):
        ref = O.mf_gemm(4, a, b, m, n, k, atb=atb)
        assert np.all(qd_entry_err(c_host, ref) <= 4 * k * 2.0 ** -208 * qd_abs_prod(a, b, atb) + 1e-300)
