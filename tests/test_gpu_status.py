"""Device-side waits that give up are reported by the call they happen in.

Every spin in the library's kernels is bounded by global time and, on giving
up, sets a bit in a status word instead of trapping. These tests make a wait
run out on purpose, without a fault: the diagnostic wavefront solve
(hp_debug_trsv_wavefront) solves one 64-row block row without publishing it,
so the rows after it wait for values that never come, with a 1 ms limit. The
call must return HP_ERR_TIMEOUT, and a normal call right after it must
succeed with the oracle's answer (the context stays usable). The status query
of the stream-ordered forms (hp_device_status) must read clean after calls
that completed.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def lower_factor(n, seed):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, n))
    A = B @ B.T / n + np.eye(n)
    a = np.zeros((n, n, 2))
    a[..., 0] = (A + A.T) / 2
    return O.cholesky(a, n), rng.standard_normal(n)


def rel(x, xs):
    d = (x[:, 0] - xs[:, 0]) + (x[:, 1] - xs[:, 1])
    return np.linalg.norm(d) / np.linalg.norm(xs[:, 0])


@pytest.mark.parametrize("upper_t", [False, True])
def test_withheld_block_times_out_then_solve_recovers(gpu, upper_t):
    n = 300  # 5 block rows, the last one ragged
    L, b = lower_factor(n, 41)
    bb = np.zeros((n, 2))
    bb[:, 0] = b
    rc, _ = gpu.debug_trsv_wavefront(L, bb, n, upper_t=upper_t, wait_ns=1_000_000, withheld_block=1 if not upper_t else 3)
    assert rc == gpu.HP_ERR_TIMEOUT, (rc, gpu.lib().hp_last_error())
    assert b"gave up" in gpu.lib().hp_last_error()
    rc, x = gpu.debug_trsv_wavefront(L, bb, n, upper_t=upper_t)
    assert rc == gpu.HP_OK, gpu.lib().hp_last_error()
    ref = O.backward_solve(L, bb, n) if upper_t else O.forward_solve(L, bb, n)
    assert rel(x, ref) <= 1e-28


def test_withheld_last_block_is_not_a_timeout(gpu):
    """Nothing waits for the last block row: withholding it times nothing out."""
    n = 200
    L, b = lower_factor(n, 42)
    bb = np.zeros((n, 2))
    bb[:, 0] = b
    rc, _ = gpu.debug_trsv_wavefront(L, bb, n, wait_ns=1_000_000, withheld_block=3)
    assert rc == gpu.HP_OK
    rc, _ = gpu.debug_trsv_wavefront(L, bb, n, withheld_block=4)
    assert rc == gpu.HP_ERR_INVALID_ARG


def test_device_status_clean_after_dev_gemms(gpu):
    import torch

    from quadprec_b200.workloads import gemm_operands

    m, n, k = 300, 200, 260
    a, b = gemm_operands(m, n, k, seed=5)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    dc = torch.empty((m, n, 2), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    gpu.f128_gemm_dev(da, db, dc, m, n, k, gpu.OZAKI, stream=s)
    gpu.f128_gemm_dev(da, db, dc, m, n, k, gpu.OZAKI, atb=False, stream=s)
    rc, bits = gpu.device_status(stream=s)
    assert (rc, bits) == (gpu.HP_OK, 0), gpu.lib().hp_last_error()
