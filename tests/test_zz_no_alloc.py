"""hp_f128_gemm_noalloc_dev: the allocation-free Ozaki f128 GEMM.

Called through the C ABI on device buffers and compared with the allocating
entry point hp_f128_gemm_dev (HP_MODE_OZAKI) on two calls in a row, so that
the second call runs on scratch the first one left behind. Both must agree
within the Ozaki tolerance ||C1 - C2||_F / || |A| |B| ||_F <= 4 k 2^-104.
Kept in the last test file so it also runs after every other GPU test.
"""
import ctypes

import numpy as np
import pytest

from quadprec_b200.workloads import gemm_operands

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 64 << 20


def _dev(x):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)).to("cuda")


def _call_noalloc(gpu, a, b, c, m, n, k):
    import torch

    s = torch.cuda.current_stream().cuda_stream
    return gpu.lib().hp_f128_gemm_noalloc_dev(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, n, k, s)


def _err(gpu):
    return (gpu.lib().hp_last_error() or b"").decode()


def _normwise(c1, c2, a, b):
    d = (c1[..., 0] - c2[..., 0]) + (c1[..., 1] - c2[..., 1])
    ab = np.abs(a[..., 0] + a[..., 1]) @ np.abs(b[..., 0] + b[..., 1])
    return np.linalg.norm(d) / max(np.linalg.norm(ab), 1e-300)


@pytest.mark.parametrize("shapes", [[(200, 300, 250), (257, 129, 520)], [(512, 512, 512), (33, 700, 65)]])
def test_noalloc_matches_allocating_gemm_twice(gpu, shapes):
    import torch

    for i, (m, n, k) in enumerate(shapes):
        a, b = gemm_operands(m, n, k, seed=1000 * i + m + n + k)
        da, db = _dev(a), _dev(b)
        c_noalloc = torch.full((m, n, 2), float("nan"), dtype=torch.float64, device="cuda")
        c_alloc = torch.empty_like(c_noalloc)
        assert _call_noalloc(gpu, da, db, c_noalloc, m, n, k) == gpu.HP_OK, _err(gpu)
        gpu.f128_gemm_dev(da, db, c_alloc, m, n, k, gpu.OZAKI, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        c1, c2 = c_noalloc.cpu().numpy(), c_alloc.cpu().numpy()
        assert np.isfinite(c1).all()
        err = _normwise(c1, c2, a, b)
        assert err <= 4 * k * 2.0 ** -104, (m, n, k, err)
        # the two entry points split their residue work over threads
        # differently, with the same arithmetic per entry: same bits
        assert np.array_equal(c1, c2), (m, n, k, int(np.sum(c1 != c2)))


def test_noalloc_rejects_sizes_beyond_scratch(gpu):
    import torch

    # 1024^3 needs about 3 x 29 MiB of residue planes: more than the scratch
    m = n = k = 1024
    a = torch.zeros((m, k, 2), dtype=torch.float64, device="cuda")
    b = torch.zeros((k, n, 2), dtype=torch.float64, device="cuda")
    c = torch.zeros((m, n, 2), dtype=torch.float64, device="cuda")
    rc = _call_noalloc(gpu, a, b, c, m, n, k)
    assert rc == gpu.HP_ERR_INVALID_ARG
    msg = _err(gpu)
    assert "scratch" in msg and str(SCRATCH_BYTES) in msg, msg
