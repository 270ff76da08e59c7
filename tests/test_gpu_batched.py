"""GPU batched overlap SPD solves and Jacobi eigensolves."""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import batched_overlap_systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_batch():
    return batched_overlap_systems(count=24, seed=3, n_min=16, n_max=64)


def test_batched_solves_match_f256_oracle(gpu, small_batch):
    B = small_batch
    x, st, it = gpu.spd_solve_batched(B)
    assert np.all(st == 0), st
    off = B["offsets"]
    for s in range(len(off) - 1):
        o, e = off[s], off[s + 1]
        n = e - o
        S = O.overlap_norm_dd(B["centers"][o:e], B["alpha"][o:e])
        S4 = np.zeros((n, n, 4))
        S4[..., :2] = S
        L4 = O.mf_cholesky(4, S4, n)
        b4 = np.zeros((n, 4))
        b4[:, 0] = B["b"][o:e]
        xs = O.mf_cholesky_solve(4, L4, b4, n)
        d = (xs[:, 0] - x[o:e, 0]) + (xs[:, 1] - x[o:e, 1]) + xs[:, 2]
        assert np.linalg.norm(d) / np.linalg.norm(xs[:, 0]) <= 1e-25, s


def test_autotuned_launch_shape_gives_the_same_bits(gpu, small_batch):
    """The autotuner picks the CTA size and CTAs per SM of the persistent
    solver; every candidate must compute the same bits. Compared with the
    search switched off (HP_AUTOTUNE=0: 512 threads, one CTA per SM) in a
    fresh process on the same batch."""
    x, st, it = gpu.spd_solve_batched(small_batch)
    threads, ctas = gpu.batched_config()
    assert threads in (256, 512, 1024) and 1 <= ctas <= 4, (threads, ctas)
    code = (
        "import sys, numpy as np, quadprec_b200 as hp\n"
        "from quadprec_b200.workloads import batched_overlap_systems\n"
        "B = batched_overlap_systems(count=24, seed=3, n_min=16, n_max=64)\n"
        "x, st, it = hp.spd_solve_batched(B)\n"
        "assert hp.batched_config() == (512, 1), hp.batched_config()\n"
        "sys.stdout.buffer.write(np.ascontiguousarray(x).tobytes() + st.tobytes() + it.tobytes())\n"
    )
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=repo, env={**os.environ, "HP_AUTOTUNE": "0"},
                         capture_output=True, timeout=600)
    assert out.returncode == 0, out.stderr.decode()[-2000:]
    nx = x.size * 8
    x0 = np.frombuffer(out.stdout[:nx], dtype=np.float64).reshape(x.shape)
    st0 = np.frombuffer(out.stdout[nx:nx + st.size * 4], dtype=np.int32)
    it0 = np.frombuffer(out.stdout[nx + st.size * 4:], dtype=np.int32)
    assert np.array_equal(x, x0) and np.array_equal(st, st0) and np.array_equal(it, it0)


def test_batched_flags_only_bad_systems(gpu, small_batch):
    """A non-SPD system (exponent made negative -> S_ii = nan/neg) fails alone."""
    B = {k: np.array(v, copy=True) for k, v in small_batch.items()}
    o = B["offsets"][5]
    B["centers"][o + 1] = B["centers"][o]      # duplicate basis function ->
    B["alpha"][o + 1] = B["alpha"][o]          # S exactly singular
    x, st, it = gpu.spd_solve_batched(B)
    assert st[5] != 0
    assert np.all(np.delete(st, 5) == 0)


def f128m(a):
    out = np.zeros(a.shape + (2,))
    out[..., 0] = a
    return out


def to_f64(x):
    return x[..., 0] + x[..., 1]


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 16, 33, 64, 81, 128])
def test_jacobi_matches_reference(gpu, n):
    rng = np.random.default_rng(n)
    m = rng.standard_normal((n, n))
    a = f128m((m + m.T) / 2.0)
    ev, vec, sw = gpu.f128_jacobi_eigen(a, n, 200)
    er, vr, swr = O.jacobi_eigen(a, n, 200)
    # eigenvalues agree to f128 rounding (order may differ)
    assert np.allclose(np.sort(to_f64(ev)), np.sort(to_f64(er)), rtol=0, atol=1e-26 * max(1.0, np.abs(m).max()))
    # rows are orthonormal eigenvectors: A v = lambda v
    A = to_f64(a)
    V = to_f64(vec)
    assert np.allclose(V @ V.T, np.eye(n), atol=1e-14)
    assert np.allclose(A @ V.T, V.T * to_f64(ev)[None, :], atol=1e-13)


def test_jacobi_reference_kats(gpu):  # linalg.rs:496-541
    ev, vec, _ = gpu.f128_jacobi_eigen(f128m(np.array([[2.0, 1], [1, 2]])), 2, 100)
    e = np.sort(to_f64(ev))
    assert abs(e[0] - 1) < 1e-28 and abs(e[1] - 3) < 1e-28
    ev, _, _ = gpu.f128_jacobi_eigen(f128m(np.eye(4)), 4, 10)
    assert np.all(np.abs(to_f64(ev) - 1.0) < 1e-30)
    ev, vec, _ = gpu.f128_jacobi_eigen(f128m(np.array([[4.0, 1, 0], [1, 3, 1], [0, 1, 2]])), 3, 200)
    assert abs(to_f64(ev).sum() - 9.0) < 1e-25
    with pytest.raises(gpu.HPError):
        gpu.f128_jacobi_eigen(f128m(np.array([[2.0, 1], [1, 2]])), 2, 0)


def test_batched_jacobi_on_overlap_matrices(gpu, small_batch):
    import torch

    B = small_batch
    off = B["offsets"]
    count = len(off) - 1
    dc = torch.from_numpy(np.ascontiguousarray(B["centers"])).cuda()
    da = torch.from_numpy(B["alpha"]).cuda()
    ns = np.diff(off)
    S = torch.empty(int((ns ** 2).sum()) * 2, dtype=torch.float64, device="cuda")
    gpu.check(gpu.lib().hp_overlap_norm_dd_batched_dev(count, off.ctypes.data, dc.data_ptr(), da.data_ptr(),
                                                       S.data_ptr(), 0))
    ev = torch.empty(int(off[-1]) * 2, dtype=torch.float64, device="cuda")
    vec = torch.empty_like(S)
    sw = torch.zeros(count, dtype=torch.int32, device="cuda")
    st = torch.zeros(count, dtype=torch.int32, device="cuda")
    gpu.check(gpu.lib().hp_f128_jacobi_eigen_batched_dev(count, off.ctypes.data, S.data_ptr(), 200, ev.data_ptr(),
                                                         vec.data_ptr(), sw.data_ptr(), st.data_ptr(), 0))
    torch.cuda.synchronize()
    assert int(st.abs().sum()) == 0
    Sh = S.cpu().numpy().reshape(-1, 2)
    evh = ev.cpu().numpy().reshape(-1, 2)
    m0 = 0
    for s in range(count):
        n = int(ns[s])
        Sm = Sh[m0:m0 + n * n].reshape(n, n, 2)
        ref = O.overlap_norm_dd(B["centers"][off[s]:off[s + 1]], B["alpha"][off[s]:off[s + 1]])
        assert np.array_equal(Sm, ref)
        w = np.sort(to_f64(evh[off[s]:off[s + 1]]))
        wr = np.sort(np.linalg.eigvalsh(to_f64(ref)))
        assert np.allclose(w, wr, atol=1e-12)
        m0 += n * n


def test_batched_jacobi_mixed_sizes(gpu):
    """A batch spanning both launches of the batched Jacobi (n > 80 first,
    largest first, then the rest with less shared memory per CTA): every
    matrix converges to eigenpairs of its own matrix, eigenvalues matching
    numpy's to f64 rounding, in the caller's order."""
    import torch

    ns = [5, 90, 40, 128, 81, 12, 2]
    rng = np.random.default_rng(5)
    mats = []
    for n in ns:
        m = rng.standard_normal((n, n))
        mats.append((m + m.T) / 2.0)
    off = np.zeros(len(ns) + 1, dtype=np.int64)
    off[1:] = np.cumsum(ns)
    A = np.concatenate([f128m(m).reshape(-1, 2) for m in mats])
    dA = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    ev = torch.empty((int(off[-1]), 2), dtype=torch.float64, device="cuda")
    vec = torch.empty_like(dA)
    sw = torch.zeros(len(ns), dtype=torch.int32, device="cuda")
    st = torch.zeros(len(ns), dtype=torch.int32, device="cuda")
    gpu.check(gpu.lib().hp_f128_jacobi_eigen_batched_dev(len(ns), off.ctypes.data, dA.data_ptr(), 200,
                                                         ev.data_ptr(), vec.data_ptr(), sw.data_ptr(),
                                                         st.data_ptr(), 0))
    torch.cuda.synchronize()
    assert int(st.abs().sum()) == 0
    evh, vh = to_f64(ev.cpu().numpy()), to_f64(vec.cpu().numpy())
    m0 = 0
    for s, (n, m) in enumerate(zip(ns, mats)):
        lam = evh[off[s]:off[s + 1]]
        V = vh[m0:m0 + n * n].reshape(n, n)  # rows are eigenvectors
        m0 += n * n
        assert np.allclose(np.sort(lam), np.linalg.eigvalsh(m), rtol=0, atol=1e-12 * max(1.0, np.abs(m).max()))
        assert np.allclose(V @ V.T, np.eye(n), atol=1e-13)
        assert np.allclose(m @ V.T, V.T * lam[None, :], atol=1e-12 * max(1.0, np.abs(m).max()))


def test_batched_solve_size_limit(gpu):
    """Systems beyond what a CTA's shared memory holds (n > 1163) are refused
    with HP_ERR_UNSUPPORTED, not launched."""
    B = batched_overlap_systems(count=1, seed=9, n_min=1168, n_max=1168)
    assert int(B["offsets"][-1]) == 1168
    with pytest.raises(gpu.HPError) as ei:
        gpu.spd_solve_batched(B)
    assert ei.value.code == gpu.HP_ERR_UNSUPPORTED


def _batch_of_sizes(sizes, seed0):
    """Batch whose system s is a one-system cluster of exactly sizes[s] functions."""
    parts = [batched_overlap_systems(count=1, seed=seed0 + s, n_min=n, n_max=n) for s, n in enumerate(sizes)]
    off = np.zeros(len(sizes) + 1, dtype=np.int64)
    off[1:] = np.cumsum(sizes)
    return {"offsets": off, "centers": np.concatenate([p["centers"] for p in parts]),
            "alpha": np.concatenate([p["alpha"] for p in parts]), "b": np.concatenate([p["b"] for p in parts])}


def test_batched_graph_replays_only_for_identical_offsets(gpu):
    """hp_spd_solve_batched_dev keeps one CUDA graph with device copies of the
    first call's offsets and queue order. A second call on the same buffers
    whose offsets differ only at entries a sparse sample of the array would
    skip (here offsets[3] and offsets[67] of 130 systems, total unchanged) must
    not replay the stale graph: its x must equal a fresh solve of the new
    batch, bit for bit."""
    import torch

    rng = np.random.default_rng(11)
    sizes1 = [int(4 * v) for v in rng.integers(4, 9, size=130)]
    sizes2 = list(sizes1)
    sizes2[2] += 8
    sizes2[3] -= 8 if sizes2[3] > 16 else -8
    sizes2[4] -= sizes2[2] + sizes2[3] - sizes1[2] - sizes1[3]  # offsets[4:] unchanged
    sizes2[66] += 4
    sizes2[67] -= 4
    assert all(16 <= n <= 48 for n in sizes2) and sum(sizes2) == sum(sizes1)
    B1, B2 = _batch_of_sizes(sizes1, 500), _batch_of_sizes(sizes2, 900)
    diff = np.nonzero(B1["offsets"] != B2["offsets"])[0]
    assert set(diff.tolist()) <= {3, 4, 67} and 3 in diff and 67 in diff, diff
    N = int(B1["offsets"][-1])
    dc = torch.empty((N, 3), dtype=torch.float64, device="cuda")
    da = torch.empty(N, dtype=torch.float64, device="cuda")
    db = torch.zeros((N, 2), dtype=torch.float64, device="cuda")
    dx = torch.empty((N, 2), dtype=torch.float64, device="cuda")
    dst = torch.empty(130, dtype=torch.int32, device="cuda")
    dit = torch.empty(130, dtype=torch.int32, device="cuda")
    offs = np.empty(131, dtype=np.int64)  # one host array, rewritten between the calls
    for B in (B1, B2):
        dc.copy_(torch.from_numpy(B["centers"]))
        da.copy_(torch.from_numpy(B["alpha"]))
        db[:, 0].copy_(torch.from_numpy(B["b"]))
        offs[:] = B["offsets"]
        gpu.check(gpu.lib().hp_spd_solve_batched_dev(130, offs.ctypes.data, dc.data_ptr(), da.data_ptr(),
                                                     db.data_ptr(), dx.data_ptr(), dst.data_ptr(), dit.data_ptr(),
                                                     1e-28, 10, 0))
        torch.cuda.synchronize()
        x_fresh, st_fresh, _ = gpu.spd_solve_batched(B)
        assert np.all(st_fresh == 0)
        assert np.array_equal(dst.cpu().numpy(), st_fresh)
        assert np.array_equal(dx.cpu().numpy(), x_fresh)
