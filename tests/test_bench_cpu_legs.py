"""CPU checks of the bench's CPU-baseline helpers (no GPU): the batched
Jacobi baseline runs the oracle's jacobi_eigen (the reference's cyclic
order) on a size-ordered sample, scales the sample's rate to the whole set
by sum n^3, and compares eigenvalues with the GPU's after sorting both."""
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402
import oracle  # noqa: E402
from quadprec_b200.workloads import overlap_spd_problem  # noqa: E402


def _matrices(count):
    mats, ns, evs = [], [], []
    for seed in range(count):
        cen, alpha, _ = overlap_spd_problem(1, 2, 2 + seed % 3, seed=seed)
        n = len(alpha)
        S = oracle.overlap_norm_dd(cen, alpha)
        ev, _, _ = oracle.jacobi_eigen(S, n, 200)
        mats.append(np.asarray(S).reshape(-1))
        ns.append(n)
        evs.append(ev)
    return mats, np.array(ns), evs


def test_jacobi_baseline_matches_permuted_eigenvalues():
    mats, ns, evs = _matrices(6)
    gpu_like = np.concatenate([ev[::-1].reshape(-1) for ev in evs])  # another order, same values
    out = bench.cpu_jacobi_sample(np.concatenate(mats), ns, gpu_like, stride=2)
    assert out["max_eigenvalue_diff_over_max_vs_gpu"] == 0.0
    assert out["kind"] == "port" and out["value"] > 0 and out["value_1_core"] > 0
    assert "3 of 6 matrices" in out["sample"]


def test_jacobi_baseline_reports_a_wrong_eigenvalue():
    mats, ns, evs = _matrices(4)
    bad = [ev.copy() for ev in evs]
    top = int(np.argmax(np.abs(bad[0][:, 0])))
    bad[0][top, 1] += bad[0][top, 0] * 1e-20  # the first matrix's largest eigenvalue off by 1e-20 (low limb)
    out = bench.cpu_jacobi_sample(np.concatenate(mats), ns, np.concatenate([e.reshape(-1) for e in bad]), stride=1)
    assert 1e-22 < out["max_eigenvalue_diff_over_max_vs_gpu"] < 1e-18
