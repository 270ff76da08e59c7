"""Generates the f512 reference solutions of a sample of the 4096-system batch.

The batch is the benchmark's (quadprec_b200.workloads.batched_overlap_systems,
count 4096, seed 0: n in [16, 384]). For every system the oracle evaluates the
f128 overlap matrix S (bit-identical to the GPU's hp_overlap_norm_dd), factors
it with the restated f128 cholesky (crates/quad/src/linalg.rs:42-96) and takes
cond_estimate (linalg.rs:185-194) as its kappa; systems whose f128 factor
fails get kappa = inf. The sample is 48 systems at evenly spaced ranks of the
size order (the smallest and the largest n included) plus the 16 largest
kappa, 64 distinct systems in all. Each sampled S is promoted exactly to
MultiFloat<8>, factored with mf_cholesky<8> (multifloat/linalg.rs:89-141) and
solved with mf_cholesky_solve<8> (:145-172); x* is stored rounded to 4 limbs.

Run from the repository root:  python tests/golden/make_batched_fixture.py
Output: tests/golden/batched_4096_sample.npz (index, n, kappa, offsets of the
sampled systems in x_star, x_star, meta).
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from quadprec_b200.workloads import batched_overlap_systems  # noqa: E402

N_SPREAD, N_KAPPA = 48, 16


def system(B, s):
    o, e = int(B["offsets"][s]), int(B["offsets"][s + 1])
    return B["centers"][o:e], B["alpha"][o:e], B["b"][o:e]


def kappa_f128(cen, alpha):
    n = len(alpha)
    S = oracle.overlap_norm_dd(cen, alpha)
    try:
        L = oracle.cholesky(S, n)
    except oracle.CholeskyError:
        return float("inf")
    return float(oracle.cond_estimate(L, n))


def main():
    t0 = time.time()
    B = batched_overlap_systems(4096, seed=0)
    ns = np.diff(B["offsets"])
    kap = np.array([kappa_f128(*system(B, s)[:2]) for s in range(len(ns))])
    order = np.argsort(ns, kind="stable")
    spread = order[np.round(np.linspace(0, len(ns) - 1, N_SPREAD)).astype(int)]
    chosen = list(dict.fromkeys(spread.tolist()))
    for s in np.argsort(-kap, kind="stable"):
        if len(chosen) >= N_SPREAD + N_KAPPA:
            break
        if int(s) not in chosen:
            chosen.append(int(s))
    chosen = np.array(sorted(chosen), dtype=np.int64)
    xs, offs = [], [0]
    for s in chosen:
        cen, alpha, b = system(B, s)
        n = len(alpha)
        S8 = np.zeros((n, n, 8))
        S8[..., :2] = oracle.overlap_norm_dd(cen, alpha)
        L8 = oracle.mf_cholesky(8, S8, n)
        b8 = np.zeros((n, 8))
        b8[:, 0] = b
        xs.append(oracle.mf_cholesky_solve(8, L8, b8, n)[:, :4])
        offs.append(offs[-1] + n)
    meta = {"batch": "batched_overlap_systems(4096, seed=0)", "sample": len(chosen), "spread": N_SPREAD,
            "largest_kappa": N_KAPPA, "n_min": int(ns[chosen].min()), "n_max": int(ns[chosen].max()),
            "kappa_max_finite": float(kap[chosen][np.isfinite(kap[chosen])].max()),
            "kappa_inf": int(np.isinf(kap[chosen]).sum()), "seconds": time.time() - t0,
            "threads": oracle.num_threads(),
            "precision": "MultiFloat<8> (f512) oracle, stored as 4 limbs; kappa = f128 cond_estimate"}
    np.savez_compressed(os.path.join(HERE, "batched_4096_sample.npz"), index=chosen, n=ns[chosen],
                        kappa=kap[chosen], x_offsets=np.array(offs, dtype=np.int64),
                        x_star=np.concatenate(xs), meta=json.dumps(meta))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
