"""Generates the f512 reference solutions of the overlap SPD workloads.

For a lattice basis (quadprec_b200.workloads.overlap_spd_problem) the f128
problem matrix S is evaluated by the oracle (bit-identical to the GPU's
hp_overlap_norm_dd), promoted exactly to MultiFloat<8>, factored with the
oracle's mf_cholesky<8> (crates/quad/src/multifloat/linalg.rs:89-141) and
solved with mf_cholesky_solve<8> (:145-172). The solution x* is stored
rounded to 4 limbs (f256), which is exact to ~1e-63 relative.

Run from the repository root:  python tests/golden/make_overlap_fixtures.py [name ...]
Outputs tests/golden/<name>.npz (x_star, b, meta).
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from quadprec_b200.workloads import overlap_spd_problem  # noqa: E402

CASES = {
    "overlap_2x2x2": (2, 2, 2),      # n = 32
    "overlap_3x4x5": (3, 4, 5),      # n = 240
    "overlap_5x10x10": (5, 10, 10),  # n = 2000, the benchmark workload
}


def make(name):
    nx, ny, nz = CASES[name]
    cen, alpha, b = overlap_spd_problem(nx, ny, nz, seed=0)
    n = len(alpha)
    t0 = time.time()
    S = oracle.overlap_norm_dd(cen, alpha)
    S8 = np.zeros((n, n, 8))
    S8[..., :2] = S
    L8 = oracle.mf_cholesky(8, S8, n)
    b8 = np.zeros((n, 8))
    b8[:, 0] = b
    x8 = oracle.mf_cholesky_solve(8, L8, b8, n)
    meta = {"name": name, "lattice": [nx, ny, nz], "n": n, "seed": 0, "seconds": time.time() - t0,
            "threads": oracle.num_threads(), "precision": "MultiFloat<8> (f512) oracle, stored as 4 limbs"}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), x_star=x8[:, :4], b=b, meta=json.dumps(meta))
    print(json.dumps(meta))


if __name__ == "__main__":
    for nm in (sys.argv[1:] or list(CASES)):
        make(nm)
