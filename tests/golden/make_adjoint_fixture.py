"""Generates the f256 finite-difference gradient of the n = 1000 adjoint workload.

Workload: quadprec_b200.workloads.overlap_spd_problem(5, 5, 10, seed=0), 250
jittered lattice centres x 4 exponents, b ~ N(0,1), L = b^T S^-1 b. The
sample is every parameter of 8 centres spread over the lattice: their 24
coordinates and the 32 log-exponents of their basis functions (56
parameters). Each derivative is a MultiFloat<4> central difference with
h = 1e-20 (oracle.fd_grad_f256: S assembled from the f256 formula, the
unperturbed block factored once by the restated mf_cholesky<4>, each
perturbed loss by block elimination), stored as 4 limbs.

Run from the repository root:  python tests/golden/make_adjoint_fixture.py
Output: tests/golden/adjoint_fd_1000.npz (centres, funcs, gR, ga, meta).
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

LATTICE = (5, 5, 10)
CENTRES = [0, 37, 74, 111, 148, 185, 222, 249]
H = 1e-20


def main():
    t0 = time.time()
    cen, alpha, b = overlap_spd_problem(*LATTICE, seed=0)
    n = len(alpha)
    co = np.arange(n) // 4
    gR, funcs, ga = oracle.fd_grad_f256(cen, alpha, b, co, CENTRES, h=H)
    meta = {"lattice": list(LATTICE), "n": n, "centres": CENTRES, "h": H, "parameters": int(gR.size // 4 + len(funcs)),
            "seconds": time.time() - t0, "threads": oracle.num_threads(),
            "precision": "MultiFloat<4> central differences, stored as 4 limbs"}
    np.savez_compressed(os.path.join(HERE, "adjoint_fd_1000.npz"), centres=np.array(CENTRES), funcs=funcs, gR=gR,
                        ga=ga, meta=json.dumps(meta))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
