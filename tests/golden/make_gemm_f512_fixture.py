"""Generates the f512 reference entries of the benchmark GEMMs.

Inputs are the benchmark's operands (quadprec_b200.workloads.gemm_operands,
SplitMix64 seed 0, full double-double entries): C = A B and C = A^T B at
m = n = k = 2048 in f128, and the f256 C = A B at m = n = k = 1024 (the same
generator, limb-extended). The sample is 4096 entries (i, j) drawn from
SplitMix64 seed 7 plus two full rows (0 and m - 1), in the order of
quadprec_b200.workloads.sample_index (which regenerates them). Each entry is
computed by the oracle's MultiFloat<8> dot product of the exactly promoted
inputs (oracle.gemm_entries_f512) and stored as its 3 (f128 cases) or 4
(f256 case) leading limbs.

Run from the repository root:  python tests/golden/make_gemm_f512_fixture.py
Output: tests/golden/gemm_f512_sample.npz
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from quadprec_b200.workloads import dd_to_qd, gemm_operands, sample_index  # noqa: E402

CASES = {"f128_gemm_2048": (2048, False, 2), "f128_gemm_atb_2048": (2048, True, 2), "f256_gemm_1024": (1024, False, 4)}


def main():
    out, meta = {}, {"sample": "4096 SplitMix64(seed 7) entries + rows 0 and m-1", "cases": {}}
    for name, (s, atb, limbs) in CASES.items():
        t0 = time.time()
        a, b = gemm_operands(s, s, s, seed=0, atb=atb)
        if limbs == 4:
            a, b = dd_to_qd(a), dd_to_qd(b)
        idx = sample_index(s, s)
        c, _ = oracle.gemm_entries_f512(a, b, s, s, s, idx, atb=atb)
        out[name] = c[:, :limbs + 1] if limbs == 2 else c
        meta["cases"][name] = {"m": s, "n": s, "k": s, "atb": atb, "entries": len(idx),
                               "seconds": time.time() - t0, "threads": oracle.num_threads()}
    np.savez_compressed(os.path.join(HERE, "gemm_f512_sample.npz"), meta=json.dumps(meta), **out)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
