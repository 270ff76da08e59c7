"""GPU parity for overlap assembly (crates/overlap)."""
import math

import numpy as np
import pytest

import oracle as O
from quadprec_b200.workloads import overlap_lattice

pytestmark = pytest.mark.gpu


def _norm(alpha):
    return (2.0 * alpha / math.pi) ** 0.75


def random_s_basis(nsh, seed):
    rng = np.random.default_rng(seed)
    cen = rng.uniform(-6, 6, size=(nsh, 3))
    al, co = [], []
    for s in range(nsh):
        k = int(rng.integers(1, 4))
        a = 10.0 ** rng.uniform(-2, 2, size=k)
        al.append(list(a))
        co.append(list(rng.uniform(0.1, 1.0, size=k) * np.array([_norm(x) for x in a])))
    return cen, al, co


def test_h2_reference_case(gpu):  # assemble.rs:116-139
    al = [3.42525, 0.62391, 0.16886]
    co = [0.15433 * _norm(3.42525), 0.53533 * _norm(0.62391), 0.44463 * _norm(0.16886)]
    cen = np.array([[0.0, 0, 0], [1.4, 0, 0]])
    s, tiers = gpu.assemble_overlap_s(cen, [al, al], [co, co])
    so, to = O.assemble_overlap_s(cen, [al, al], [co, co])
    assert tiers == to and tiers["f128_pairs"] == 0
    assert 0.5 < s[0, 1] < 0.8 and np.allclose(s, so, rtol=1e-14, atol=0)


def test_diffuse_triggers_f128(gpu):  # assemble.rs:141-164
    al = [50.0, 0.04]
    co = [0.3 * _norm(50.0), 0.7 * _norm(0.04)]
    cen = np.array([[0.0, 0, 0], [2.0, 0, 0]])
    s, tiers = gpu.assemble_overlap_s(cen, [al, al], [co, co])
    so, to = O.assemble_overlap_s(cen, [al, al], [co, co])
    assert tiers == to and tiers["f128_pairs"] > 0
    assert np.allclose(s, so, rtol=1e-13, atol=1e-300)


@pytest.mark.parametrize("nsh", [1, 7, 150, 333])
def test_random_s_bases(gpu, nsh):
    cen, al, co = random_s_basis(nsh, seed=nsh)
    s, tiers = gpu.assemble_overlap_s(cen, al, co)
    so, to = O.assemble_overlap_s(cen, al, co)
    assert tiers == to
    # f64 exp differs from glibc's by at most a few ulps
    assert np.allclose(s, so, rtol=1e-13, atol=1e-300)
    assert np.array_equal(s == 0.0, so == 0.0)


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 2, 2), (3, 4, 5), (5, 10, 10)])
def test_overlap_norm_dd_bitexact(gpu, dims):
    cen, alpha = overlap_lattice(*dims, seed=sum(dims))
    s = gpu.overlap_norm_dd(cen, alpha)
    if len(alpha) <= 600:
        assert np.array_equal(s, O.overlap_norm_dd(cen, alpha))
    else:  # 2000 x 2000: compare a sample of rows
        ref = O.overlap_norm_dd(cen, alpha)
        assert np.array_equal(s, ref)
    n = len(alpha)
    assert np.array_equal(s[np.arange(n), np.arange(n)], np.tile([1.0, 0.0], (n, 1)))
