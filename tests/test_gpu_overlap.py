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


def random_cart_basis(nsh, seed):
    """Shells of kinds S, P, D, F (l = 0..3) with 1-3 primitives, exponents
    spanning diffuse and tight, so that all three screening tiers occur."""
    rng = np.random.default_rng(seed)
    ls = [int(x) for x in rng.integers(0, 4, size=nsh)]
    cen = rng.uniform(-6, 6, size=(nsh, 3))
    al, co = [], []
    for s in range(nsh):
        k = int(rng.integers(1, 4))
        a = 10.0 ** rng.uniform(-2, 2, size=k)
        al.append(np.array(a))
        co.append(rng.uniform(0.1, 1.0, size=k) * np.array([_norm(x) for x in a]))
    return ls, cen, al, co


@pytest.mark.parametrize("nsh", [1, 4, 60, 211])
def test_obara_saika_bases_match_oracle(gpu, nsh):
    """assemble_overlap_mixed with P/D/F shells (Obara-Saika, integral.rs:144-352):
    the same tiers as the oracle, values to the last ulps of f64 (CUDA's exp)."""
    ls, cen, al, co = random_cart_basis(nsh, seed=100 + nsh)
    s, tiers = gpu.assemble_overlap(ls, cen, al, co)
    so, to = O.assemble_overlap(ls, cen, al, co)
    assert np.array_equal(tiers, to), (tiers, to)
    assert s.shape == so.shape
    assert np.allclose(s, so, rtol=1e-13, atol=1e-16 * max(1.0, np.abs(so).max()))
    assert np.array_equal(s == 0.0, so == 0.0)
    if nsh >= 60:
        assert to[0] > 0 and to[1] > 0 and to[2] > 0


def test_obara_saika_s_only_equals_s_assembly(gpu):
    cen, al, co = random_s_basis(40, seed=5)
    s1, t1 = gpu.assemble_overlap([0] * 40, cen, [np.array(a) for a in al], [np.array(c) for c in co])
    s2, t2 = gpu.assemble_overlap_s(cen, al, co)
    assert np.array_equal(s1, s2) and list(t1) == [t2["f64_pairs"], t2["f128_pairs"], t2["skipped_pairs"]]


def test_obara_saika_rejects_unknown_kinds(gpu):
    with pytest.raises(gpu.HPError):
        gpu.assemble_overlap([4], [[0.0, 0.0, 0.0]], [np.array([1.0])], [np.array([1.0])])
