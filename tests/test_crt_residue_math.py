"""The arithmetic of the f128 and f256 Ozaki GEMMs' tensor-core residue and CRT kernels
(ozaki.cu residue_tc_kernel, crt_tc_kernel), restated in Python and checked
with exact integers on the CPU, for every moduli count those kernels serve
(28..32):

* residues: an entry's scaled integer X, |X| < 2^109, offset to
  X' = X + 2^111, has bytes x_0..x_13 (and x_14 = 1, x_15 = 0); with the
  weights w_lb = 2^(8b) mod m_l (b < 14), w_l14 = -2^111 mod m_l, the sum
  S_l = sum_b x_b w_lb stays below 2^24, and S_l - m_l umulhi(S_l,
  ceil(2^32 / m_l)) is X mod m_l exactly;
* CRT: from the residues r_l of C, |C| <= M/4, the byte sums
  S_q = sum_l r_l byte_q(W_l) give the 16-bit limbs U_h of V = sum r_l W_l,
  the quotient estimate q = rint(top limbs * 2^192/M) is the exact
  (V - C) / M, the digits d_h = U_h - q M_h carried into balanced 48-bit
  chunks |b_k| <= 2^47 rebuild C exactly, and their double-double sum from
  the top (quick two-sums) is C to f128 accuracy;
* f256 CRT: two groups' chunks combine exactly into G1 2^105 + G2 as nine
  balanced chunks, whose four-limb sum is C to ~2^-206 (exactly below 2^150).
"""
import math
import random
from fractions import Fraction

import pytest


def moduli(count=49):
    """Pairwise-coprime moduli <= 256, greedy from 256 down (the table order)."""
    out = []
    for m in range(256, 1, -1):
        if all(math.gcd(m, x) == 1 for x in out):
            out.append(m)
        if len(out) == count:
            break
    return out


MODS = moduli()


def umulhi(a, b):
    return (a * b) >> 32


def residue_tc(X, m):
    """residue_tc_kernel's byte of X for modulus m (X' bytes, weights, one reduction)."""
    Xp = X + (1 << 111)
    assert 0 < Xp < (1 << 112)
    x = [(Xp >> (8 * b)) & 0xFF for b in range(14)] + [1, 0]
    w = [pow(2, 8 * b, m) for b in range(14)]
    c111 = (pow(2, 104, m) * 128) % m
    w += [(m - c111) % m, 0]
    S = sum(a * b for a, b in zip(x, w))
    assert S < (1 << 24)
    cm = 0xFFFFFFFF // m + 1  # ceil(2^32 / m)
    return S - umulhi(S, cm) * m


@pytest.mark.parametrize("L", [28, 29, 30, 31, 32])
def test_residue_bytes_exact(L):
    rng = random.Random(L)
    xs = [0, 1, -1, (1 << 109) - 1, -(1 << 109) + 1, 1 << 108, -(1 << 108)]
    xs += [rng.randrange(-(1 << 109) + 1, 1 << 109) for _ in range(400)]
    for X in xs:
        for m in MODS[:L]:
            assert residue_tc(X, m) == X % m, (X, m)


def test_ceil_magic_floor_exact_below_2_24():
    """floor(S / m) = umulhi(S, ceil(2^32 / m)) for every S < 2^24 that the sums
    can take: the error term S (ceil(2^32/m) m - 2^32) / (m 2^32) < 1/m."""
    rng = random.Random(5)
    for m in MODS[:32]:
        cm = 0xFFFFFFFF // m + 1
        for S in list(range(0, 4096)) + [rng.randrange(1 << 24) for _ in range(4000)] + [(1 << 24) - 1]:
            assert umulhi(S, cm) == S // m


def crt_tables(L):
    """What host_tables() fills for crt_tc_kernel: bytes of W_l, 16-bit limbs of M, 2^192 / M."""
    mods = MODS[:L]
    M = 1
    for m in mods:
        M *= m
    W = []
    for m in mods:
        P = M // m
        W.append(P * pow(P % m, -1, m))
    wb = [[(W[l] >> (8 * q)) & 0xFF for l in range(L)] for q in range(32)]
    mlimb = [(M >> (16 * h)) & 0xFFFF for h in range(16)]
    k192 = float(Fraction(1 << 192, M))
    return mods, M, W, wb, mlimb, k192


def quick_two_sum(a, b):
    s = a + b
    return s, b - (s - a)


def crt_tc(r, L, tables):
    """crt_tc_kernel's finish for one entry: returns (hi, lo, q, chunks)."""
    mods, M, W, wb, mlimb, k192 = tables
    S = [sum(r[l] * wb[q][l] for l in range(L)) for q in range(32)]
    assert max(S) < (1 << 21)
    U = [S[2 * h] + (S[2 * h + 1] << 8) for h in range(16)]
    vt = (float(U[15]) * 2.0 ** 48 + float(U[14]) * 2.0 ** 32) + (float(U[13]) * 2.0 ** 16 + float(U[12]))
    q = int(round(vt * k192))
    d = [U[h] - q * mlimb[h] for h in range(16)] + [0, 0]
    chunks, carry = [], 0
    for k in range(6):
        c = d[3 * k] + d[3 * k + 1] * 65536 + d[3 * k + 2] * 4294967296 + carry
        assert abs(c) < (1 << 63)  # an int64 in the kernel
        carry = (c + (1 << 47)) >> 48 if k < 5 else 0
        b = c - carry * (1 << 48)
        assert k == 5 or -(1 << 47) <= b < (1 << 47)
        chunks.append(b)
    v = [math.ldexp(float(b), 48 * k) for k, b in enumerate(chunks)]  # exact
    for k, b in enumerate(chunks):
        assert int(v[k]) == b << (48 * k)
    hi, lo = v[5], 0.0
    for k in range(4, -1, -1):
        hs, he = quick_two_sum(hi, v[k])
        hi, lo = quick_two_sum(hs, he + lo)
    return hi, lo, q, chunks


@pytest.mark.parametrize("L", [28, 29, 30, 31, 32])
def test_crt_reconstruction(L):
    tables = crt_tables(L)
    mods, M, W, wb, mlimb, k192 = tables
    assert M.bit_length() <= 256
    rng = random.Random(100 + L)
    bound = M // 4
    cs = [0, 1, -1, bound, -bound, bound - 12345, 1 << 200, -(1 << 150) - 7]
    cs += [rng.randrange(-bound, bound + 1) for _ in range(300)]
    cs += [rng.randrange(-(1 << 60), 1 << 60) for _ in range(100)]  # small entries (cancellation)
    for C in cs:
        r = [C % m for m in mods]
        V = sum(rl * w for rl, w in zip(r, W))
        hi, lo, q, chunks = crt_tc(r, L, tables)
        assert V - q * M == C, (L, C)
        assert sum(b << (48 * k) for k, b in enumerate(chunks)) == C
        # the double-double is C to f128 accuracy (relative to |C|)
        got = Fraction(hi) + Fraction(lo)
        assert abs(got - C) <= abs(Fraction(C)) * Fraction(1, 1 << 104) + Fraction(0), (L, C)


def two_sum(a, b):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


@pytest.mark.parametrize("L", [28, 29, 30, 31, 32])
def test_f256_crt_combination(L):
    """The f256 GEMM's CRT: two reconstructions G1, G2 (each as the f128 CRT's
    balanced 48-bit chunks), combined as G1 2^105 + G2 (105 = 2 chunks + 9 bits)
    with one carry pass into 9 balanced chunks, then summed from the top into
    four limbs: exact integer, and the limbs equal it to ~2^-208 relative."""
    tables = crt_tables(L)
    mods, M, W, wb, mlimb, k192 = tables
    rng = random.Random(200 + L)
    bound = M // 4
    pairs = [(0, 0), (0, 1), (0, -1), (1, -(1 << 105) + 3), (-1, (1 << 105) - 5), (bound, bound), (-bound, -bound),
             (1 << 100, -(1 << 205)), (3, -(3 << 105))]
    pairs += [(rng.randrange(-bound, bound + 1), rng.randrange(-bound, bound + 1)) for _ in range(200)]
    pairs += [(rng.randrange(-(1 << 40), 1 << 40), rng.randrange(-(1 << 100), 1 << 100)) for _ in range(100)]
    for G1, G2 in pairs:
        b1 = crt_tc([G1 % m for m in mods], L, tables)[3]
        b2 = crt_tc([G2 % m for m in mods], L, tables)[3]
        c = [0] * 9
        for k in range(6):
            c[k] += b2[k]
            c[k + 2] += b1[k] * 512
        carry = 0
        for k in range(9):
            x = c[k] + carry
            carry = (x + (1 << 47)) >> 48 if k < 8 else 0
            c[k] = x - carry * (1 << 48)
            assert k == 8 or -(1 << 47) <= c[k] < (1 << 47)
        C = G1 * (1 << 105) + G2
        assert sum(ck << (48 * k) for k, ck in enumerate(c)) == C
        x = [0.0, 0.0, 0.0, 0.0]
        for k in range(8, -1, -1):
            v = math.ldexp(float(c[k]), 48 * k)
            x[0], e = two_sum(x[0], v)
            x[1], e = two_sum(x[1], e)
            x[2], e = two_sum(x[2], e)
            x[3] = x[3] + e
        x[2], x[3] = two_sum(x[2], x[3])
        x[1], x[2] = two_sum(x[1], x[2])
        x[0], x[1] = two_sum(x[0], x[1])
        x[1], x[2] = two_sum(x[1], x[2])
        x[2], x[3] = two_sum(x[2], x[3])
        got = sum(Fraction(v) for v in x)
        assert abs(got - C) <= abs(Fraction(C)) * Fraction(1, 1 << 206), (L, C)
        if abs(C) < (1 << 150):
            assert got == C, (L, C)
