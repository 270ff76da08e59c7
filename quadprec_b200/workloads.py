"""Deterministic synthetic inputs for the benchmark configurations.

RNG: SplitMix64 (seed 0 unless stated); U[0,1) = (x >> 11) * 2^-53.
All generators are vectorised numpy and reproduce bit-for-bit on any host.

Configurations (sizes as benchmarked):
  * dense_dd(m, k, seed, offset): full double-double entries,
    hi ~ U[-1,1), lo = hi * 2^-53 * U[-1,1), renormalised with
    quick_two_sum (crates/quad/src/dd.rs:86-89). Used for the f128 GEMM at
    m = n = k = 2048 and, limb-extended, for f256 GEMM at 1024.
  * shifted_hilbert(n): A_ij = 1/(i+j+1) (f64), A_ii += 1, b = ones
    (the README / linalg.rs:548-557 construction), n = 512.
  * overlap_lattice(...): s-Gaussian basis on a jittered cubic lattice.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(count: int, seed: int = 0, offset: int = 0) -> np.ndarray:
    """The outputs number offset+1 .. offset+count of SplitMix64(seed)."""
    with np.errstate(over="ignore"):
        idx = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform(count: int, seed: int = 0, offset: int = 0) -> np.ndarray:
    return (splitmix64(count, seed, offset) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def quick_two_sum(a: np.ndarray, b: np.ndarray):
    s = a + b
    return s, b - (s - a)


def dense_dd(rows: int, cols: int, seed: int = 0, offset: int = 0) -> np.ndarray:
    """rows x cols f128 matrix (shape (rows, cols, 2)); consumes 2 draws/entry."""
    u = uniform(2 * rows * cols, seed, offset).reshape(rows * cols, 2)
    hi = 2.0 * u[:, 0] - 1.0
    lo = hi * 2.0 ** -53 * (2.0 * u[:, 1] - 1.0)
    s, e = quick_two_sum(hi, lo)
    return np.stack([s, e], axis=-1).reshape(rows, cols, 2)


def gemm_operands(m: int, n: int, k: int, seed: int = 0, atb: bool = False):
    """A (m x k, or k x m if atb) then B (k x n), one SplitMix64 stream."""
    a = dense_dd(k, m, seed, 0) if atb else dense_dd(m, k, seed, 0)
    b = dense_dd(k, n, seed, 2 * m * k)
    return a, b


def sample_index(m: int, n: int, count: int = 4096, seed: int = 7, rows=None) -> np.ndarray:
    """(i, j) pairs: `count` entries from SplitMix64(seed), then every entry of
    the rows in `rows` (default: the first and the last). Used to state a
    GEMM's error against an f512 evaluation of sampled entries."""
    u = uniform(2 * count, seed, 0).reshape(count, 2)
    ij = np.stack([np.minimum((u[:, 0] * m).astype(np.int64), m - 1),
                   np.minimum((u[:, 1] * n).astype(np.int64), n - 1)], -1)
    rows = (0, m - 1) if rows is None else rows
    full = [np.stack([np.full(n, r, dtype=np.int64), np.arange(n, dtype=np.int64)], -1) for r in rows]
    return np.concatenate([ij, *full]).astype(np.int64)


def sample_abs_products(a: np.ndarray, b: np.ndarray, idx: np.ndarray, atb: bool = False,
                        chunk: int = 512) -> np.ndarray:
    """sum_p |a_ip| |b_pj| (leading limbs) for each sampled (i, j): the entries
    of |op(A)| |B| that normalise a sampled GEMM error."""
    A = np.abs(a[..., 0])
    A = A.T if atb else A
    B = np.abs(b[..., 0])
    out = np.empty(len(idx))
    for c0 in range(0, len(idx), chunk):
        i, j = idx[c0:c0 + chunk, 0], idx[c0:c0 + chunk, 1]
        out[c0:c0 + chunk] = np.einsum("ek,ke->e", A[i], B[:, j])
    return out


def sampled_error(c: np.ndarray, c_star: np.ndarray, absab: np.ndarray, idx: np.ndarray) -> tuple[float, float]:
    """Error of a computed GEMM over sampled entries against reference values
    c_star (limbs, leading first): (||C - C*||_F / || |A| |B| ||_F,
    ||C - C*||_F / ||C*||_F). The difference is taken limb by limb (each limb
    difference is exact while the two values agree to that limb) and the
    limb differences are summed from the leading one."""
    got = c[idx[:, 0], idx[:, 1]]
    nl = max(got.shape[-1], c_star.shape[-1])
    d = np.zeros(len(idx))
    for t in range(nl):
        g = got[:, t] if t < got.shape[-1] else 0.0
        r = c_star[:, t] if t < c_star.shape[-1] else 0.0
        d = d + (g - r)
    return float(np.linalg.norm(d) / np.linalg.norm(absab)), float(np.linalg.norm(d) / np.linalg.norm(c_star[:, 0]))


def dd_to_qd(x: np.ndarray) -> np.ndarray:
    """Limb-extend f128 entries to f256 (MultiFloat<4>::from_f128, conv.rs:121-126)."""
    out = np.zeros(x.shape[:-1] + (4,))
    out[..., :2] = x
    return out


def shifted_hilbert(n: int):
    """f128 matrix 1/(i+j+1) (from f64) + I, and b = ones (README construction)."""
    i = np.arange(n, dtype=np.float64)
    h = 1.0 / (i[:, None] + i[None, :] + 1.0)
    a = np.zeros((n, n, 2))
    a[..., 0] = h
    # f128::from_f64(h_ii) + f128::from_f64(1.0): exact two_sum of two doubles
    d = np.diag(h).copy()
    s = d + 1.0
    v = s - d
    e = (d - (s - v)) + (1.0 - v)
    a[np.arange(n), np.arange(n), 0] = s
    a[np.arange(n), np.arange(n), 1] = e
    b = np.zeros((n, 2))
    b[:, 0] = 1.0
    return a, b


def normal(count: int, seed: int = 0, offset: int = 0) -> np.ndarray:
    """Approximately N(0,1): Irwin-Hall sum of 12 SplitMix64 uniforms minus 6.

    Only additions, so b is bit-reproducible on any host (a Box-Muller b would
    inherit the host libm's last-ulp differences, which an extended-precision
    solve amplifies far above the 1e-25 accuracy target).
    """
    u = uniform(12 * count, seed, offset).reshape(count, 12)
    acc = np.zeros(count)
    for t in range(12):
        acc = acc + u[:, t]
    return acc - 6.0


def overlap_lattice(nx: int, ny: int, nz: int, spacing: float = 1.4, jitter: float = 0.05, n_exp: int = 4,
                    lo: float = 0.01, hi: float = 10.0, seed: int = 0):
    """s-Gaussian basis on a jittered cubic lattice (center-major order).

    Centres are visited in row-major (ix, iy, iz) order; each takes 3 jitter
    draws (coordinate + jitter*(2U-1)) then n_exp exponent draws,
    log-uniform in [lo, hi]. Returns (centers (N,3), alpha (N,)) with one
    entry per basis function, N = nx*ny*nz*n_exp.
    """
    nc = nx * ny * nz
    per = 3 + n_exp
    u = uniform(nc * per, seed, 0).reshape(nc, per)
    grid = np.array([(ix, iy, iz) for ix in range(nx) for iy in range(ny) for iz in range(nz)], dtype=np.float64)
    cen = grid * spacing + jitter * (2.0 * u[:, :3] - 1.0)
    alpha = lo * (hi / lo) ** u[:, 3:]
    return np.repeat(cen, n_exp, axis=0), alpha.reshape(-1)


def overlap_spd_problem(nx: int, ny: int, nz: int, seed: int = 0):
    """Overlap SPD workload: lattice basis and b ~ N(0,1) (n = nx*ny*nz*4)."""
    cen, alpha = overlap_lattice(nx, ny, nz, seed=seed)
    n = len(alpha)
    b = normal(n, seed, offset=10 ** 9)
    return cen, alpha, b


def batched_overlap_systems(count: int = 4096, seed: int = 0, n_min: int = 16, n_max: int = 384):
    """Uneven batch of overlap SPD systems (random 3-D clusters).

    System s uses its own SplitMix64 stream (seed, offset s * 2^24):
      n = 4 * clamp(round(n_min * (n_max/n_min)^U / 4), n_min/4, n_max/4);
      n/4 centres: the first at the origin, each next one at distance
      U[1.2, 2.0] bohr from a uniformly chosen existing centre along a
      direction drawn by rejection from the unit ball (no libm calls),
      rejected (up to 64 tries) if closer than 1.2 to any existing centre;
      4 exponents per centre, log-uniform in [0.01, 10]; b ~ N(0,1)
      (Irwin-Hall, see normal()).
    Returns dict with offsets (count+1), n (count), centers (N,3), alpha (N,), b (N,).
    """
    import math

    ns, cens, alphas, bs = [], [], [], []
    for s in range(count):
        u = uniform(1 << 15, seed, s << 24).tolist()
        pos = 0
        n = 4 * int(min(max(round(n_min * (n_max / n_min) ** u[pos] / 4.0), n_min // 4), n_max // 4))
        pos += 1
        pts = [(0.0, 0.0, 0.0)]
        while len(pts) < n // 4:
            for _try in range(64):
                bx, by, bz = pts[int(u[pos] * len(pts)) % len(pts)]
                pos += 1
                while True:
                    dx, dy, dz = 2 * u[pos] - 1, 2 * u[pos + 1] - 1, 2 * u[pos + 2] - 1
                    pos += 3
                    r2 = dx * dx + dy * dy + dz * dz
                    if 0.01 < r2 <= 1.0:
                        break
                sc = (1.2 + 0.8 * u[pos]) / math.sqrt(r2)
                pos += 1
                cand = (bx + sc * dx, by + sc * dy, bz + sc * dz)
                if min(math.sqrt((p[0] - cand[0]) ** 2 + (p[1] - cand[1]) ** 2 + (p[2] - cand[2]) ** 2)
                       for p in pts) >= 1.2:
                    break
            pts.append(cand)
        ex = np.array([0.01 * 1000.0 ** u[pos + t] for t in range(n)])
        cen = np.repeat(np.array(pts), 4, axis=0)
        ns.append(n)
        cens.append(cen)
        alphas.append(ex)
        bs.append(normal(n, seed, (s << 24) + (1 << 20)))
    off = np.zeros(count + 1, dtype=np.int64)
    off[1:] = np.cumsum(ns)
    return {"offsets": off, "n": np.array(ns, dtype=np.int64), "centers": np.concatenate(cens),
            "alpha": np.concatenate(alphas), "b": np.concatenate(bs)}
