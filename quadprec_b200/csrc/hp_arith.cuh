// Device-side extended-precision arithmetic: f128 (double-double) and
// MultiFloat<4> (f256, quad-double) with the exact operation order of
// hyperprec's Rust code (crates/quad/src/dd.rs, multifloat/{core,add,mul,
// div,math}.rs). Every floating-point operation is an explicit
// round-to-nearest intrinsic (__dadd_rn, __dmul_rn, __fma_rn, ...), so the
// compiler can neither fuse nor reorder them: a kernel that applies these
// functions in the reference's order produces the reference's bits.
#pragma once
#include <cstdint>

namespace hp {

struct dd {
  double hi, lo;
};

__device__ __forceinline__ double ADD(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double SUB(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double MUL(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double DIV(double a, double b) { return __ddiv_rn(a, b); }

// dd.rs:16-35 / multifloat/core.rs:20-42
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = ADD(a, b);
  double v = SUB(s, a);
  e = ADD(SUB(a, SUB(s, v)), SUB(b, v));
}
__device__ __forceinline__ void quick_two_sum(double a, double b, double& s, double& e) {
  s = ADD(a, b);
  e = SUB(b, SUB(s, a));
}
__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  p = MUL(a, b);
  e = __fma_rn(a, b, -p);
}

__device__ __forceinline__ dd dd_from(double x) { return dd{x, 0.0}; }
__device__ __forceinline__ dd dd_renorm(double hi, double lo) {  // dd.rs:86-89
  dd r;
  quick_two_sum(hi, lo, r.hi, r.lo);
  return r;
}
__device__ __forceinline__ dd dd_neg(dd a) { return dd{-a.hi, -a.lo}; }
__device__ __forceinline__ dd dd_add(dd a, dd b) {  // dd.rs:147-157
  double s1, e1, s2, e2, s, e;
  two_sum(a.hi, b.hi, s1, e1);
  two_sum(a.lo, b.lo, s2, e2);
  e = ADD(e1, s2);
  quick_two_sum(s1, e, s, e);
  return dd_renorm(s, ADD(e, e2));
}
__device__ __forceinline__ dd dd_sub(dd a, dd b) { return dd_add(a, dd_neg(b)); }
__device__ __forceinline__ dd dd_mul(dd a, dd b) {  // dd.rs:175-183
  double p1, e1;
  two_prod(a.hi, b.hi, p1, e1);
  double e = ADD(e1, ADD(MUL(a.hi, b.lo), MUL(a.lo, b.hi)));
  return dd_renorm(p1, e);
}
__device__ __forceinline__ dd dd_div(dd a, dd b) {  // dd.rs:185-195
  double q1 = DIV(a.hi, b.hi);
  dd r = dd_sub(a, dd_mul(dd_from(q1), b));
  double q2 = DIV(r.hi, b.hi);
  return dd_renorm(q1, q2);
}
__device__ __forceinline__ dd dd_abs(dd a) { return signbit(a.hi) ? dd_neg(a) : a; }
__device__ __forceinline__ bool dd_lt(dd a, dd b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
__device__ __forceinline__ dd dd_recip(dd a) {  // dd.rs:80-83
  dd x0 = dd_from(DIV(1.0, a.hi));
  return dd_add(x0, dd_mul(x0, dd_sub(dd_from(1.0), dd_mul(a, x0))));
}
__device__ __forceinline__ dd dd_sqrt(dd a) {  // dd.rs:61-78
  if (a.hi < 0.0) return dd{__longlong_as_double(0x7ff8000000000000ll), 0.0};
  if (a.hi == 0.0) return dd{0.0, 0.0};
  if (!isfinite(a.hi)) return dd{a.hi, 0.0};
  dd x = dd_from(DIV(1.0, __dsqrt_rn(a.hi)));
  dd ax = dd_mul(a, x);
  dd hx = dd_mul(x, dd_from(0.5));
  dd r = dd_add(ax, dd_mul(ax, dd_sub(dd_from(0.5), dd_mul(ax, hx))));
  return dd_mul(dd_add(r, dd_div(a, r)), dd_from(0.5));
}
// x / b for a small positive integer b with y = RN(1/b): the correctly
// rounded quotient, i.e. the bits of DIV(x, b). q1 = q0 + (x - q0 b) y is a
// faithful quotient, and Markstein's final step q1 + (x - q1 b) y with
// y within half an ulp of 1/b then rounds to RN(x / b). Zeros, values below
// 2^-900 (whose remainders would be subnormal) and non-finite values take
// the IEEE division.
__device__ __forceinline__ double div_small_int(double x, double b, double y) {
  if (!(fabs(x) >= 0x1p-900) || !(fabs(x) <= 1.7976931348623157e308)) return DIV(x, b);
  const double q0 = MUL(x, y);
  const double q1 = __fma_rn(__fma_rn(-q0, b, x), y, q0);
  return __fma_rn(__fma_rn(-q1, b, x), y, q1);
}
// dd_div(a, dd_from(b)) for a small positive integer b, bit for bit: both
// double quotients through div_small_int, and q1 * (b, 0) without its two
// zero cross products (for finite q1 they add exactly +0 to the error term,
// which only turns a -0 into +0: e1 + 0.0 does the same).
__device__ __forceinline__ dd dd_div_small_int(dd a, double b, double y) {
  const double q1 = div_small_int(a.hi, b, y);
  double p1, e1;
  two_prod(q1, b, p1, e1);
  const dd r = dd_sub(a, dd_renorm(p1, ADD(e1, 0.0)));
  const double q2 = div_small_int(r.hi, b, y);
  return dd_renorm(q1, q2);
}
// dd.rs:106-121 (argument reduction by ln 2, Taylor series, 2^k by bit trick).
// The Taylor loop is unrolled, so each term divides by a constant i with its
// reciprocal folded at compile time (dd_div_small_int: the same bits as the
// reference's division).
__device__ __forceinline__ dd dd_exp(dd a) {
  if (a.hi == 0.0 && a.lo == 0.0) return dd_from(1.0);
  const dd LN2 = {0.6931471805599453, 2.3190468138462996e-17};  // dd.rs:40
  double k = round(DIV(a.hi, LN2.hi));
  dd r = dd_sub(a, dd_mul(dd_from(k), LN2));
  dd term = dd_from(1.0), sum = dd_from(1.0);
#pragma unroll
  for (int i = 1; i <= 25; i++) {
    term = dd_div_small_int(dd_mul(term, r), (double)i, 1.0 / (double)i);
    sum = dd_add(sum, term);
    if (dd_abs(term).hi < 1e-35) break;
  }
  double scale = __longlong_as_double((long long)((uint64_t)(1023 + (int64_t)k) << 52));
  return dd_mul(sum, dd_from(scale));
}

// ---------------------------------------------------------------------------
// MultiFloat<4> (f256). The reference's data-dependent loops (insertion sort,
// grow-expansion length, renormalisation emit index, carry cascades) are
// rewritten with static indices and predicated selects so that the limbs
// stay in registers; each rewrite produces the same values as the loop it
// replaces (argued at each site).
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Fast f128 helpers for the chosen-path kernels only (not the reference's
// operation order; never used where results must match the reference's bits).
// ---------------------------------------------------------------------------
// a - b c with 16 operations instead of the 29 of a reference-order multiply
// and add: the exact product p + pe of the high parts, the cross terms
// b.hi c.lo + b.lo c.hi, one two_sum of the high parts and a final
// renormalisation (the "sloppy" addition). Error below ~3 2^-104
// (|a| + |b c|), the bound the backward-error analyses of Cholesky and
// substitution assume of each update.
__device__ __forceinline__ dd dd_fms_fast(dd a, dd b, dd c) {
  const double p = __dmul_rn(b.hi, c.hi);
  const double pe = __fma_rn(b.hi, c.hi, -p);
  const double t = __fma_rn(b.hi, c.lo, __dmul_rn(b.lo, c.hi));
  double s, se;
  two_sum(a.hi, -p, s, se);
  const double e = __dadd_rn(se, __dsub_rn(a.lo, __dadd_rn(pe, t)));
  return dd_renorm(s, e);
}
// Plane rotation of a pair, x = c a - s b and y = s a + c b, each output as
// the exact products of the high parts (FMA error terms), the cross terms,
// one two_sum of the high products and a final renormalisation: 17
// operations per output instead of the 40 of a reference-order multiply,
// multiply and add. Error below ~4 2^-104 (|c a| + |s b|), as for
// dd_fms_fast.
__device__ __forceinline__ dd dd_dot2_fast(dd c, dd a, dd s, dd b) {  // c a + s b
  const double p1 = __dmul_rn(c.hi, a.hi), e1 = __fma_rn(c.hi, a.hi, -p1);
  const double p2 = __dmul_rn(s.hi, b.hi), e2 = __fma_rn(s.hi, b.hi, -p2);
  const double t = __fma_rn(c.hi, a.lo, __fma_rn(c.lo, a.hi, __fma_rn(s.hi, b.lo, __dmul_rn(s.lo, b.hi))));
  double h, he;
  two_sum(p1, p2, h, he);
  return dd_renorm(h, __dadd_rn(he, __dadd_rn(__dadd_rn(e1, e2), t)));
}
__device__ __forceinline__ void dd_rot_fast(dd c, dd s, dd a, dd b, dd& x, dd& y) {
  x = dd_dot2_fast(c, a, dd{-s.hi, -s.lo}, b);
  y = dd_dot2_fast(s, a, c, b);
}
// 1/d to ~2^-103 from the correctly rounded f64 seed x = 1/d.hi by one
// Newton step x1 = x + x e, e = 1 - d x (relative error of x at most
// 2^-53, so e, of that size, is needed only to ~2^-104 absolute: the fma
// gives 1 - d.hi x to 2^-106, d.lo x is its small correction); the
// result's error is delta^2 + O(2^-104).
__device__ __forceinline__ dd dd_recip_fast(dd d) {
  const double x = __drcp_rn(d.hi);
  const double e = __fma_rn(-d.lo, x, __fma_rn(-d.hi, x, 1.0));
  return dd_renorm(x, __dmul_rn(x, e));
}
// 1/sqrt(d) to ~2^-103 from the f64 seed x = rsqrt(d.hi) (relative error
// delta of a few 2^-53) by one Newton step x1 = x + x e / 2, e = 1 - d x^2.
// e is ~delta, so it is needed only to ~2^-104 absolute: with x^2 = s + s'
// exact (FMA), e = fma(-d.hi, s, 1) - (d.hi s' + d.lo s), each rounding
// below 2^-104; x1 = x + c, c = x e / 2, is kept unevaluated as (x, c)
// renormalised. The result's error is 1.5 delta^2 + O(2^-104).
__device__ __forceinline__ dd dd_rsqrt_fast(dd d) {
  const double x = rsqrt(d.hi);
  const double s = __dmul_rn(x, x), s2 = __fma_rn(x, x, -s);
  const double t = __fma_rn(-d.hi, s, 1.0);
  const double u = __fma_rn(d.hi, s2, __dmul_rn(d.lo, s));
  const double c = __dmul_rn(__dmul_rn(x, __dsub_rn(t, u)), 0.5);
  return dd_renorm(x, c);
}

struct qd {
  double l[4];
};

__device__ __forceinline__ qd qd_zero() { return qd{{0.0, 0.0, 0.0, 0.0}}; }
__device__ __forceinline__ qd qd_from(double x) { return qd{{x, 0.0, 0.0, 0.0}}; }
__device__ __forceinline__ qd qd_neg(const qd& a) { return qd{{-a.l[0], -a.l[1], -a.l[2], -a.l[3]}}; }

// Top-down quick_two_sum compaction of core.rs:77-91 over M inputs into the
// first NOUT output slots. The reference writes out[k] with a running k;
// here every slot t is updated by select(k == t), which writes the same
// values. With NOUT < M it is core.rs:148-166 (stop once NOUT limbs exist).
template <int M, int NOUT>
__device__ __forceinline__ void compact_top_down(const double* t, double* out) {
#pragma unroll
  for (int i = 0; i < NOUT; i++) out[i] = 0.0;
  double s = t[0];
  int k = 0;
#pragma unroll
  for (int i = 1; i < M; i++) {
    double ns, e;
    quick_two_sum(s, t[i], ns, e);
    s = ns;
    bool emit = (e != 0.0) && (k < NOUT);
#pragma unroll
    for (int q = 0; q < NOUT; q++)
      if (emit && k == q) out[q] = s;
    if (e != 0.0) {
      s = e;
      k++;
    }
  }
  // Reference: out[k] = s if k < NOUT (the NOUT == M case always has k < M).
#pragma unroll
  for (int q = 0; q < NOUT; q++)
    if (k == q) out[q] = s;
}
// Bottom-up two_sum sweep of core.rs:67-75.
template <int M>
__device__ __forceinline__ void sweep_bottom_up(double* t) {
  double s, e;
  two_sum(t[M - 2], t[M - 1], s, e);
  t[M - 1] = e;
#pragma unroll
  for (int i = M - 3; i >= 0; i--) {
    double ns;
    two_sum(t[i], s, ns, e);
    s = ns;
    t[i + 1] = e;
  }
  t[0] = s;
}
// core.rs:58-93 for N = 4.
__device__ __forceinline__ void qd_renormalize(double* l) {
#pragma unroll
  for (int pass = 0; pass < 2; pass++) {
    sweep_bottom_up<4>(l);
    double out[4];
    compact_top_down<4, 4>(l, out);
#pragma unroll
    for (int i = 0; i < 4; i++) l[i] = out[i];
  }
}
// core.rs:100-168 for N = 4, M = 8. The early return at k >= N in the
// reference leaves the remaining inputs unused; compact_top_down<8,4> stops
// writing once four limbs are emitted, which is the same result.
__device__ __forceinline__ void qd_renormalize_from8(const double* in, double* out4) {
  double t[8];
#pragma unroll
  for (int i = 0; i < 8; i++) t[i] = in[i];
  sweep_bottom_up<8>(t);
  double buf[8];
  compact_top_down<8, 8>(t, buf);
  sweep_bottom_up<8>(buf);
  compact_top_down<8, 4>(buf, out4);
}

// add.rs:23-105 for N = 4.
// (1) Insertion sort by descending |x| (stable: an element never passes an
//     equal-magnitude one). Replaced by a sorting network on the key
//     (|x| descending, original index ascending), which is a total order
//     whose sorted sequence is exactly the stable insertion-sort result.
// (2) Grow-expansion: the reference walks only the exp_len live slots of a
//     compact array whose remaining slots are zero; two_sum(0, c) = (c, 0)
//     exactly for c != 0, so walking all 8 slots leaves the same array.
__device__ __forceinline__ void cmp_swap(double& a, int& ia, double& b, int& ib) {
  double ma = fabs(a), mb = fabs(b);
  bool sw = (ma < mb) || (ma == mb && ia > ib);
  double ta = sw ? b : a, tb = sw ? a : b;
  int ja = sw ? ib : ia, jb = sw ? ia : ib;
  a = ta;
  b = tb;
  ia = ja;
  ib = jb;
}
__device__ __forceinline__ qd qd_add(const qd& a, const qd& b) {
  double w[8];
  int id[8];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    two_sum(a.l[i], b.l[i], w[2 * i], w[2 * i + 1]);
    id[2 * i] = 2 * i;
    id[2 * i + 1] = 2 * i + 1;
  }
  // Batcher odd-even merge sort network for 8 keys (19 comparators).
#define CS(x, y) cmp_swap(w[x], id[x], w[y], id[y])
  CS(0, 1); CS(2, 3); CS(4, 5); CS(6, 7);
  CS(0, 2); CS(1, 3); CS(4, 6); CS(5, 7);
  CS(1, 2); CS(5, 6);
  CS(0, 4); CS(1, 5); CS(2, 6); CS(3, 7);
  CS(2, 4); CS(3, 5);
  CS(1, 2); CS(3, 4); CS(5, 6);
#undef CS
  double ex[8];
#pragma unroll
  for (int i = 0; i < 8; i++) ex[i] = 0.0;
  int exp_len = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    double term = w[i];
    if (term != 0.0) {
      if (exp_len == 0) {
        ex[0] = term;
        exp_len = 1;
      } else {
        double carry = term;
#pragma unroll
        for (int j = 7; j >= 0; j--) {
          double s, e;
          two_sum(ex[j], carry, s, e);
          ex[j] = e;
          carry = s;
        }
        if (carry != 0.0) {
#pragma unroll
          for (int k = 7; k > 0; k--) ex[k] = ex[k - 1];
          ex[0] = carry;
          exp_len++;
        }
      }
    }
  }
  qd r;
#pragma unroll
  for (int i = 0; i < 4; i++) r.l[i] = ex[i];  // slots >= exp_len are zero
  qd_renormalize(r.l);
  return r;
}
__device__ __forceinline__ qd qd_sub(const qd& a, const qd& b) { return qd_add(a, qd_neg(b)); }

// mul.rs:31-42 accumulate(work, idx, val, limit=8): the cascade stops at the
// first zero error; later slots are written only while the cascade is live.
template <int IDX>
__device__ __forceinline__ void qd_accumulate(double* work, double val) {
  double s, e;
  two_sum(work[IDX], val, s, e);
  work[IDX] = s;
  bool live = true;
#pragma unroll
  for (int k = IDX + 1; k < 8; k++) {
    live = live && (e != 0.0);
    double s2, e2;
    two_sum(work[k], e, s2, e2);
    if (live) {
      work[k] = s2;
      e = e2;
    }
  }
}
// mul.rs:16-110 for N = 4.
__device__ __forceinline__ qd qd_mul(const qd& a, const qd& b) {
  double work[8];
#pragma unroll
  for (int i = 0; i < 8; i++) work[i] = 0.0;
#define TERM(I, J)                        \
  {                                       \
    double p, e;                          \
    two_prod(a.l[I], b.l[J], p, e);       \
    qd_accumulate<(I) + (J)>(work, p);    \
    qd_accumulate<(I) + (J) + 1>(work, e); \
  }
  TERM(0, 0) TERM(0, 1) TERM(0, 2) TERM(0, 3)
  TERM(1, 0) TERM(1, 1) TERM(1, 2)
  TERM(2, 0) TERM(2, 1)
  TERM(3, 0)
#undef TERM
  qd r;
  qd_renormalize_from8(work, r.l);
  return r;
}
// div.rs:14-41 (N = 4: ceil(log2 4) + 2 = 4 Newton steps).
__device__ __forceinline__ qd qd_recip(const qd& a) {
  if (a.l[0] == 0.0) return qd_from(signbit(a.l[0]) ? -INFINITY : INFINITY);
  if (!isfinite(a.l[0])) return qd_from(0.0);
  qd x = qd_from(DIV(1.0, a.l[0]));
  const qd one = qd_from(1.0);
  for (int s = 0; s < 4; s++) {
    qd residual = qd_sub(one, qd_mul(a, x));
    x = qd_add(x, qd_mul(x, residual));
  }
  return x;
}
// div.rs:52-76
__device__ __forceinline__ qd qd_div(const qd& a, const qd& b) {
  if (b.l[0] == 0.0) {
    double sign = (signbit(a.l[0]) == signbit(b.l[0])) ? 1.0 : -1.0;
    return qd_from(a.l[0] == 0.0 ? __longlong_as_double(0x7ff8000000000000ll) : sign * INFINITY);
  }
  if (a.l[0] == 0.0) return qd_zero();
  if (!isfinite(a.l[0]) || !isfinite(b.l[0])) return qd_from(DIV(a.l[0], b.l[0]));
  return qd_mul(a, qd_recip(b));
}
// math.rs:22-40 (N = 4: ceil(log2 4) + 1 = 3 Heron steps).
__device__ __forceinline__ qd qd_sqrt(const qd& a) {
  if (a.l[0] < 0.0) return qd_from(__longlong_as_double(0x7ff8000000000000ll));
  if (a.l[0] == 0.0) return qd_zero();
  if (!isfinite(a.l[0])) return qd_from(a.l[0]);
  qd x = qd_from(__dsqrt_rn(a.l[0]));
  const qd half = qd_from(0.5);
  for (int s = 0; s < 3; s++) x = qd_mul(qd_add(x, qd_div(a, x)), half);
  return x;
}

}  // namespace hp
