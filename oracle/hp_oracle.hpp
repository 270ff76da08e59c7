// CPU oracle: a line-by-line C++ restatement of hyperprec's Rust arithmetic
// (m0at/quadprec, crates/quad, crates/solver, crates/overlap).
//
// TEST INFRASTRUCTURE ONLY. This code is the checker for the CUDA library in
// quadprec_b200/csrc and the timed CPU baseline in bench.py. The product path
// never links, loads or calls it.
//
// Build rules that keep it faithful to the Rust code (the reference cannot be
// compiled here: no Rust toolchain exists on either machine):
//   * -ffp-contract=off : Rust never fuses a*b+c on its own;
//   * f64::mul_add -> std::fma; f64::round -> std::round (half away from 0);
//   * powi(n) -> repeated multiplication; exp/ln/sqrt/pow -> the C library.
// Every function cites the Rust file:line it restates.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------------------
// Error-free transformations: crates/quad/src/dd.rs:15-35 and
// crates/quad/src/multifloat/core.rs:17-42 (identical in both files).
// ---------------------------------------------------------------------------
static inline void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double v = s - a;
  e = (a - (s - v)) + (b - v);
}
static inline void quick_two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  e = b - (s - a);
}
static inline void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = std::fma(a, b, -p);
}

// ---------------------------------------------------------------------------
// f128 double-double: crates/quad/src/dd.rs
// ---------------------------------------------------------------------------
struct dd {
  double hi, lo;
};
static inline dd dd_from(double x) { return dd{x, 0.0}; }           // dd.rs:48
static inline double dd_to_f64(dd a) { return a.hi + a.lo; }        // dd.rs:53
static inline dd dd_renorm(double hi, double lo) {                  // dd.rs:86
  dd r;
  quick_two_sum(hi, lo, r.hi, r.lo);
  return r;
}
static inline dd dd_neg(dd a) { return dd{-a.hi, -a.lo}; }          // dd.rs:167
static inline dd dd_add(dd a, dd b) {                               // dd.rs:147-157
  double s1, e1, s2, e2, s, e;
  two_sum(a.hi, b.hi, s1, e1);
  two_sum(a.lo, b.lo, s2, e2);
  e = e1 + s2;
  quick_two_sum(s1, e, s, e);
  return dd_renorm(s, e + e2);
}
static inline dd dd_sub(dd a, dd b) { return dd_add(a, dd_neg(b)); }  // dd.rs:159-165
static inline dd dd_mul(dd a, dd b) {                               // dd.rs:175-183
  double p1, e1;
  two_prod(a.hi, b.hi, p1, e1);
  double e = e1 + (a.hi * b.lo + a.lo * b.hi);
  return dd_renorm(p1, e);
}
static inline dd dd_div(dd a, dd b) {                               // dd.rs:185-195
  double q1 = a.hi / b.hi;
  dd r = dd_sub(a, dd_mul(dd_from(q1), b));
  double q2 = r.hi / b.hi;
  return dd_renorm(q1, q2);
}
static inline dd dd_abs(dd a) { return std::signbit(a.hi) ? dd_neg(a) : a; }  // dd.rs:57-59
static inline dd dd_recip(dd a) {                                   // dd.rs:80-83
  dd x0 = dd_from(1.0 / a.hi);
  return dd_add(x0, dd_mul(x0, dd_sub(dd_from(1.0), dd_mul(a, x0))));
}
static inline dd dd_sqrt(dd a) {                                    // dd.rs:61-78
  if (a.hi < 0.0) return dd{NAN, 0.0};
  if (a.hi == 0.0) return dd{0.0, 0.0};
  if (!std::isfinite(a.hi)) return dd{a.hi, 0.0};
  dd x = dd_from(1.0 / std::sqrt(a.hi));
  dd ax = dd_mul(a, x);
  dd hx = dd_mul(x, dd_from(0.5));
  dd r = dd_add(ax, dd_mul(ax, dd_sub(dd_from(0.5), dd_mul(ax, hx))));
  return dd_mul(dd_add(r, dd_div(a, r)), dd_from(0.5));
}
// Mixed f128/f64 ops: dd.rs:228-260
static inline dd dd_add_f64(dd a, double b) {
  double s1, e1;
  two_sum(a.hi, b, s1, e1);
  return dd_renorm(s1, e1 + a.lo);
}
static inline dd dd_mul_f64(dd a, double b) {
  double p1, e1;
  two_prod(a.hi, b, p1, e1);
  return dd_renorm(p1, e1 + a.lo * b);
}
static inline dd dd_div_f64(dd a, double b) {
  double q1 = a.hi / b;
  dd r = dd_sub(a, dd_mul(dd_from(q1), dd_from(b)));
  return dd_renorm(q1, r.hi / b);
}
static const dd DD_LN2 = {0.6931471805599453, 2.3190468138462996e-17};  // dd.rs:40
static inline dd dd_exp(dd a) {                                     // dd.rs:106-121
  if (a.hi == 0.0 && a.lo == 0.0) return dd_from(1.0);
  double k = std::round(a.hi / DD_LN2.hi);
  dd r = dd_sub(a, dd_mul(dd_from(k), DD_LN2));
  dd term = dd_from(1.0), sum = dd_from(1.0);
  for (int i = 1; i <= 25; i++) {
    term = dd_div(dd_mul(term, r), dd_from((double)i));
    sum = dd_add(sum, term);
    if (dd_abs(term).hi < 1e-35) break;
  }
  uint64_t bits = (uint64_t)(1023 + (int64_t)k) << 52;
  double scale;
  std::memcpy(&scale, &bits, 8);
  return dd_mul(sum, dd_from(scale));
}
static inline dd dd_ln(dd a) {                                      // dd.rs:124-137
  if (a.hi <= 0.0) return dd{NAN, NAN};
  if (a.hi == 1.0 && a.lo == 0.0) return dd{0.0, 0.0};
  dd x = dd_from(std::log(a.hi));
  for (int i = 0; i < 3; i++) {
    dd e = dd_exp(dd_neg(x));
    x = dd_add(x, dd_sub(dd_mul(a, e), dd_from(1.0)));
  }
  return x;
}
// f128 ordering (dd.rs:50-57 of the PartialOrd impl): hi first, then lo.
static inline bool dd_lt(dd a, dd b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }

// ---------------------------------------------------------------------------
// MultiFloat<N>: crates/quad/src/multifloat/{core,add,mul,div,math}.rs
// ---------------------------------------------------------------------------
template <int N>
struct mf {
  double l[N];
};
template <int N>
static inline mf<N> mf_zero() {
  mf<N> r;
  for (int i = 0; i < N; i++) r.l[i] = 0.0;
  return r;
}
template <int N>
static inline mf<N> mf_from(double x) {  // core.rs:185-189
  mf<N> r = mf_zero<N>();
  r.l[0] = x;
  return r;
}
template <int N>
static inline double mf_to_f64(const mf<N>& a) { return N >= 2 ? a.l[0] + a.l[1] : a.l[0]; }  // core.rs:193

// core.rs:58-93 (two passes of bottom-up two_sum, top-down quick_two_sum)
template <int N>
static inline void mf_renormalize(double* limbs) {
  if (N <= 1) return;
  for (int pass = 0; pass < 2; pass++) {
    double s, e;
    two_sum(limbs[N - 2], limbs[N - 1], s, e);
    limbs[N - 1] = e;
    for (int i = N - 3; i >= 0; i--) {
      double ns;
      two_sum(limbs[i], s, ns, e);
      s = ns;
      limbs[i + 1] = e;
    }
    limbs[0] = s;
    double out[N];
    for (int i = 0; i < N; i++) out[i] = 0.0;
    s = limbs[0];
    int k = 0;
    for (int i = 1; i < N; i++) {
      double ns;
      quick_two_sum(s, limbs[i], ns, e);
      s = ns;
      if (e != 0.0) {
        out[k] = s;
        s = e;
        k++;
      }
    }
    out[k] = s;
    for (int i = 0; i < N; i++) limbs[i] = out[i];
  }
}

// core.rs:100-168
template <int N, int M>
static inline void mf_renormalize_from(const double* input, double* outN) {
  double t[M];
  for (int i = 0; i < M; i++) t[i] = input[i];
  {
    double s, e;
    two_sum(t[M - 2], t[M - 1], s, e);
    t[M - 1] = e;
    for (int i = M - 3; i >= 0; i--) {
      double ns;
      two_sum(t[i], s, ns, e);
      s = ns;
      t[i + 1] = e;
    }
    t[0] = s;
    double buf[M];
    for (int i = 0; i < M; i++) buf[i] = 0.0;
    s = t[0];
    int k = 0;
    for (int i = 1; i < M; i++) {
      double ns;
      quick_two_sum(s, t[i], ns, e);
      s = ns;
      if (e != 0.0) {
        buf[k] = s;
        s = e;
        k++;
      }
    }
    buf[k] = s;
    for (int i = 0; i < M; i++) t[i] = buf[i];
  }
  {
    double s, e;
    two_sum(t[M - 2], t[M - 1], s, e);
    t[M - 1] = e;
    for (int i = M - 3; i >= 0; i--) {
      double ns;
      two_sum(t[i], s, ns, e);
      s = ns;
      t[i + 1] = e;
    }
    t[0] = s;
    for (int i = 0; i < N; i++) outN[i] = 0.0;
    s = t[0];
    int k = 0;
    for (int i = 1; i < M; i++) {
      double ns;
      quick_two_sum(s, t[i], ns, e);
      s = ns;
      if (e != 0.0) {
        outN[k] = s;
        s = e;
        k++;
        if (k >= N) return;
      }
    }
    if (k < N) outN[k] = s;
  }
}

template <int N>
static inline mf<N> mf_neg(const mf<N>& a) {  // add.rs:4-17
  mf<N> r;
  for (int i = 0; i < N; i++) r.l[i] = -a.l[i];
  return r;
}

// add.rs:19-106: pairwise two_sum, insertion sort by |.| descending,
// grow-expansion, renormalize.
template <int N>
static inline mf<N> mf_add(const mf<N>& a, const mf<N>& b) {
  const int MAX_WORK = 32;
  const int work_len = 2 * N;
  double work[MAX_WORK];
  for (int i = 0; i < MAX_WORK; i++) work[i] = 0.0;
  for (int i = 0; i < N; i++) two_sum(a.l[i], b.l[i], work[2 * i], work[2 * i + 1]);
  for (int i = 1; i < work_len; i++) {
    double val = work[i];
    double mag = std::fabs(val);
    int j = i;
    while (j > 0 && std::fabs(work[j - 1]) < mag) {
      work[j] = work[j - 1];
      j--;
    }
    work[j] = val;
  }
  double ex[MAX_WORK];
  for (int i = 0; i < MAX_WORK; i++) ex[i] = 0.0;
  int exp_len = 0;
  for (int i = 0; i < work_len; i++) {
    double term = work[i];
    if (term == 0.0) continue;
    if (exp_len == 0) {
      ex[0] = term;
      exp_len = 1;
      continue;
    }
    double carry = term;
    for (int j = exp_len - 1; j >= 0; j--) {
      double s, e;
      two_sum(ex[j], carry, s, e);
      ex[j] = e;
      carry = s;
    }
    if (carry != 0.0) {
      int new_len = exp_len < MAX_WORK ? exp_len + 1 : MAX_WORK;
      for (int k = new_len - 1; k > 0; k--) ex[k] = ex[k - 1];
      ex[0] = carry;
      exp_len = new_len;
    }
  }
  mf<N> r = mf_zero<N>();
  for (int i = 0; i < N && i < exp_len; i++) r.l[i] = ex[i];
  mf_renormalize<N>(r.l);
  return r;
}
template <int N>
static inline mf<N> mf_sub(const mf<N>& a, const mf<N>& b) { return mf_add<N>(a, mf_neg<N>(b)); }  // add.rs:108-113

// mul.rs:12-111: convolution over i+j<N with cascaded accumulate, then
// renormalize_from<N, 2N>.
template <int N>
static inline void mf_accumulate(double* work, int idx, double val, int limit) {  // mul.rs:31-42
  double s, e;
  two_sum(work[idx], val, s, e);
  work[idx] = s;
  int k = idx + 1;
  while (e != 0.0 && k < limit) {
    double s2, e2;
    two_sum(work[k], e, s2, e2);
    work[k] = s2;
    e = e2;
    k++;
  }
}
template <int N>
static inline mf<N> mf_mul(const mf<N>& a, const mf<N>& b) {
  double work[16];
  for (int i = 0; i < 16; i++) work[i] = 0.0;
  const int limit = 2 * N;
  for (int i = 0; i < N; i++) {
    for (int j = 0; j < N; j++) {
      if (i + j >= N) break;
      double p, e;
      two_prod(a.l[i], b.l[j], p, e);
      mf_accumulate<N>(work, i + j, p, limit);
      if (i + j + 1 < limit) mf_accumulate<N>(work, i + j + 1, e, limit);
    }
  }
  mf<N> r;
  mf_renormalize_from<N, 2 * N>(work, r.l);
  return r;
}
// mul.rs:124-202 (MultiFloat * f64)
template <int N>
static inline mf<N> mf_mul_f64(const mf<N>& a, double rhs) {
  double work[16];
  for (int i = 0; i < 16; i++) work[i] = 0.0;
  for (int i = 0; i < N; i++) {
    double p, e, s, err;
    two_prod(a.l[i], rhs, p, e);
    two_sum(work[i], p, s, err);
    work[i] = s;
    if (i + 1 < 2 * N) {
      double s2, err2;
      two_sum(work[i + 1], e, s2, err2);
      work[i + 1] = s2;
      if (i + 2 < 2 * N) work[i + 2] += err2;
      double s3, err3;
      two_sum(work[i + 1], err, s3, err3);
      work[i + 1] = s3;
      if (i + 2 < 2 * N) work[i + 2] += err3;
    }
  }
  mf<N> r;
  mf_renormalize_from<N, 2 * N>(work, r.l);
  return r;
}
// conv.rs:67-82 (MultiFloat + f64)
template <int N>
static inline mf<N> mf_add_f64(const mf<N>& a, double rhs) {
  mf<N> r = a;
  double s, e;
  two_sum(r.l[0], rhs, s, e);
  r.l[0] = s;
  for (int i = 1; i < N; i++) {
    double e2;
    two_sum(r.l[i], e, s, e2);
    r.l[i] = s;
    e = e2;
  }
  mf_renormalize<N>(r.l);
  return r;
}

static inline int ceil_log2_int(int n) {  // (N as f64).log2().ceil() for N = 1..8
  int b = 0;
  while ((1 << b) < n) b++;
  return b;
}

// div.rs:14-41
template <int N>
static inline mf<N> mf_recip(const mf<N>& a) {
  if (a.l[0] == 0.0) {
    mf<N> r = mf_zero<N>();
    r.l[0] = std::signbit(a.l[0]) ? -INFINITY : INFINITY;
    return r;
  }
  if (!std::isfinite(a.l[0])) return mf_from<N>(0.0);
  mf<N> x = mf_from<N>(1.0 / a.l[0]);
  mf<N> one = mf_from<N>(1.0);
  int steps = N <= 1 ? 1 : ceil_log2_int(N) + 2;
  for (int s = 0; s < steps; s++) {
    mf<N> residual = mf_sub<N>(one, mf_mul<N>(a, x));
    x = mf_add<N>(x, mf_mul<N>(x, residual));
  }
  return x;
}
// div.rs:44-77
template <int N>
static inline mf<N> mf_div(const mf<N>& a, const mf<N>& b) {
  if (b.l[0] == 0.0) {
    double sign = (std::signbit(a.l[0]) == std::signbit(b.l[0])) ? 1.0 : -1.0;
    mf<N> r = mf_zero<N>();
    r.l[0] = (a.l[0] == 0.0) ? NAN : sign * INFINITY;
    return r;
  }
  if (a.l[0] == 0.0) return mf_zero<N>();
  if (!std::isfinite(a.l[0]) || !std::isfinite(b.l[0])) return mf_from<N>(a.l[0] / b.l[0]);
  return mf_mul<N>(a, mf_recip<N>(b));
}
template <int N>
static inline mf<N> mf_abs(const mf<N>& a) { return std::signbit(a.l[0]) ? mf_neg<N>(a) : a; }  // math.rs:14-20
// math.rs:22-40
template <int N>
static inline mf<N> mf_sqrt(const mf<N>& a) {
  if (a.l[0] < 0.0) return mf_from<N>(NAN);
  if (a.l[0] == 0.0) return mf_zero<N>();
  if (!std::isfinite(a.l[0])) return mf_from<N>(a.l[0]);
  mf<N> x = mf_from<N>(std::sqrt(a.l[0]));
  mf<N> half = mf_from<N>(0.5);
  int steps = ceil_log2_int(N) + 1;
  for (int s = 0; s < steps; s++) x = mf_mul<N>(mf_add<N>(x, mf_div<N>(a, x)), half);
  return x;
}

// transcendental.rs:4-23 (4-limb constants) and :140-148, :179-243 (exp)
static const double LN2_LIMBS_4[4] = {6.931471805599452862e-01, 2.319046813846299558e-17,
                                      5.707708438416212066e-34, -3.582432210601811423e-50};
template <int N>
static inline double mf_epsilon() {  // transcendental.rs:36-42
  double eps = 1.0;
  for (int i = 0; i < N; i++) eps *= 2.220446049250313e-16;
  return eps;
}
template <int N>
static inline bool mf_is_negligible(const mf<N>& t, double eps) {  // transcendental.rs:47-61
  double mag = std::fabs(t.l[0]);
  if (mag > eps) return false;
  if (mag == 0.0)
    for (int i = 1; i < N; i++)
      if (std::fabs(t.l[i]) > eps) return false;
  return true;
}
template <int N>
mf<N> mf_ln2();
template <int N>
static inline mf<N> mf_arctanh_series(const mf<N>& x) {  // transcendental.rs:78-96
  mf<N> x2 = mf_mul<N>(x, x), power = x, sum = x;
  double eps = mf_epsilon<N>();
  int mx = N * 20 * 2;
  for (int i = 1; i <= mx; i++) {
    power = mf_mul<N>(power, x2);
    mf<N> term = mf_div<N>(power, mf_from<N>((double)(2 * i + 1)));
    sum = mf_add<N>(sum, term);
    if (mf_is_negligible<N>(term, eps)) break;
  }
  return sum;
}
template <int N>
mf<N> mf_ln2() {  // transcendental.rs:126-131, 140-146
  if (N <= 4) {
    mf<N> r = mf_zero<N>();
    for (int i = 0; i < N && i < 4; i++) r.l[i] = LN2_LIMBS_4[i];
    mf_renormalize<N>(r.l);
    return r;
  }
  mf<N> third = mf_div<N>(mf_from<N>(1.0), mf_from<N>(3.0));
  return mf_mul<N>(mf_from<N>(2.0), mf_arctanh_series<N>(third));
}
template <int N>
static inline mf<N> mf_exp(const mf<N>& a) {  // transcendental.rs:179-243
  if (std::isnan(a.l[0])) return a;
  if (a.l[0] == 0.0) return mf_from<N>(1.0);
  if (!std::isfinite(a.l[0])) return a.l[0] > 0.0 ? mf_from<N>(INFINITY) : mf_zero<N>();
  if (a.l[0] > 709.0) return mf_from<N>(INFINITY);
  if (a.l[0] < -745.0) return mf_zero<N>();
  mf<N> ln2 = mf_ln2<N>();
  double k = std::round(a.l[0] / ln2.l[0]);
  mf<N> r = mf_sub<N>(a, mf_mul<N>(mf_from<N>(k), ln2));
  int m = N <= 2 ? 3 : N * 2;
  double scale_down = (double)(1ull << m);
  mf<N> rs = mf_div<N>(r, mf_from<N>(scale_down));
  mf<N> term = mf_from<N>(1.0), sum = mf_from<N>(1.0);
  double eps = mf_epsilon<N>();
  int max_terms = N * 20;
  for (int i = 1; i <= max_terms; i++) {
    term = mf_div<N>(mf_mul<N>(term, rs), mf_from<N>((double)i));
    sum = mf_add<N>(sum, term);
    if (mf_is_negligible<N>(term, eps)) break;
  }
  for (int i = 0; i < m; i++) sum = mf_mul<N>(sum, sum);
  int64_t ki = (int64_t)k;
  if (ki >= -1022 && ki <= 1023) {
    uint64_t bits = (uint64_t)(1023 + ki) << 52;
    double scale;
    std::memcpy(&scale, &bits, 8);
    return mf_mul<N>(sum, mf_from<N>(scale));
  }
  int64_t half = ki / 2, other = ki - half;
  uint64_t b1 = (uint64_t)(1023 + half) << 52, b2 = (uint64_t)(1023 + other) << 52;
  double s1, s2;
  std::memcpy(&s1, &b1, 8);
  std::memcpy(&s2, &b2, 8);
  return mf_mul<N>(mf_mul<N>(sum, mf_from<N>(s1)), mf_from<N>(s2));
}

}  // namespace oracle
