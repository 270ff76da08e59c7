// CPU oracle, C ABI for the test suite and bench.py's CPU baseline.
//
// TEST INFRASTRUCTURE ONLY (see hp_oracle.hpp). Restates hyperprec's Rust
// linear algebra (crates/quad/src/linalg.rs, crates/quad/src/multifloat/
// linalg.rs), its SPD solver (crates/solver/src/lib.rs, ortho.rs) and its
// s-type overlap assembly (crates/overlap/src/{integral,screen,assemble}.rs).
// rayon row-parallel loops become OpenMP loops over the same rows; each output
// is still computed by one thread in the reference's operation order, so the
// results do not depend on the thread count.
//
// Buffers are the reference's in-memory layouts: f128 = {hi, lo} (16 B),
// MultiFloat<N> = N doubles, most significant first; row-major, no padding.
#include "hp_oracle.hpp"

#include <algorithm>
#include <cfloat>
#include <omp.h>
#include <vector>

using namespace oracle;

namespace {
const size_t PAR_THRESHOLD = 64;  // linalg.rs:4, multifloat/linalg.rs:4

inline dd ld(const double* p, size_t i) { return dd{p[2 * i], p[2 * i + 1]}; }
inline void st(double* p, size_t i, dd v) {
  p[2 * i] = v.hi;
  p[2 * i + 1] = v.lo;
}
template <int N>
inline mf<N> ldm(const double* p, size_t i) {
  mf<N> r;
  for (int t = 0; t < N; t++) r.l[t] = p[N * i + t];
  return r;
}
template <int N>
inline void stm(double* p, size_t i, const mf<N>& v) {
  for (int t = 0; t < N; t++) p[N * i + t] = v.l[t];
}

// linalg.rs:42-96, operating on a vector<dd>.
int cholesky_vec(std::vector<dd>& a, size_t n, int64_t* pivot, double* value) {
  std::vector<dd> row_j(n, dd{0, 0});
  for (size_t j = 0; j < n; j++) {
    dd sum{0, 0};
    for (size_t k = 0; k < j; k++) {
      dd ljk = a[j * n + k];
      sum = dd_add(sum, dd_mul(ljk, ljk));
    }
    dd diag = dd_sub(a[j * n + j], sum);
    if (diag.hi <= 0.0) {
      if (pivot) *pivot = (int64_t)j;
      if (value) *value = dd_to_f64(diag);
      return -2;
    }
    dd ljj = dd_sqrt(diag);
    a[j * n + j] = ljj;
    dd ljj_inv = dd_recip(ljj);
    for (size_t k = 0; k < j; k++) row_j[k] = a[j * n + k];
    size_t remaining = n - j - 1;
    if (remaining == 0) continue;
    bool par = remaining >= PAR_THRESHOLD && j >= 4;
#pragma omp parallel for schedule(static) if (par)
    for (size_t idx = 0; idx < remaining; idx++) {
      dd* row = &a[(j + 1 + idx) * n];
      dd s{0, 0};
      for (size_t k = 0; k < j; k++) s = dd_add(s, dd_mul(row[k], row_j[k]));
      row[j] = dd_mul(dd_sub(row[j], s), ljj_inv);
    }
  }
  return 0;
}

// linalg.rs:224-235
void trsm_right_lt(const std::vector<dd>& l, size_t jb, std::vector<dd>& b, size_t m) {
  for (size_t j = 0; j < jb; j++) {
    dd ljj_inv = dd_recip(l[j * jb + j]);
    for (size_t i = 0; i < m; i++) {
      dd s = b[i * jb + j];
      for (size_t k = 0; k < j; k++) s = dd_sub(s, dd_mul(b[i * jb + k], l[j * jb + k]));
      b[i * jb + j] = dd_mul(s, ljj_inv);
    }
  }
}

std::vector<dd> load_vec(const double* p, size_t len) {
  std::vector<dd> v(len);
  for (size_t i = 0; i < len; i++) v[i] = ld(p, i);
  return v;
}
void store_vec(double* p, const std::vector<dd>& v) {
  for (size_t i = 0; i < v.size(); i++) st(p, i, v[i]);
}

// linalg.rs:99-108
std::vector<dd> forward_solve_v(const std::vector<dd>& l, const std::vector<dd>& b, size_t n) {
  std::vector<dd> y = b;
  for (size_t i = 0; i < n; i++) {
    for (size_t j = 0; j < i; j++) y[i] = dd_sub(y[i], dd_mul(l[i * n + j], y[j]));
    y[i] = dd_div(y[i], l[i * n + i]);
  }
  return y;
}
// linalg.rs:111-120
std::vector<dd> backward_solve_v(const std::vector<dd>& l, const std::vector<dd>& y, size_t n) {
  std::vector<dd> x = y;
  for (size_t ii = n; ii-- > 0;) {
    for (size_t j = ii + 1; j < n; j++) x[ii] = dd_sub(x[ii], dd_mul(l[j * n + ii], x[j]));
    x[ii] = dd_div(x[ii], l[ii * n + ii]);
  }
  return x;
}
// linalg.rs:129-147
std::vector<dd> matvec_v(const std::vector<dd>& a, const std::vector<dd>& x, size_t n) {
  std::vector<dd> y(n, dd{0, 0});
#pragma omp parallel for schedule(static) if (n >= PAR_THRESHOLD)
  for (size_t i = 0; i < n; i++) {
    dd s{0, 0};
    for (size_t j = 0; j < n; j++) s = dd_add(s, dd_mul(a[i * n + j], x[j]));
    y[i] = s;
  }
  return y;
}
// linalg.rs:185-194
double cond_estimate_v(const std::vector<dd>& l, size_t n) {
  double dmax = 0.0, dmin = DBL_MAX;
  for (size_t i = 0; i < n; i++) {
    double d = std::fabs(dd_to_f64(l[i * n + i]));
    dmax = std::fmax(dmax, d);
    dmin = std::fmin(dmin, d);
  }
  double r = dmax / dmin;
  return r * r;
}
// solver/src/lib.rs:243-249
double norm_f128_v(const std::vector<dd>& x) {
  dd s{0, 0};
  for (const dd& v : x) s = dd_add(s, dd_mul(v, v));
  return dd_to_f64(dd_sqrt(s));
}
// solver/src/lib.rs:237-241
double residual_norm_v(const std::vector<dd>& a, const std::vector<dd>& x, const std::vector<dd>& b,
                       size_t n) {
  std::vector<dd> ax = matvec_v(a, x, n);
  std::vector<dd> r(n);
  for (size_t i = 0; i < n; i++) r[i] = dd_sub(b[i], ax[i]);
  return norm_f128_v(r);
}

// Classical max-pivot Jacobi of solver/src/ortho.rs:60-145 (eigenvectors as
// columns).
void ortho_jacobi(std::vector<dd>& a, size_t n, std::vector<dd>& evals, std::vector<dd>& v) {
  v.assign(n * n, dd{0, 0});
  for (size_t i = 0; i < n; i++) v[i * n + i] = dd{1, 0};
  size_t max_iter = 100 * n * n;
  for (size_t it = 0; it < max_iter; it++) {
    double max_val = 0.0;
    size_t p = 0, q = 1;
    for (size_t i = 0; i < n; i++)
      for (size_t j = i + 1; j < n; j++) {
        double val = std::fabs(dd_to_f64(a[i * n + j]));
        if (val > max_val) {
          max_val = val;
          p = i;
          q = j;
        }
      }
    if (max_val < 1e-60) break;
    dd app = a[p * n + p], aqq = a[q * n + q], apq = a[p * n + q];
    dd diff = dd_sub(aqq, app);
    dd c, s;
    if (std::fabs(dd_to_f64(apq)) < 1e-70) {
      c = dd{1, 0};
      s = dd{0, 0};
    } else {
      dd tau = dd_div(diff, dd_add(apq, apq));
      dd tau_abs = dd_abs(tau);
      dd one{1, 0};
      dd den = dd_add(tau_abs, dd_sqrt(dd_add(one, dd_mul(tau, tau))));
      dd t = tau.hi >= 0.0 ? dd_div(one, den) : dd_div(dd_neg(one), den);
      c = dd_div(one, dd_sqrt(dd_add(one, dd_mul(t, t))));
      s = dd_mul(t, c);
    }
    for (size_t j = 0; j < n; j++) {
      if (j == p || j == q) continue;
      dd ajp = a[j * n + p], ajq = a[j * n + q];
      dd njp = dd_sub(dd_mul(c, ajp), dd_mul(s, ajq));
      dd njq = dd_add(dd_mul(s, ajp), dd_mul(c, ajq));
      a[j * n + p] = njp;
      a[p * n + j] = njp;
      a[j * n + q] = njq;
      a[q * n + j] = njq;
    }
    dd two{2, 0};
    dd new_pp = dd_add(dd_sub(dd_mul(dd_mul(c, c), app), dd_mul(dd_mul(dd_mul(two, c), s), apq)),
                       dd_mul(dd_mul(s, s), aqq));
    dd new_qq = dd_add(dd_add(dd_mul(dd_mul(s, s), app), dd_mul(dd_mul(dd_mul(two, c), s), apq)),
                       dd_mul(dd_mul(c, c), aqq));
    a[p * n + p] = new_pp;
    a[q * n + q] = new_qq;
    a[p * n + q] = dd{0, 0};
    a[q * n + p] = dd{0, 0};
    for (size_t i = 0; i < n; i++) {
      dd vip = v[i * n + p], viq = v[i * n + q];
      v[i * n + p] = dd_sub(dd_mul(c, vip), dd_mul(s, viq));
      v[i * n + q] = dd_add(dd_mul(s, vip), dd_mul(c, viq));
    }
  }
  evals.resize(n);
  for (size_t i = 0; i < n; i++) evals[i] = a[i * n + i];
}

template <int N>
int mf_cholesky_t(double* a, size_t n) {  // multifloat/linalg.rs:89-141
  std::vector<mf<N>> row_j(n, mf_zero<N>());
  for (size_t j = 0; j < n; j++) {
    mf<N> sum = mf_zero<N>();
    for (size_t k = 0; k < j; k++) {
      mf<N> ljk = ldm<N>(a, j * n + k);
      sum = mf_add<N>(sum, mf_mul<N>(ljk, ljk));
    }
    mf<N> diag = mf_sub<N>(ldm<N>(a, j * n + j), sum);
    if (diag.l[0] <= 0.0) return -2;
    mf<N> ljj = mf_sqrt<N>(diag);
    stm<N>(a, j * n + j, ljj);
    mf<N> ljj_inv = mf_recip<N>(ljj);
    for (size_t k = 0; k < j; k++) row_j[k] = ldm<N>(a, j * n + k);
    size_t remaining = n - j - 1;
    if (remaining == 0) continue;
    bool par = remaining >= PAR_THRESHOLD && j >= 4;
#pragma omp parallel for schedule(static) if (par)
    for (size_t idx = 0; idx < remaining; idx++) {
      size_t r = j + 1 + idx;
      mf<N> s = mf_zero<N>();
      for (size_t k = 0; k < j; k++) s = mf_add<N>(s, mf_mul<N>(ldm<N>(a, r * n + k), row_j[k]));
      stm<N>(a, r * n + j, mf_mul<N>(mf_sub<N>(ldm<N>(a, r * n + j), s), ljj_inv));
    }
  }
  return 0;
}

template <int N>
void mf_cholesky_solve_t(const double* l, const double* b, double* x, size_t n) {
  // multifloat/linalg.rs:145-172
  std::vector<mf<N>> y(n);
  for (size_t i = 0; i < n; i++) y[i] = ldm<N>(b, i);
  for (size_t i = 0; i < n; i++) {
    for (size_t j = 0; j < i; j++) y[i] = mf_sub<N>(y[i], mf_mul<N>(ldm<N>(l, i * n + j), y[j]));
    y[i] = mf_div<N>(y[i], ldm<N>(l, i * n + i));
  }
  std::vector<mf<N>> xv = y;
  for (size_t ii = n; ii-- > 0;) {
    for (size_t j = ii + 1; j < n; j++)
      xv[ii] = mf_sub<N>(xv[ii], mf_mul<N>(ldm<N>(l, j * n + ii), xv[j]));
    xv[ii] = mf_div<N>(xv[ii], ldm<N>(l, ii * n + ii));
  }
  for (size_t i = 0; i < n; i++) stm<N>(x, i, xv[i]);
}

template <int N>
void mf_gemm_t(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, bool atb,
               size_t row0, size_t row1) {
  // multifloat/linalg.rs:39-61 (gemm) and :64-85 (gemm_atb)
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t i = row0; i < row1; i++) {
    for (size_t j = 0; j < n; j++) {
      mf<N> s = mf_zero<N>();
      for (size_t p = 0; p < k; p++) {
        mf<N> av = atb ? ldm<N>(a, p * m + i) : ldm<N>(a, i * k + p);
        s = mf_add<N>(s, mf_mul<N>(av, ldm<N>(b, p * n + j)));
      }
      stm<N>(c, i * n + j, s);
    }
  }
}

template <int N>
void mf_gemv_t(const double* a, const double* x, double* y, size_t n, size_t m) {
  // multifloat/linalg.rs:17-36
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) {
    mf<N> s = mf_zero<N>();
    for (size_t j = 0; j < m; j++) s = mf_add<N>(s, mf_mul<N>(ldm<N>(a, i * m + j), ldm<N>(x, j)));
    stm<N>(y, i, s);
  }
}

// ---- overlap (s-type) ----
double dist2_f64(const double* a, const double* b) {  // integral.rs:355-360, screen.rs:104-109
  double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return dx * dx + dy * dy + dz * dz;
}
double overlap_primitive_f64(double ai, const double* ci, double aj, const double* cj) {
  // integral.rs:15-25
  double gamma = ai + aj;
  double mu = ai * aj / gamma;
  double r2 = dist2_f64(ci, cj);
  double t = std::sqrt(M_PI / gamma);
  double prefactor = t * t * t;  // powi(3)
  return prefactor * std::exp(-mu * r2);
}
dd overlap_primitive_f128(double ai_, const double* ci, double aj_, const double* cj) {
  // integral.rs:29-56
  dd ai = dd_from(ai_), aj = dd_from(aj_);
  dd gamma = dd_add(ai, aj);
  dd mu = dd_div(dd_mul(ai, aj), gamma);
  dd dx = dd_from(ci[0] - cj[0]), dy = dd_from(ci[1] - cj[1]), dz = dd_from(ci[2] - cj[2]);
  dd r2 = dd_add(dd_add(dd_mul(dx, dx), dd_mul(dy, dy)), dd_mul(dz, dz));
  dd pi = dd_from(M_PI);
  dd ratio = dd_div(pi, gamma);
  dd prefactor = dd_mul(ratio, dd_sqrt(ratio));
  dd neg_mu_r2 = dd_mul(dd_sub(dd{0, 0}, mu), r2);
  dd exp_hi = dd_from(std::exp(neg_mu_r2.hi));
  dd exp_val = dd_mul(exp_hi, dd_add(dd{1, 0}, dd_from(neg_mu_r2.lo)));
  return dd_mul(prefactor, exp_val);
}
}  // namespace

// Normalised s-Gaussian pair overlap in f128 arithmetic:
//   S = (4 a b / (a+b)^2)^{3/4} * exp(-a b/(a+b) * |R-R'|^2)
// with the reference's f128 ops (dd.rs:61-121, including its Taylor exp).
// This is the definition of the dd problem matrix for the overlap SPD
// workloads; the CUDA kernel evaluates the identical op sequence.
// Exponents below -700 are flushed to S = 0 (true value < 1e-304), because
// dd.rs:119's bit trick for 2^k is only valid for k >= -1022.
static dd overlap_norm_dd(double a_, const double* ca, double b_, const double* cb) {
  dd a = dd_from(a_), b = dd_from(b_);
  dd sum = dd_add(a, b);
  dd prod = dd_mul(a, b);
  dd ratio = dd_div(dd_mul(dd_from(4.0), prod), dd_mul(sum, sum));
  dd sq = dd_sqrt(ratio);
  dd pref = dd_mul(sq, dd_sqrt(sq));
  dd mu = dd_div(prod, sum);
  dd dx = dd_sub(dd_from(ca[0]), dd_from(cb[0]));
  dd dy = dd_sub(dd_from(ca[1]), dd_from(cb[1]));
  dd dz = dd_sub(dd_from(ca[2]), dd_from(cb[2]));
  dd r2 = dd_add(dd_add(dd_mul(dx, dx), dd_mul(dy, dy)), dd_mul(dz, dz));
  dd arg = dd_neg(dd_mul(mu, r2));
  if (arg.hi < -700.0) return dd{0.0, 0.0};
  return dd_mul(pref, dd_exp(arg));
}

extern "C" {

int or_num_threads(void) { return omp_get_max_threads(); }
void or_set_num_threads(int t) { omp_set_num_threads(t); }

// ---- scalar f128 ops (dd.rs) ----
void or_dd_add(const double* a, const double* b, double* o) { st(o, 0, dd_add(ld(a, 0), ld(b, 0))); }
void or_dd_sub(const double* a, const double* b, double* o) { st(o, 0, dd_sub(ld(a, 0), ld(b, 0))); }
void or_dd_mul(const double* a, const double* b, double* o) { st(o, 0, dd_mul(ld(a, 0), ld(b, 0))); }
void or_dd_div(const double* a, const double* b, double* o) { st(o, 0, dd_div(ld(a, 0), ld(b, 0))); }
void or_dd_sqrt(const double* a, double* o) { st(o, 0, dd_sqrt(ld(a, 0))); }
void or_dd_recip(const double* a, double* o) { st(o, 0, dd_recip(ld(a, 0))); }
void or_dd_exp(const double* a, double* o) { st(o, 0, dd_exp(ld(a, 0))); }
void or_dd_ln(const double* a, double* o) { st(o, 0, dd_ln(ld(a, 0))); }

// ---- scalar MultiFloat<N> ops, N in {2, 4, 8} ----
#define MF_DISPATCH(N, CALL)      \
  switch (N) {                    \
    case 2: { CALL(2); } break;   \
    case 4: { CALL(4); } break;   \
    case 8: { CALL(8); } break;   \
    default: return -1;           \
  }                               \
  return 0;
int or_mf_add(int N, const double* a, const double* b, double* o) {
#define C(K) stm<K>(o, 0, mf_add<K>(ldm<K>(a, 0), ldm<K>(b, 0)))
  MF_DISPATCH(N, C)
#undef C
}
int or_mf_mul(int N, const double* a, const double* b, double* o) {
#define C(K) stm<K>(o, 0, mf_mul<K>(ldm<K>(a, 0), ldm<K>(b, 0)))
  MF_DISPATCH(N, C)
#undef C
}
int or_mf_div(int N, const double* a, const double* b, double* o) {
#define C(K) stm<K>(o, 0, mf_div<K>(ldm<K>(a, 0), ldm<K>(b, 0)))
  MF_DISPATCH(N, C)
#undef C
}
int or_mf_sqrt(int N, const double* a, double* o) {
#define C(K) stm<K>(o, 0, mf_sqrt<K>(ldm<K>(a, 0)))
  MF_DISPATCH(N, C)
#undef C
}
int or_mf_exp(int N, const double* a, double* o) {
#define C(K) stm<K>(o, 0, mf_exp<K>(ldm<K>(a, 0)))
  MF_DISPATCH(N, C)
#undef C
}
int or_mf_renormalize(int N, double* a) {
#define C(K) mf_renormalize<K>(a)
  MF_DISPATCH(N, C)
#undef C
}

// ---- f128 linear algebra (linalg.rs) ----
// linalg.rs:150-165 / :168-182. Rows [row0, row1) of C only (bench samples).
void or_f128_gemm_rows(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                       int atb, size_t row0, size_t row1) {
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t i = row0; i < row1; i++) {
    for (size_t j = 0; j < n; j++) {
      dd s{0, 0};
      if (atb)
        for (size_t p = 0; p < k; p++) s = dd_add(s, dd_mul(ld(a, p * m + i), ld(b, p * n + j)));
      else
        for (size_t p = 0; p < k; p++) s = dd_add(s, dd_mul(ld(a, i * k + p), ld(b, p * n + j)));
      st(c, i * n + j, s);
    }
  }
}
void or_f128_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k) {
  or_f128_gemm_rows(a, b, c, m, n, k, 0, 0, m);
}
void or_f128_gemm_atb(const double* a, const double* b, double* c, size_t m, size_t n, size_t k) {
  or_f128_gemm_rows(a, b, c, m, n, k, 1, 0, m);
}
// Single entries C[i][j] (for sampled checks at large sizes).
void or_f128_gemm_entries(const double* a, const double* b, double* out, size_t m, size_t n,
                          size_t k, int atb, const int64_t* idx, size_t count) {
#pragma omp parallel for schedule(static)
  for (size_t t = 0; t < count; t++) {
    size_t i = (size_t)idx[2 * t], j = (size_t)idx[2 * t + 1];
    dd s{0, 0};
    for (size_t p = 0; p < k; p++)
      s = dd_add(s, dd_mul(atb ? ld(a, p * m + i) : ld(a, i * k + p), ld(b, p * n + j)));
    st(out, t, s);
  }
}
// linalg.rs:7-26 (dot). rayon's reduction tree over 1024-element chunks is
// replaced by a left fold over the same chunks (deterministic).
void or_f128_dot(const double* a, const double* b, size_t len, double* out) {
  dd total{0, 0};
  const size_t CHUNK = 1024;
  if (len < CHUNK) {
    for (size_t i = 0; i < len; i++) total = dd_add(total, dd_mul(ld(a, i), ld(b, i)));
  } else {
    for (size_t c0 = 0; c0 < len; c0 += CHUNK) {
      dd s{0, 0};
      for (size_t i = c0; i < std::min(len, c0 + CHUNK); i++) s = dd_add(s, dd_mul(ld(a, i), ld(b, i)));
      total = dd_add(total, s);
    }
  }
  st(out, 0, total);
}
// linalg.rs:29-38
void or_f128_gemv(const double* a, size_t rows, size_t cols, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < rows; i++) {
    dd s{0, 0};
    for (size_t j = 0; j < cols; j++) s = dd_add(s, dd_mul(ld(a, i * cols + j), ld(x, j)));
    st(y, i, s);
  }
}
void or_f128_matvec(const double* a, const double* x, double* y, size_t n) {
  std::vector<dd> av = load_vec(a, n * n), xv = load_vec(x, n);
  store_vec(y, matvec_v(av, xv, n));
}
int or_f128_cholesky(double* a, size_t n, int64_t* pivot, double* value) {
  std::vector<dd> v = load_vec(a, n * n);
  int rc = cholesky_vec(v, n, pivot, value);
  if (rc == 0) store_vec(a, v);
  return rc;
}
// linalg.rs:238-293
int or_f128_cholesky_blocked(double* a_, size_t n, size_t nb, int64_t* pivot, double* value) {
  if (n == 0) return 0;
  if (nb == 0) nb = 64;
  std::vector<dd> a = load_vec(a_, n * n);
  std::vector<dd> diag_buf(nb * nb), panel_buf(n * nb);
  size_t j_block = 0;
  while (j_block < n) {
    size_t jb = std::min(nb, n - j_block);
    std::vector<dd> d(jb * jb);
    for (size_t i = 0; i < jb; i++)
      for (size_t j = 0; j < jb; j++) d[i * jb + j] = a[(j_block + i) * n + j_block + j];
    int64_t pv = 0;
    double val = 0;
    if (cholesky_vec(d, jb, &pv, &val) != 0) {
      if (pivot) *pivot = pv + (int64_t)j_block;
      if (value) *value = val;
      return -2;
    }
    for (size_t i = 0; i < jb; i++)
      for (size_t j = 0; j < jb; j++) a[(j_block + i) * n + j_block + j] = d[i * jb + j];
    size_t remaining = n - j_block - jb;
    if (remaining > 0) {
      std::vector<dd> panel(remaining * jb);
      for (size_t i = 0; i < remaining; i++)
        for (size_t j = 0; j < jb; j++) panel[i * jb + j] = a[(j_block + jb + i) * n + j_block + j];
      trsm_right_lt(d, jb, panel, remaining);
      for (size_t i = 0; i < remaining; i++)
        for (size_t j = 0; j < jb; j++) a[(j_block + jb + i) * n + j_block + j] = panel[i * jb + j];
      size_t ts = j_block + jb;
#pragma omp parallel for schedule(dynamic, 4) if (remaining >= PAR_THRESHOLD)
      for (size_t i = 0; i < remaining; i++) {
        for (size_t cj = 0; cj <= i; cj++) {
          dd s{0, 0};
          for (size_t k = 0; k < jb; k++) s = dd_add(s, dd_mul(panel[i * jb + k], panel[cj * jb + k]));
          a[(ts + i) * n + ts + cj] = dd_sub(a[(ts + i) * n + ts + cj], s);
        }
      }
    }
    j_block += jb;
  }
  store_vec(a_, a);
  return 0;
}
void or_f128_forward_solve(const double* l, const double* b, double* y, size_t n) {
  store_vec(y, forward_solve_v(load_vec(l, n * n), load_vec(b, n), n));
}
void or_f128_backward_solve(const double* l, const double* y, double* x, size_t n) {
  store_vec(x, backward_solve_v(load_vec(l, n * n), load_vec(y, n), n));
}
void or_f128_solve_cholesky(const double* l, const double* b, double* x, size_t n) {
  std::vector<dd> lv = load_vec(l, n * n);
  store_vec(x, backward_solve_v(lv, forward_solve_v(lv, load_vec(b, n), n), n));
}
double or_f128_cond_estimate(const double* l, size_t n) { return cond_estimate_v(load_vec(l, n * n), n); }

// linalg.rs:299-362. Returns 0, or -3 when max_iter sweeps do not converge.
int or_f128_jacobi_eigen(const double* a_, size_t n, size_t max_iter, double* evals_out,
                         double* evecs_out, size_t* sweeps_out) {
  std::vector<dd> s = load_vec(a_, n * n);
  std::vector<dd> v(n * n, dd{0, 0});
  for (size_t i = 0; i < n; i++) v[i * n + i] = dd{1, 0};
  const dd threshold = dd_from(1e-30);
  const dd tiny = dd_from(1e-60);
  for (size_t it = 0; it < max_iter; it++) {
    dd off{0, 0};
    for (size_t i = 0; i < n; i++)
      for (size_t j = i + 1; j < n; j++) {
        dd val = s[i * n + j];
        off = dd_add(off, dd_mul(val, val));
      }
    off = dd_sqrt(off);
    if (dd_lt(off, threshold)) {
      for (size_t i = 0; i < n; i++) st(evals_out, i, s[i * n + i]);
      for (size_t i = 0; i < n; i++)
        for (size_t j = 0; j < n; j++) st(evecs_out, i * n + j, v[j * n + i]);
      if (sweeps_out) *sweeps_out = it;
      return 0;
    }
    for (size_t p = 0; p < n; p++) {
      for (size_t q = p + 1; q < n; q++) {
        dd apq = s[p * n + q];
        if (dd_lt(dd_abs(apq), tiny)) continue;
        dd app = s[p * n + p], aqq = s[q * n + q];
        dd tau = dd_div(dd_sub(aqq, app), dd_mul(dd_from(2.0), apq));
        dd tau_abs = dd_abs(tau);
        dd one = dd_from(1.0);
        dd t_denom = dd_add(tau_abs, dd_sqrt(dd_add(one, dd_mul(tau, tau))));
        dd t = tau.hi >= 0.0 ? dd_div(one, t_denom) : dd_div(dd_neg(one), t_denom);
        dd c = dd_div(one, dd_sqrt(dd_add(one, dd_mul(t, t))));
        dd s_rot = dd_mul(t, c);
        s[p * n + p] = dd_sub(app, dd_mul(t, apq));
        s[q * n + q] = dd_add(aqq, dd_mul(t, apq));
        s[p * n + q] = dd{0, 0};
        s[q * n + p] = dd{0, 0};
        for (size_t r = 0; r < n; r++) {
          if (r == p || r == q) continue;
          dd srp = s[r * n + p], srq = s[r * n + q];
          dd np = dd_sub(dd_mul(c, srp), dd_mul(s_rot, srq));
          dd nq = dd_add(dd_mul(s_rot, srp), dd_mul(c, srq));
          s[r * n + p] = np;
          s[p * n + r] = np;
          s[r * n + q] = nq;
          s[q * n + r] = nq;
        }
        for (size_t r = 0; r < n; r++) {
          dd vrp = v[r * n + p], vrq = v[r * n + q];
          v[r * n + p] = dd_sub(dd_mul(c, vrp), dd_mul(s_rot, vrq));
          v[r * n + q] = dd_add(dd_mul(s_rot, vrp), dd_mul(c, vrq));
        }
      }
    }
  }
  if (sweeps_out) *sweeps_out = max_iter;
  return -3;
}

// ---- MultiFloat<N> linear algebra (multifloat/linalg.rs) ----
int or_mf_gemm_rows(int N, const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                    int atb, size_t row0, size_t row1) {
#define C(K) mf_gemm_t<K>(a, b, c, m, n, k, atb != 0, row0, row1)
  MF_DISPATCH(N, C)
#undef C
}
int or_mf_gemm(int N, const double* a, const double* b, double* c, size_t m, size_t n, size_t k) {
  return or_mf_gemm_rows(N, a, b, c, m, n, k, 0, 0, m);
}
int or_mf_gemm_atb(int N, const double* a, const double* b, double* c, size_t m, size_t n, size_t k) {
  return or_mf_gemm_rows(N, a, b, c, m, n, k, 1, 0, m);
}
int or_mf_gemm_entries(int N, const double* a, const double* b, double* out, size_t m, size_t n,
                       size_t k, int atb, const int64_t* idx, size_t count) {
#define C(K)                                                                          \
  _Pragma("omp parallel for schedule(dynamic, 1)") for (size_t t = 0; t < count; t++) { \
    size_t i = (size_t)idx[2 * t], j = (size_t)idx[2 * t + 1];                        \
    mf<K> s = mf_zero<K>();                                                           \
    for (size_t p = 0; p < k; p++)                                                    \
      s = mf_add<K>(s, mf_mul<K>(atb ? ldm<K>(a, p * m + i) : ldm<K>(a, i * k + p),   \
                                 ldm<K>(b, p * n + j)));                              \
    stm<K>(out, t, s);                                                                \
  }
  MF_DISPATCH(N, C)
#undef C
}
// f512 (MultiFloat<8>) entries of C = op(A) B for f128 (in_limbs = 2) or f256
// (in_limbs = 4) inputs, each promoted exactly to MultiFloat<8> (the f512
// checker of the GEMMs: every product of two 2- or 4-limb values and their
// running sum is held to ~2^-420). out: count x 4 (the leading limbs of the
// f512 value); absab: count doubles, sum_p |a_ip| |b_pj| over the leading limbs
// (the normwise denominator).
int or_gemm_entries_f512(int in_limbs, const double* a, const double* b, double* out, double* absab, size_t m,
                         size_t n, size_t k, int atb, const int64_t* idx, size_t count) {
  if (in_limbs != 2 && in_limbs != 4) return -1;
  const size_t L = (size_t)in_limbs;
  auto ld8 = [&](const double* p, size_t e) {
    mf<8> r = mf_zero<8>();
    for (size_t t = 0; t < L; t++) r.l[t] = p[L * e + t];
    return r;
  };
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t t = 0; t < count; t++) {
    const size_t i = (size_t)idx[2 * t], j = (size_t)idx[2 * t + 1];
    mf<8> s = mf_zero<8>();
    double ab = 0.0;
    for (size_t p = 0; p < k; p++) {
      const size_t ea = atb ? p * m + i : i * k + p, eb = p * n + j;
      s = mf_add<8>(s, mf_mul<8>(ld8(a, ea), ld8(b, eb)));
      ab += std::fabs(a[L * ea]) * std::fabs(b[L * eb]);
    }
    for (int q = 0; q < 4; q++) out[4 * t + q] = s.l[q];
    absab[t] = ab;
  }
  return 0;
}
int or_mf_gemv(int N, const double* a, const double* x, double* y, size_t n, size_t m) {
#define C(K) mf_gemv_t<K>(a, x, y, n, m)
  MF_DISPATCH(N, C)
#undef C
}
int or_mf_cholesky(int N, double* a, size_t n) {
  switch (N) {
    case 2: return mf_cholesky_t<2>(a, n);
    case 4: return mf_cholesky_t<4>(a, n);
    case 8: return mf_cholesky_t<8>(a, n);
    default: return -1;
  }
}
int or_mf_cholesky_solve(int N, const double* l, const double* b, double* x, size_t n) {
#define C(K) mf_cholesky_solve_t<K>(l, b, x, n)
  MF_DISPATCH(N, C)
#undef C
}

// ---- solver (crates/solver/src/lib.rs) ----
// Outputs: x (f128, n), x_f64 (n), info[0]=kappa, info[1]=residual_norm,
// info[2]=strategy (0 Float64, 1 MixedPrecision, 2 Float128),
// info[3]=refinement_iters. Returns 0, or -2 with *pivot on a non-SPD matrix.
static void finish_solution(const std::vector<dd>& x128, double* x_out, double* xf_out) {
  for (size_t i = 0; i < x128.size(); i++) {
    st(x_out, i, x128[i]);
    if (xf_out) xf_out[i] = dd_to_f64(x128[i]);
  }
}
// lib.rs:127-144
static int solve_pure_f128_v(const std::vector<dd>& a128, const std::vector<dd>& b128, size_t n,
                             double* x_out, double* xf_out, double* info, int64_t* pivot) {
  std::vector<dd> l = a128;
  int64_t pv = 0;
  double val = 0;
  if (cholesky_vec(l, n, &pv, &val) != 0) {
    if (pivot) *pivot = pv;
    return -2;
  }
  double kappa = cond_estimate_v(l, n);
  std::vector<dd> x = backward_solve_v(l, forward_solve_v(l, b128, n), n);
  finish_solution(x, x_out, xf_out);
  info[0] = kappa;
  info[1] = residual_norm_v(a128, x, b128, n);
  info[2] = 2;
  info[3] = 0;
  return 0;
}
// Refined SPD solve to ~1e-25 on the host (the CPU counterpart of the GPU's
// plain refined mode, used as its timed baseline): the reference's f128
// cholesky (linalg.rs:42-96) and solve_cholesky (linalg.rs:123-126), and the
// iterative_refinement loop of solver/src/lib.rs:75-125 with its residual
// evaluated in MultiFloat<4> (mf_gemv semantics, multifloat/linalg.rs:17-37:
// S and x promoted exactly, r = b - S x accumulated in f256 and rounded to
// f128) instead of f128, until max|dx| <= tol max|x| or max_iter steps.
// S: n x n f128, b: n f128; x: n f128. Returns the steps taken, or -2 if
// the factorisation fails.
int or_spd_solve_refined(const double* S, const double* b, size_t n, double tol, int max_iter, double* x_out) {
  std::vector<dd> L = load_vec(S, n * n);
  int64_t pv;
  double val;
  if (cholesky_vec(L, n, &pv, &val) != 0) return -2;
  const std::vector<dd> bv = load_vec(b, n);
  std::vector<dd> x = backward_solve_v(L, forward_solve_v(L, bv, n), n);
  int it = 0;
  for (; it < max_iter; it++) {
    std::vector<dd> r(n);
#pragma omp parallel for schedule(static) if (n >= PAR_THRESHOLD)
    for (size_t i = 0; i < n; i++) {
      mf<4> acc = mf_zero<4>();
      for (size_t j = 0; j < n; j++) {
        mf<4> sij = mf_zero<4>(), xj = mf_zero<4>();
        sij.l[0] = S[2 * (i * n + j)];
        sij.l[1] = S[2 * (i * n + j) + 1];
        xj.l[0] = x[j].hi;
        xj.l[1] = x[j].lo;
        acc = mf_add<4>(acc, mf_mul<4>(sij, xj));
      }
      mf<4> bi = mf_zero<4>();
      bi.l[0] = bv[i].hi;
      bi.l[1] = bv[i].lo;
      const mf<4> ri = mf_sub<4>(bi, acc);
      r[i] = dd_renorm(ri.l[0], ri.l[1] + ri.l[2]);
    }
    const std::vector<dd> dx = backward_solve_v(L, forward_solve_v(L, r, n), n);
    double mdx = 0.0, mx = 0.0;
    for (size_t i = 0; i < n; i++) {
      x[i] = dd_add(x[i], dx[i]);
      mdx = std::max(mdx, std::fabs(dx[i].hi));
      mx = std::max(mx, std::fabs(x[i].hi));
    }
    if (mdx <= tol * mx) {
      it++;
      break;
    }
  }
  store_vec(x_out, x);
  return it;
}
// A batch of overlap SPD systems solved on the host (the CPU counterpart of
// the GPU's batched solver): OpenMP over systems, each assembled in f128
// (the normalised s-Gaussian formula, dd.rs arithmetic) and solved by
// or_spd_solve_refined on one thread. System s owns basis functions
// offsets[s] .. offsets[s+1]-1 (centres 3 doubles, exponents, b f64); x is
// f128 per basis function; iters[s] = steps taken or -2 (not SPD).
int or_batched_refined(int count, const int64_t* offsets, const double* centers, const double* alpha,
                       const double* b, double tol, int max_iter, double* x, int32_t* iters) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int s = 0; s < count; s++) {
    const size_t o = (size_t)offsets[s], n = (size_t)(offsets[s + 1] - offsets[s]);
    std::vector<double> S(n * n * 2), bb(n * 2, 0.0);
    for (size_t i = 0; i < n; i++) {
      bb[2 * i] = b[o + i];
      for (size_t j = 0; j <= i; j++) {
        const dd v = overlap_norm_dd(alpha[o + i], centers + 3 * (o + i), alpha[o + j], centers + 3 * (o + j));
        st(S.data(), i * n + j, v);
        st(S.data(), j * n + i, v);
      }
    }
    iters[s] = or_spd_solve_refined(S.data(), bb.data(), n, tol, max_iter, x + 2 * o);
  }
  return 0;
}

int or_solve_spd_f128(const double* a, const double* b, size_t n, double* x_out, double* xf_out,
                      double* info, int64_t* pivot) {
  return solve_pure_f128_v(load_vec(a, n * n), load_vec(b, n), n, x_out, xf_out, info, pivot);
}
// lib.rs:38-68, with the non-macOS f64 path (:168-213) and IR (:75-125).
int or_solve_spd(const double* a_f64, const double* b_f64, size_t n, double* x_out, double* xf_out,
                 double* info, int64_t* pivot) {
  std::vector<dd> a128(n * n), b128(n);
  for (size_t i = 0; i < n * n; i++) a128[i] = dd_from(a_f64[i]);
  for (size_t i = 0; i < n; i++) b128[i] = dd_from(b_f64[i]);
  // cholesky_f64 (lib.rs:169-195)
  std::vector<double> l(a_f64, a_f64 + n * n);
  bool ok = true;
  for (size_t j = 0; j < n && ok; j++) {
    double sum = 0.0;
    for (size_t k = 0; k < j; k++) sum += l[j * n + k] * l[j * n + k];
    double diag = l[j * n + j] - sum;
    if (diag <= 0.0) {
      ok = false;
      break;
    }
    double ljj = std::sqrt(diag);
    l[j * n + j] = ljj;
    double inv = 1.0 / ljj;
    for (size_t i = j + 1; i < n; i++) {
      double s = 0.0;
      for (size_t k = 0; k < j; k++) s += l[i * n + k] * l[j * n + k];
      l[i * n + j] = (l[i * n + j] - s) * inv;
    }
    for (size_t i = 0; i < j; i++) l[i * n + j] = 0.0;
  }
  if (!ok) return solve_pure_f128_v(a128, b128, n, x_out, xf_out, info, pivot);
  // solve_cholesky_f64 (lib.rs:198-213)
  std::vector<double> y(b_f64, b_f64 + n);
  for (size_t i = 0; i < n; i++) {
    for (size_t j = 0; j < i; j++) y[i] -= l[i * n + j] * y[j];
    y[i] /= l[i * n + i];
  }
  for (size_t ii = n; ii-- > 0;) {
    for (size_t j = ii + 1; j < n; j++) y[ii] -= l[j * n + ii] * y[j];
    y[ii] /= l[ii * n + ii];
  }
  // cond_estimate_f64 (lib.rs:215-224)
  double dmax = 0.0, dmin = DBL_MAX;
  for (size_t i = 0; i < n; i++) {
    double d = std::fabs(l[i * n + i]);
    dmax = std::fmax(dmax, d);
    dmin = std::fmin(dmin, d);
  }
  double kappa = (dmax / dmin) * (dmax / dmin);
  if (kappa < 1e10) {
    std::vector<dd> x128(n);
    for (size_t i = 0; i < n; i++) x128[i] = dd_from(y[i]);
    for (size_t i = 0; i < n; i++) {
      st(x_out, i, x128[i]);
      if (xf_out) xf_out[i] = y[i];
    }
    info[0] = kappa;
    info[1] = residual_norm_v(a128, x128, b128, n);
    info[2] = 0;
    info[3] = 0;
    return 0;
  }
  // iterative_refinement (lib.rs:75-125)
  std::vector<dd> l128 = a128;
  int64_t pv = 0;
  double val = 0;
  if (cholesky_vec(l128, n, &pv, &val) != 0) {
    if (pivot) *pivot = pv;
    return -2;
  }
  double kappa128 = cond_estimate_v(l128, n);
  std::vector<dd> x128(n);
  for (size_t i = 0; i < n; i++) x128[i] = dd_from(y[i]);
  double bnorm = norm_f128_v(b128);
  double best = DBL_MAX;
  int iters = 0;
  for (int it = 0; it < 30; it++) {
    std::vector<dd> ax = matvec_v(a128, x128, n);
    std::vector<dd> r(n);
    for (size_t i = 0; i < n; i++) r[i] = dd_sub(b128[i], ax[i]);
    double rnorm = norm_f128_v(r);
    iters++;
    if (rnorm < 1e-28 * bnorm) break;
    if (iters > 3 && rnorm > 0.5 * best) break;
    if (rnorm < best) best = rnorm;
    std::vector<dd> dx = backward_solve_v(l128, forward_solve_v(l128, r, n), n);
    for (size_t i = 0; i < n; i++) x128[i] = dd_add(x128[i], dx[i]);
  }
  finish_solution(x128, x_out, xf_out);
  info[0] = kappa128;
  info[1] = residual_norm_v(a128, x128, b128, n);
  info[2] = 1;
  info[3] = iters;
  return 0;
}

// solver/src/ortho.rs:151-183. Writes X (n x n_orth, row-major, f128) and
// returns n_orth.
size_t or_canonical_orthogonalize(const double* s, size_t n, double threshold, double* x_out) {
  std::vector<dd> work = load_vec(s, n * n), evals, evecs;
  ortho_jacobi(work, n, evals, evecs);
  std::vector<std::pair<size_t, dd>> surv;
  for (size_t i = 0; i < n; i++)
    if (dd_to_f64(evals[i]) > threshold) surv.push_back({i, evals[i]});
  std::stable_sort(surv.begin(), surv.end(),
                   [](const std::pair<size_t, dd>& a, const std::pair<size_t, dd>& b) {
                     return dd_to_f64(a.second) < dd_to_f64(b.second);
                   });
  size_t m = surv.size();
  for (size_t k = 0; k < m; k++) {
    dd inv_sqrt = dd_recip(dd_sqrt(surv[k].second));
    for (size_t i = 0; i < n; i++) st(x_out, i * m + k, dd_mul(evecs[i * n + surv[k].first], inv_sqrt));
  }
  return m;
}

// solver/src/ortho.rs:41-55: C (m x p) = A (m x n) B (n x p), i-k-j order,
// zero a_ik skipped.
static std::vector<dd> gemm_rect_v(const std::vector<dd>& a, const std::vector<dd>& b, size_t m, size_t n,
                                   size_t p) {
  std::vector<dd> c(m * p, dd{0, 0});
  for (size_t i = 0; i < m; i++)
    for (size_t k = 0; k < n; k++) {
      const dd aik = a[i * n + k];
      if (aik.hi == 0.0 && aik.lo == 0.0) continue;
      for (size_t j = 0; j < p; j++) c[i * p + j] = dd_add(c[i * p + j], dd_mul(aik, b[k * p + j]));
    }
  return c;
}

// solver/src/ortho.rs:191-239. Writes the m eigenvalues (ascending) and C
// (n x m, row-major, column k = eigenvector k); returns m.
size_t or_solve_gen_eigen(const double* f, const double* s, size_t n, double threshold, double* evals_out,
                          double* c_out) {
  std::vector<double> xb(n * n * 2, 0.0);
  const size_t m = or_canonical_orthogonalize(s, n, threshold, xb.data());
  if (m == 0) return 0;
  std::vector<dd> x = load_vec(xb.data(), n * m), fm = load_vec(f, n * n);
  std::vector<dd> tmp = gemm_rect_v(fm, x, n, n, m);
  // F' = X^T tmp: linalg.rs:168-182 gemm_atb with A = X (k x m, k = n)
  std::vector<dd> fp(m * m);
  for (size_t i = 0; i < m; i++)
    for (size_t j = 0; j < m; j++) {
      dd acc{0, 0};
      for (size_t q = 0; q < n; q++) acc = dd_add(acc, dd_mul(x[q * m + i], tmp[q * m + j]));
      fp[i * m + j] = acc;
    }
  for (size_t i = 0; i < m; i++)
    for (size_t j = i + 1; j < m; j++) {
      const dd avg = dd_mul(dd_add(fp[i * m + j], fp[j * m + i]), dd{0.5, 0.0});
      fp[i * m + j] = avg;
      fp[j * m + i] = avg;
    }
  std::vector<dd> evals, evecs;
  ortho_jacobi(fp, m, evals, evecs);
  std::vector<size_t> order(m);
  for (size_t i = 0; i < m; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return dd_to_f64(evals[a]) < dd_to_f64(evals[b]); });
  std::vector<dd> sorted(m * m);
  for (size_t nk = 0; nk < m; nk++)
    for (size_t i = 0; i < m; i++) sorted[i * m + nk] = evecs[i * m + order[nk]];
  std::vector<dd> c = gemm_rect_v(x, sorted, n, m, m);
  for (size_t k = 0; k < m; k++) st(evals_out, k, evals[order[k]]);
  for (size_t q = 0; q < n * m; q++) st(c_out, q, c[q]);
  return m;
}

// ---- overlap (crates/overlap) ----
double or_overlap_primitive_f64(double ai, const double* ci, double aj, const double* cj) {
  return overlap_primitive_f64(ai, ci, aj, cj);
}
void or_overlap_primitive_f128(double ai, const double* ci, double aj, const double* cj, double* out) {
  st(out, 0, overlap_primitive_f128(ai, ci, aj, cj));
}
// screen.rs:57-101 for s shells. Returns 0 F64, 1 F128, 2 Skip.
static int screen_pair(const double* ca, const double* alpha_a, const int n_a, const double* cb,
                       const double* alpha_b, const int n_b, const double* params) {
  double r2 = dist2_f64(ca, cb);
  double amin_a = INFINITY, amin_b = INFINITY, amax_a = 0.0, amax_b = 0.0;
  for (int i = 0; i < n_a; i++) {
    amin_a = std::fmin(amin_a, alpha_a[i]);
    amax_a = std::fmax(amax_a, alpha_a[i]);
  }
  for (int i = 0; i < n_b; i++) {
    amin_b = std::fmin(amin_b, alpha_b[i]);
    amax_b = std::fmax(amax_b, alpha_b[i]);
  }
  double alpha_sum = amin_a + amin_b;
  double gamma = amin_a * amin_b / alpha_sum;
  double exponent = gamma * r2;
  if (exponent > -std::log(params[2])) return 2;
  bool ad = amin_a < params[0], bd = amin_b < params[0];
  if (!ad && !bd) return 0;
  double ratio = std::fmax(amax_a / amin_b, amax_b / amin_a);
  double r = std::sqrt(r2);
  if (ratio > params[1] && r < params[3]) return 1;
  if (ad && bd && r < params[3]) return 1;
  return 0;
}
// assemble.rs:35-85 for a basis of s shells. Shell s has centre centers[3s..],
// primitives prim_off[s]..prim_off[s+1] with (alpha, coeff). params =
// {diffuse_threshold, ratio_threshold, eps_skip, safe_distance}.
// tier_counts = {f64_pairs, f128_pairs, skipped_pairs}.
void or_assemble_overlap_s(size_t n_shells, const double* centers, const int64_t* prim_off,
                           const double* alpha, const double* coeff, const double* params,
                           double* matrix, int64_t* tier_counts) {
  size_t n = n_shells;
  std::fill(matrix, matrix + n * n, 0.0);
  std::vector<int> tiers(n * (n + 1) / 2);
  std::vector<double> vals(n * (n + 1) / 2);
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t i = 0; i < n; i++) {
    for (size_t j = 0; j <= i; j++) {
      size_t pidx = i * (i + 1) / 2 + j;
      const double *ci = centers + 3 * i, *cj = centers + 3 * j;
      int ni = (int)(prim_off[i + 1] - prim_off[i]), nj = (int)(prim_off[j + 1] - prim_off[j]);
      const double *ai = alpha + prim_off[i], *aj = alpha + prim_off[j];
      const double *ki = coeff + prim_off[i], *kj = coeff + prim_off[j];
      int tier = screen_pair(ci, ai, ni, cj, aj, nj, params);
      double v = 0.0;
      if (tier == 0) {  // integral.rs:175-187
        double sum = 0.0;
        for (int p = 0; p < ni; p++)
          for (int q = 0; q < nj; q++) sum += ki[p] * kj[q] * overlap_primitive_f64(ai[p], ci, aj[q], cj);
        v = sum;
      } else if (tier == 1) {  // integral.rs:202-215
        dd sum{0, 0};
        for (int p = 0; p < ni; p++)
          for (int q = 0; q < nj; q++) {
            dd sp = overlap_primitive_f128(ai[p], ci, aj[q], cj);
            sum = dd_add(sum, dd_mul(dd_mul(dd_from(ki[p]), dd_from(kj[q])), sp));
          }
        v = dd_to_f64(sum);
      }
      tiers[pidx] = tier;
      vals[pidx] = v;
    }
  }
  tier_counts[0] = tier_counts[1] = tier_counts[2] = 0;
  for (size_t i = 0; i < n; i++)
    for (size_t j = 0; j <= i; j++) {
      size_t pidx = i * (i + 1) / 2 + j;
      tier_counts[tiers[pidx]]++;
      if (tiers[pidx] == 2) continue;
      matrix[i * n + j] = vals[pidx];
      if (i != j) matrix[j * n + i] = vals[pidx];
    }
}
// ---- Obara-Saika overlaps of Cartesian shells (integral.rs:144-352) ----
namespace {
// integral.rs:156-186: S[i][j], i <= la, j <= lb, row stride lb + 1.
void os1d_f64(int la, int lb, double pa, double pb, double gamma, double* s) {
  const int nb = lb + 1;
  const double oo2g = 0.5 / gamma;
  for (int q = 0; q < (la + 1) * nb; q++) s[q] = 0.0;
  s[0] = 1.0;
  for (int i = 0; i < la; i++) s[(i + 1) * nb] = pa * s[i * nb] + oo2g * (double)i * (i > 0 ? s[(i - 1) * nb] : 0.0);
  for (int j = 0; j < lb; j++)
    for (int i = 0; i <= la; i++) {
      const double term_im1 = oo2g * (double)i * (i > 0 ? s[(i - 1) * nb + j] : 0.0);
      const double term_jm1 = oo2g * (double)j * (j > 0 ? s[i * nb + j - 1] : 0.0);
      s[i * nb + j + 1] = pb * s[i * nb + j] + term_im1 + term_jm1;
    }
}
// integral.rs:188-219
void os1d_f128(int la, int lb, dd pa, dd pb, dd gamma, dd* s) {
  const int nb = lb + 1;
  const dd oo2g = dd_div(dd_from(0.5), gamma);
  for (int q = 0; q < (la + 1) * nb; q++) s[q] = dd{0, 0};
  s[0] = dd_from(1.0);
  for (int i = 0; i < la; i++) {
    const dd fi = dd_from((double)i);
    const dd prev = i > 0 ? s[(i - 1) * nb] : dd{0, 0};
    s[(i + 1) * nb] = dd_add(dd_mul(pa, s[i * nb]), dd_mul(dd_mul(oo2g, fi), prev));
  }
  for (int j = 0; j < lb; j++) {
    const dd fj = dd_from((double)j);
    for (int i = 0; i <= la; i++) {
      const dd fi = dd_from((double)i);
      const dd im1 = i > 0 ? s[(i - 1) * nb + j] : dd{0, 0};
      const dd jm1 = j > 0 ? s[i * nb + j - 1] : dd{0, 0};
      s[i * nb + j + 1] =
          dd_add(dd_add(dd_mul(pb, s[i * nb + j]), dd_mul(dd_mul(oo2g, fi), im1)), dd_mul(dd_mul(oo2g, fj), jm1));
    }
  }
}
// integral.rs:223-233: (lx, ly, lz) with lx descending, then ly descending.
int cart_components(int l, int (*c)[3]) {
  int k = 0;
  for (int lx = l; lx >= 0; lx--)
    for (int ly = l - lx; ly >= 0; ly--) c[k][0] = lx, c[k][1] = ly, c[k][2] = l - lx - ly, k++;
  return k;
}
struct ShellRef {
  int l;
  const double* center;
  const double* alpha;
  const double* coeff;
  int np;
};
// integral.rs:235-284, block += over primitive pairs (ni x nj, row-major).
void os_contracted_f64(const ShellRef& A, const ShellRef& B, double* block) {
  int ca[10][3], cb[10][3];
  const int ni = cart_components(A.l, ca), nj = cart_components(B.l, cb), nb = B.l + 1;
  double sx[16], sy[16], sz[16];
  for (int q = 0; q < ni * nj; q++) block[q] = 0.0;
  for (int p = 0; p < A.np; p++)
    for (int r = 0; r < B.np; r++) {
      const double ai = A.alpha[p], aj = B.alpha[r];
      const double gamma = ai + aj;
      const double mu = ai * aj / gamma;
      const double r2 = dist2_f64(A.center, B.center);
      const double t = std::sqrt(M_PI / gamma);
      const double prefactor = t * t * t * std::exp(-mu * r2);
      double pa[3], pb[3];
      for (int c = 0; c < 3; c++) {
        const double pc = (ai * A.center[c] + aj * B.center[c]) / gamma;
        pa[c] = pc - A.center[c];
        pb[c] = pc - B.center[c];
      }
      os1d_f64(A.l, B.l, pa[0], pb[0], gamma, sx);
      os1d_f64(A.l, B.l, pa[1], pb[1], gamma, sy);
      os1d_f64(A.l, B.l, pa[2], pb[2], gamma, sz);
      for (int x = 0; x < ni; x++)
        for (int y = 0; y < nj; y++) {
          const double val = sx[ca[x][0] * nb + cb[y][0]] * sy[ca[x][1] * nb + cb[y][1]] *
                             sz[ca[x][2] * nb + cb[y][2]] * prefactor * A.coeff[p] * B.coeff[r];
          block[x * nj + y] += val;
        }
    }
}
// integral.rs:286-352
void os_contracted_f128(const ShellRef& A, const ShellRef& B, double* block) {
  int ca[10][3], cb[10][3];
  const int ni = cart_components(A.l, ca), nj = cart_components(B.l, cb), nb = B.l + 1;
  dd sx[16], sy[16], sz[16], b128[100];
  for (int q = 0; q < ni * nj; q++) b128[q] = dd{0, 0};
  for (int p = 0; p < A.np; p++)
    for (int r = 0; r < B.np; r++) {
      const dd ai = dd_from(A.alpha[p]), aj = dd_from(B.alpha[r]);
      const dd gamma = dd_add(ai, aj);
      const dd mu = dd_div(dd_mul(ai, aj), gamma);
      const dd dx = dd_from(A.center[0] - B.center[0]);
      const dd dy = dd_from(A.center[1] - B.center[1]);
      const dd dz = dd_from(A.center[2] - B.center[2]);
      const dd r2 = dd_add(dd_add(dd_mul(dx, dx), dd_mul(dy, dy)), dd_mul(dz, dz));
      const dd ratio = dd_div(dd_from(M_PI), gamma);
      const dd prefactor = dd_mul(ratio, dd_sqrt(ratio));
      const dd neg_mu_r2 = dd_mul(dd_sub(dd{0, 0}, mu), r2);
      const dd exp_hi = dd_from(std::exp(neg_mu_r2.hi));
      const dd exp_val = dd_mul(exp_hi, dd_add(dd_from(1.0), dd_from(neg_mu_r2.lo)));
      const dd total_pre = dd_mul(prefactor, exp_val);
      dd pa[3], pb[3];
      for (int c = 0; c < 3; c++) {
        const dd cic = dd_from(A.center[c]), cjc = dd_from(B.center[c]);
        const dd pc = dd_div(dd_add(dd_mul(ai, cic), dd_mul(aj, cjc)), gamma);
        pa[c] = dd_sub(pc, cic);
        pb[c] = dd_sub(pc, cjc);
      }
      os1d_f128(A.l, B.l, pa[0], pb[0], gamma, sx);
      os1d_f128(A.l, B.l, pa[1], pb[1], gamma, sy);
      os1d_f128(A.l, B.l, pa[2], pb[2], gamma, sz);
      const dd coeff = dd_mul(dd_mul(dd_from(A.coeff[p]), dd_from(B.coeff[r])), total_pre);
      for (int x = 0; x < ni; x++)
        for (int y = 0; y < nj; y++) {
          const dd val = dd_mul(dd_mul(dd_mul(sx[ca[x][0] * nb + cb[y][0]], sy[ca[x][1] * nb + cb[y][1]]),
                                       sz[ca[x][2] * nb + cb[y][2]]),
                                coeff);
          b128[x * nj + y] = dd_add(b128[x * nj + y], val);
        }
    }
  for (int q = 0; q < ni * nj; q++) block[q] = dd_to_f64(b128[q]);
}
// integral.rs:66-138 overlap_shell_pair for tiers 0 (F64) and 1 (F128).
void overlap_shell_pair(const ShellRef& A, const ShellRef& B, int tier, double* block) {
  if (A.l == 0 && B.l == 0) {
    if (tier == 0) {
      double sum = 0.0;
      for (int p = 0; p < A.np; p++)
        for (int r = 0; r < B.np; r++)
          sum += A.coeff[p] * B.coeff[r] * overlap_primitive_f64(A.alpha[p], A.center, B.alpha[r], B.center);
      block[0] = sum;
    } else {
      dd sum{0, 0};
      for (int p = 0; p < A.np; p++)
        for (int r = 0; r < B.np; r++) {
          const dd sp = overlap_primitive_f128(A.alpha[p], A.center, B.alpha[r], B.center);
          sum = dd_add(sum, dd_mul(dd_mul(dd_from(A.coeff[p]), dd_from(B.coeff[r])), sp));
        }
      block[0] = dd_to_f64(sum);
    }
  } else if (tier == 0) {
    os_contracted_f64(A, B, block);
  } else {
    os_contracted_f128(A, B, block);
  }
}
}  // namespace

// assemble_overlap_mixed (assemble.rs:35-85) for shells of any kind
// S, P, D, F (shell_l[s] = 0..3; basis.rs:9-28, n_cart = (l+1)(l+2)/2 AOs in
// cart_components order). matrix: n_ao x n_ao f64.
int or_assemble_overlap(size_t n_shells, const int32_t* shell_l, const double* centers, const int64_t* prim_off,
                        const double* alpha, const double* coeff, const double* params, double* matrix,
                        int64_t* tier_counts) {
  std::vector<size_t> off(n_shells + 1, 0);
  for (size_t s = 0; s < n_shells; s++) {
    if (shell_l[s] < 0 || shell_l[s] > 3) return -1;
    off[s + 1] = off[s] + (size_t)((shell_l[s] + 1) * (shell_l[s] + 2) / 2);
  }
  const size_t n_ao = off[n_shells];
  std::fill(matrix, matrix + n_ao * n_ao, 0.0);
  const size_t npairs = n_shells * (n_shells + 1) / 2;
  std::vector<int> tiers(npairs);
  std::vector<double> blocks(npairs * 100);
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t i = 0; i < n_shells; i++)
    for (size_t j = 0; j <= i; j++) {
      const size_t pidx = i * (i + 1) / 2 + j;
      const ShellRef A{shell_l[i], centers + 3 * i, alpha + prim_off[i], coeff + prim_off[i],
                       (int)(prim_off[i + 1] - prim_off[i])};
      const ShellRef B{shell_l[j], centers + 3 * j, alpha + prim_off[j], coeff + prim_off[j],
                       (int)(prim_off[j + 1] - prim_off[j])};
      const int tier = screen_pair(A.center, A.alpha, A.np, B.center, B.alpha, B.np, params);
      tiers[pidx] = tier;
      if (tier != 2) overlap_shell_pair(A, B, tier, &blocks[pidx * 100]);
    }
  tier_counts[0] = tier_counts[1] = tier_counts[2] = 0;
  for (size_t i = 0; i < n_shells; i++)
    for (size_t j = 0; j <= i; j++) {
      const size_t pidx = i * (i + 1) / 2 + j;
      tier_counts[tiers[pidx]]++;
      if (tiers[pidx] == 2) continue;
      const size_t ni = off[i + 1] - off[i], nj = off[j + 1] - off[j];
      for (size_t a = 0; a < ni; a++)
        for (size_t b = 0; b < nj; b++) {
          const double v = blocks[pidx * 100 + a * nj + b];
          matrix[(off[i] + a) * n_ao + off[j] + b] = v;
          if (i != j) matrix[(off[j] + b) * n_ao + off[i] + a] = v;
        }
    }
  return 0;
}
// The dd problem matrix for the overlap SPD workloads (normalised s
// Gaussians, one primitive per basis function). Full symmetric n x n.
void or_overlap_norm_dd(size_t n, const double* centers, const double* alpha, double* s_out) {
#pragma omp parallel for schedule(dynamic, 8)
  for (size_t i = 0; i < n; i++)
    for (size_t j = 0; j <= i; j++) {
      dd v = overlap_norm_dd(alpha[i], centers + 3 * i, alpha[j], centers + 3 * j);
      st(s_out, i * n + j, v);
      st(s_out, j * n + i, v);
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint of L = b^T S^-1 b for the normalised s-Gaussian overlap matrix
// (test infrastructure for the GPU adjoint).
//   dS_uv/dR_u = -2 p (R_u - R_v) S_uv,  p = a b / (a + b)
//   a dS_uv/da = S_uv [ (3/4)(b - a)/(a + b) - r^2 a b^2 / (a + b)^2 ]
//   dL/dtheta = -lambda^T (dS/dtheta) lambda,  lambda = S^-1 b
// ---------------------------------------------------------------------------
extern "C" {

// "Reference-primitive" gradient: lambda from the reference's f128
// cholesky + solve_cholesky (linalg.rs:42-126) and the contraction in f128
// operations, row by row in index order.
}  // extern "C"

namespace {
// Loss and gradient of L = b^T S^-1 b given lambda = S^-1 b (f128): the
// contraction g = -lambda^T (dS/dtheta) lambda with dS built from f128 ops.
// grad_R: n_centers x 3 f128, grad_lnalpha: n f128.
void adjoint_contract(size_t n, const double* centers, const double* alpha, const std::vector<dd>& S,
                      const std::vector<dd>& bv, const std::vector<dd>& lam, const int32_t* center_of,
                      size_t n_centers, double* loss, double* grad_R, double* grad_lnalpha) {
  dd Lsum{0, 0};
  for (size_t i = 0; i < n; i++) Lsum = dd_add(Lsum, dd_mul(bv[i], lam[i]));
  st(loss, 0, Lsum);
  std::vector<dd> per(3 * n);
#pragma omp parallel for schedule(dynamic, 8)
  for (size_t u = 0; u < n; u++) {
    dd accR[3] = {{0, 0}, {0, 0}, {0, 0}}, acca{0, 0};
    const dd a = dd_from(alpha[u]);
    for (size_t v = 0; v < n; v++) {
      if (v == u) continue;
      const dd bb = dd_from(alpha[v]);
      const dd sum = dd_add(a, bb);
      const dd p = dd_div(dd_mul(a, bb), sum);
      dd d[3], r2{0, 0};
      for (int c = 0; c < 3; c++) {
        d[c] = dd_sub(dd_from(centers[3 * u + c]), dd_from(centers[3 * v + c]));
        r2 = dd_add(r2, dd_mul(d[c], d[c]));
      }
      const dd w = dd_mul(lam[v], S[u * n + v]);
      for (int c = 0; c < 3; c++) accR[c] = dd_add(accR[c], dd_mul(w, dd_mul(p, d[c])));
      const dd f = dd_sub(dd_div(dd_mul(dd_from(0.75), dd_sub(bb, a)), sum),
                          dd_div(dd_mul(r2, dd_mul(a, dd_mul(bb, bb))), dd_mul(sum, sum)));
      acca = dd_add(acca, dd_mul(w, f));
    }
    const dd l4 = dd_mul(dd_from(4.0), lam[u]);
    for (int c = 0; c < 3; c++) per[3 * u + c] = dd_mul(l4, accR[c]);  // per basis function first
    st(grad_lnalpha, u, dd_mul(dd_from(-2.0), dd_mul(lam[u], acca)));
  }
  // sum basis-function contributions per centre (index order)
  std::vector<dd> gR(3 * n_centers, dd{0, 0});
  for (size_t u = 0; u < n; u++)
    for (int c = 0; c < 3; c++) gR[3 * center_of[u] + c] = dd_add(gR[3 * center_of[u] + c], per[3 * u + c]);
  for (size_t c = 0; c < 3 * n_centers; c++) st(grad_R, c, gR[c]);
}

std::vector<dd> overlap_matrix_dd(size_t n, const double* centers, const double* alpha) {
  std::vector<dd> S(n * n);
  for (size_t i = 0; i < n; i++)
    for (size_t j = 0; j <= i; j++) {
      dd v = overlap_norm_dd(alpha[i], centers + 3 * i, alpha[j], centers + 3 * j);
      S[i * n + j] = v;
      S[j * n + i] = v;
    }
  return S;
}
}  // namespace

extern "C" {

// The reference-primitive gradient: lambda from the restated f128 cholesky
// and solve_cholesky (linalg.rs:42-126), then the contraction above.
int or_adjoint_f128(size_t n, const double* centers, const double* alpha, const double* b,
                    const int32_t* center_of, size_t n_centers, double* loss, double* grad_R,
                    double* grad_lnalpha) {
  const std::vector<dd> S = overlap_matrix_dd(n, centers, alpha);
  std::vector<dd> L = S;
  int64_t pv;
  double val;
  if (cholesky_vec(L, n, &pv, &val) != 0) return -2;
  std::vector<dd> bv(n);
  for (size_t i = 0; i < n; i++) bv[i] = dd_from(b[i]);
  const std::vector<dd> lam = backward_solve_v(L, forward_solve_v(L, bv, n), n);
  adjoint_contract(n, centers, alpha, S, bv, lam, center_of, n_centers, loss, grad_R, grad_lnalpha);
  return 0;
}

// The same contraction with a given lambda (n f128), e.g. from the refined
// host solve (or_spd_solve_refined): the host counterpart of the GPU adjoint.
int or_adjoint_f128_lambda(size_t n, const double* centers, const double* alpha, const double* b,
                           const double* lam_in, const int32_t* center_of, size_t n_centers, double* loss,
                           double* grad_R, double* grad_lnalpha) {
  const std::vector<dd> S = overlap_matrix_dd(n, centers, alpha);
  std::vector<dd> bv(n);
  for (size_t i = 0; i < n; i++) bv[i] = dd_from(b[i]);
  adjoint_contract(n, centers, alpha, S, bv, load_vec(lam_in, n), center_of, n_centers, loss, grad_R,
                   grad_lnalpha);
  return 0;
}

}  // extern "C"

namespace {
// One normalised s-Gaussian overlap (the config formula) in MultiFloat<4>:
// (4 a b / (a + b)^2)^{3/4} exp(-a b / (a + b) |Ri - Rj|^2); ci, cj: 3 coordinates.
mf<4> overlap_pair_f256(const mf<4>& a, const mf<4>* ci, const mf<4>& bb, const mf<4>* cj) {
  mf<4> sum = mf_add<4>(a, bb), prod = mf_mul<4>(a, bb);
  mf<4> ratio = mf_div<4>(mf_mul<4>(mf_from<4>(4.0), prod), mf_mul<4>(sum, sum));
  mf<4> sq = mf_sqrt<4>(ratio);
  mf<4> pref = mf_mul<4>(sq, mf_sqrt<4>(sq));
  mf<4> mu = mf_div<4>(prod, sum);
  mf<4> r2 = mf_zero<4>();
  for (int c = 0; c < 3; c++) {
    mf<4> d = mf_sub<4>(ci[c], cj[c]);
    r2 = mf_add<4>(r2, mf_mul<4>(d, d));
  }
  return mf_mul<4>(pref, mf_exp<4>(mf_neg<4>(mf_mul<4>(mu, r2))));
}

// L y = v for a row-major n x n lower factor in MultiFloat<4> (the forward
// sweep of mf_cholesky_solve, multifloat/linalg.rs:145-160).
void mf4_forward(const std::vector<mf<4>>& L, size_t n, std::vector<mf<4>>& v) {
  for (size_t i = 0; i < n; i++) {
    for (size_t j = 0; j < i; j++) v[i] = mf_sub<4>(v[i], mf_mul<4>(L[i * n + j], v[j]));
    v[i] = mf_div<4>(v[i], L[i * n + i]);
  }
}
}  // namespace

extern "C" {

// L = b^T S^-1 b in MultiFloat<4> with S from f256 centres / exponents
// (for central finite differences): centers4 n x 3 x 4, alpha4 n x 4.
int or_loss_f256(size_t n, const double* centers4, const double* alpha4, const double* b, double* loss4) {
  std::vector<mf<4>> S(n * n);
  auto ldq = [&](const double* p) { return ldm<4>(p, 0); };
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t i = 0; i < n; i++)
    for (size_t j = 0; j <= i; j++) {
      mf<4> ci[3], cj[3];
      for (int c = 0; c < 3; c++) ci[c] = ldq(centers4 + 12 * i + 4 * c), cj[c] = ldq(centers4 + 12 * j + 4 * c);
      mf<4> v = overlap_pair_f256(ldq(alpha4 + 4 * i), ci, ldq(alpha4 + 4 * j), cj);
      S[i * n + j] = v;
      S[j * n + i] = v;
    }
  std::vector<double> Sp(n * n * 4), bq(n * 4, 0.0), x(n * 4);
  for (size_t i = 0; i < n * n; i++) stm<4>(Sp.data(), i, S[i]);
  for (size_t i = 0; i < n; i++) bq[4 * i] = b[i];
  if (mf_cholesky_t<4>(Sp.data(), n) != 0) return -2;
  mf_cholesky_solve_t<4>(Sp.data(), bq.data(), x.data(), n);
  mf<4> Ls = mf_zero<4>();
  for (size_t i = 0; i < n; i++) Ls = mf_add<4>(Ls, mf_mul<4>(mf_from<4>(b[i]), ldm<4>(x.data(), i)));
  stm<4>(loss4, 0, Ls);
  return 0;
}

// Central finite differences in MultiFloat<4> (step h) of L = b^T S^-1 b with
// respect to the three coordinates of each centre in cen_list and the
// log-exponent of each basis function on those centres (test infrastructure
// for the adjoint at sizes where one f256 solve per perturbation is too slow).
// The basis functions P of those centres are ordered last; the rest, S11,
// depends on none of the perturbed parameters and is factored once by the
// restated mf_cholesky<4> (multifloat/linalg.rs:89-141). Each perturbed loss
// is the block elimination of the symmetrically permuted system (the same
// value b^T S^-1 b):
//   L = z.z + y^T T^-1 y,  z = L11^-1 b1,  W = L11^-1 S12,
//   T = S22 - W^T W,  y = b2 - W^T z,
// where only the columns of W of the perturbed functions are recomputed.
// A centre coordinate moves by +-h (an exact second limb); an exponent is
// multiplied by (1 +- h) in f256 (d/d ln alpha to O(h^2)).
// gR: n_cen x 3 f256 in cen_list order; ga: |P| f256 in increasing function
// index. Returns -2 if a factorisation fails.
int or_fd_grad_f256(size_t n, const double* centers, const double* alpha, const double* b,
                    const int32_t* center_of, const int32_t* cen_list, size_t n_cen, double h, double* gR,
                    double* ga) {
  std::vector<size_t> P, R;
  std::vector<int> pos_in_list(n, -1);
  for (size_t u = 0; u < n; u++) {
    int li = -1;
    for (size_t c = 0; c < n_cen; c++)
      if (center_of[u] == cen_list[c]) li = (int)c;
    pos_in_list[u] = li;
    (li >= 0 ? P : R).push_back(u);
  }
  const size_t m = R.size(), p = P.size();
  std::vector<mf<4>> a4(n), c4(3 * n);
  for (size_t u = 0; u < n; u++) {
    a4[u] = mf_from<4>(alpha[u]);
    for (int c = 0; c < 3; c++) c4[3 * u + c] = mf_from<4>(centers[3 * u + c]);
  }
  // S11 and its factor
  std::vector<double> Sp(m * m * 4);
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t i = 0; i < m; i++)
    for (size_t j = 0; j <= i; j++) {
      mf<4> v = overlap_pair_f256(a4[R[i]], &c4[3 * R[i]], a4[R[j]], &c4[3 * R[j]]);
      stm<4>(Sp.data(), i * m + j, v);
      stm<4>(Sp.data(), j * m + i, v);
    }
  if (mf_cholesky_t<4>(Sp.data(), m) != 0) return -2;
  std::vector<mf<4>> L11(m * m);
  for (size_t i = 0; i < m * m; i++) L11[i] = ldm<4>(Sp.data(), i);
  std::vector<mf<4>> z(m);
  for (size_t i = 0; i < m; i++) z[i] = mf_from<4>(b[R[i]]);
  mf4_forward(L11, m, z);
  mf<4> zz = mf_zero<4>();
  for (size_t i = 0; i < m; i++) zz = mf_add<4>(zz, mf_mul<4>(z[i], z[i]));
  // the unperturbed columns of W = L11^-1 S12
  std::vector<std::vector<mf<4>>> W0(p, std::vector<mf<4>>(m));
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t q = 0; q < p; q++) {
    for (size_t i = 0; i < m; i++) W0[q][i] = overlap_pair_f256(a4[R[i]], &c4[3 * R[i]], a4[P[q]], &c4[3 * P[q]]);
    mf4_forward(L11, m, W0[q]);
  }
  // perturbations: (kind 0: coordinate c of centre cen_list[ci]; kind 1: exponent of P[q]) x (+h, -h)
  struct Pert {
    int kind, idx, comp;
  };
  std::vector<Pert> perts;
  for (size_t ci = 0; ci < n_cen; ci++)
    for (int c = 0; c < 3; c++) perts.push_back({0, (int)ci, c});
  for (size_t q = 0; q < p; q++) perts.push_back({1, (int)q, 0});
  std::vector<mf<4>> loss(2 * perts.size());
  int fail = 0;
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t t = 0; t < 2 * perts.size(); t++) {
    const Pert& pt = perts[t / 2];
    const double sg = (t % 2 == 0) ? 1.0 : -1.0;
    std::vector<mf<4>> ap(p), cp(3 * p);
    std::vector<char> moved(p, 0);
    for (size_t q = 0; q < p; q++) {
      ap[q] = a4[P[q]];
      for (int c = 0; c < 3; c++) cp[3 * q + c] = c4[3 * P[q] + c];
      if (pt.kind == 0 && pos_in_list[P[q]] == pt.idx) {
        mf<4> d = mf_zero<4>();
        d.l[0] = sg * h;
        cp[3 * q + pt.comp] = mf_add<4>(cp[3 * q + pt.comp], d);
        moved[q] = 1;
      }
      if (pt.kind == 1 && (int)q == pt.idx) {
        mf<4> f = mf_from<4>(1.0);
        f = mf_add<4>(f, mf_from<4>(sg * h));
        ap[q] = mf_mul<4>(ap[q], f);
        moved[q] = 1;
      }
    }
    std::vector<std::vector<mf<4>>> Wc;  // recomputed columns, others from W0
    std::vector<const std::vector<mf<4>>*> W(p);
    Wc.reserve(p);
    for (size_t q = 0; q < p; q++) {
      if (!moved[q]) {
        W[q] = &W0[q];
        continue;
      }
      Wc.emplace_back(m);
      std::vector<mf<4>>& col = Wc.back();
      for (size_t i = 0; i < m; i++) col[i] = overlap_pair_f256(a4[R[i]], &c4[3 * R[i]], ap[q], &cp[3 * q]);
      mf4_forward(L11, m, col);
      W[q] = &col;
    }
    // T = S22 - W^T W (lower triangle), y = b2 - W^T z
    std::vector<double> T(p * p * 4), y(p * 4, 0.0), xs(p * 4);
    for (size_t q = 0; q < p; q++) {
      mf<4> yq = mf_from<4>(b[P[q]]);
      for (size_t i = 0; i < m; i++) yq = mf_sub<4>(yq, mf_mul<4>((*W[q])[i], z[i]));
      stm<4>(y.data(), q, yq);
      for (size_t r = 0; r <= q; r++) {
        mf<4> v = overlap_pair_f256(ap[q], &cp[3 * q], ap[r], &cp[3 * r]);
        for (size_t i = 0; i < m; i++) v = mf_sub<4>(v, mf_mul<4>((*W[q])[i], (*W[r])[i]));
        stm<4>(T.data(), q * p + r, v);
        stm<4>(T.data(), r * p + q, v);
      }
    }
    if (mf_cholesky_t<4>(T.data(), p) != 0) {
#pragma omp atomic write
      fail = 1;
      continue;
    }
    mf_cholesky_solve_t<4>(T.data(), y.data(), xs.data(), p);
    mf<4> Ls = zz;
    for (size_t q = 0; q < p; q++) Ls = mf_add<4>(Ls, mf_mul<4>(ldm<4>(y.data(), q), ldm<4>(xs.data(), q)));
    loss[t] = Ls;
  }
  if (fail) return -2;
  const mf<4> inv2h = mf_recip<4>(mf_from<4>(2.0 * h));
  for (size_t k = 0; k < perts.size(); k++) {
    mf<4> g = mf_mul<4>(mf_sub<4>(loss[2 * k], loss[2 * k + 1]), inv2h);
    if (perts[k].kind == 0)
      stm<4>(gR, 3 * perts[k].idx + perts[k].comp, g);
    else
      stm<4>(ga, perts[k].idx, g);
  }
  return 0;
}

}  // extern "C"
