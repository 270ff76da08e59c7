// Host build of quadprec_b200/csrc/hp_arith.cuh for the CPU test suite.
// The device intrinsics are replaced by their IEEE host equivalents (each is
// one correctly rounded operation), so the header's operation sequences can
// be compared bit-for-bit against the oracle without a GPU.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <math.h>

#define __device__
#define __forceinline__ inline
static inline double __dadd_rn(double a, double b) { return a + b; }
static inline double __dsub_rn(double a, double b) { return a - b; }
static inline double __dmul_rn(double a, double b) { return a * b; }
static inline double __ddiv_rn(double a, double b) { return a / b; }
static inline double __fma_rn(double a, double b, double c) { return std::fma(a, b, c); }
static inline double __drcp_rn(double a) { return 1.0 / a; }
static inline double __dsqrt_rn(double a) { return std::sqrt(a); }
// seed of the chosen-path 1/sqrt helper (not compared bit-for-bit here)
static inline double rsqrt(double a) { return 1.0 / std::sqrt(a); }
static inline double __longlong_as_double(long long v) {
  double d;
  std::memcpy(&d, &v, 8);
  return d;
}
using std::fabs;
using std::isfinite;
using std::round;
using std::signbit;

#include "../quadprec_b200/csrc/hp_arith.cuh"
#include "../quadprec_b200/csrc/hp_mf.cuh"

using namespace hp;
extern "C" {
void sh_dd_add(const double* a, const double* b, double* o) {
  dd r = dd_add(dd{a[0], a[1]}, dd{b[0], b[1]});
  o[0] = r.hi, o[1] = r.lo;
}
void sh_dd_mul(const double* a, const double* b, double* o) {
  dd r = dd_mul(dd{a[0], a[1]}, dd{b[0], b[1]});
  o[0] = r.hi, o[1] = r.lo;
}
void sh_dd_div(const double* a, const double* b, double* o) {
  dd r = dd_div(dd{a[0], a[1]}, dd{b[0], b[1]});
  o[0] = r.hi, o[1] = r.lo;
}
void sh_dd_sqrt(const double* a, double* o) {
  dd r = dd_sqrt(dd{a[0], a[1]});
  o[0] = r.hi, o[1] = r.lo;
}
void sh_dd_recip(const double* a, double* o) {
  dd r = dd_recip(dd{a[0], a[1]});
  o[0] = r.hi, o[1] = r.lo;
}
void sh_dd_exp(const double* a, double* o) {
  dd r = dd_exp(dd{a[0], a[1]});
  o[0] = r.hi, o[1] = r.lo;
}
static qd ldq(const double* p) { return qd{{p[0], p[1], p[2], p[3]}}; }
static void stq(double* p, const qd& v) {
  for (int i = 0; i < 4; i++) p[i] = v.l[i];
}
void sh_qd_add(const double* a, const double* b, double* o) { stq(o, qd_add(ldq(a), ldq(b))); }
void sh_qd_mul(const double* a, const double* b, double* o) { stq(o, qd_mul(ldq(a), ldq(b))); }
void sh_qd_div(const double* a, const double* b, double* o) { stq(o, qd_div(ldq(a), ldq(b))); }
void sh_qd_sqrt(const double* a, double* o) { stq(o, qd_sqrt(ldq(a))); }
// div_small_int (the Taylor divisions of dd_exp) against IEEE x / i for
// i = 1..max_divisor, per_divisor random x each (random sign, mantissa and
// exponent in [-1000, 1000], a quarter next to exact multiples of i and a
// quarter on halfway points); returns the number of differing bit patterns.
long sh_div_small_mismatches(long per_divisor, int max_divisor, unsigned long long seed) {
  auto next = [&seed]() {  // SplitMix64
    uint64_t z = (seed += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  };
  long bad = 0;
  for (int i = 1; i <= max_divisor; i++) {
    const double b = (double)i, y = 1.0 / b;
    for (long t = 0; t < per_divisor; t++) {
      const uint64_t bits = next();
      const double m = 1.0 + (double)(bits >> 12) * 0x1p-52;
      double x = std::ldexp(m, (int)(next() % 2001) - 1000) * ((bits & 1) ? -1.0 : 1.0);
      if (t % 4 == 1) {
        x = std::ldexp(1.0 + (double)(next() >> 12) * 0x1p-52, (int)(next() % 200) - 100) * b;
        x = std::nextafter(x, (t & 2) ? INFINITY : -INFINITY);
      } else if (t % 4 == 2) {
        x = (std::floor(std::ldexp(1.0 + (double)(next() >> 12) * 0x1p-52, (int)(next() % 60))) + 0.5) * b;
      }
      const double got = div_small_int(x, b, y), want = x / b;
      if (std::memcmp(&got, &want, 8) != 0) bad++;
    }
  }
  return bad;
}
// dd_dot2_fast (the fused rotation of the batched Jacobi): o = c a + s b
// for count f128 entries of each operand.
void sh_dd_dot2(const double* c, const double* a, const double* s, const double* b, double* o, long count) {
  for (long i = 0; i < count; i++) {
    const dd r = dd_dot2_fast(dd{c[2 * i], c[2 * i + 1]}, dd{a[2 * i], a[2 * i + 1]}, dd{s[2 * i], s[2 * i + 1]},
                              dd{b[2 * i], b[2 * i + 1]});
    o[2 * i] = r.hi;
    o[2 * i + 1] = r.lo;
  }
}
}  // extern "C"
// The generic MultiFloat<N> templates (hp_mf.cuh) for N = 4 and 8.
template <int N>
static mfn<N> ldn(const double* p) {
  mfn<N> r;
  for (int i = 0; i < N; i++) r.l[i] = p[i];
  return r;
}
template <int N>
static void stn(double* p, const mfn<N>& v) {
  for (int i = 0; i < N; i++) p[i] = v.l[i];
}
template <int N>
static void mfn_op(int which, const double* a, const double* b, double* o) {
  switch (which) {
    case 0: stn<N>(o, mfn_add<N>(ldn<N>(a), ldn<N>(b))); break;
    case 1: stn<N>(o, mfn_mul<N>(ldn<N>(a), ldn<N>(b))); break;
    case 2: stn<N>(o, mfn_div<N>(ldn<N>(a), ldn<N>(b))); break;
    case 3: stn<N>(o, mfn_sqrt<N>(ldn<N>(a))); break;
  }
}
extern "C" {
// ops 20-23: MultiFloat<8>, 30-33: MultiFloat<4> through the templates.
void sh_mfn_batch(int op, const double* a, const double* b, double* o, long count) {
  const int N = op >= 30 ? 4 : 8;
  for (long i = 0; i < count; i++) {
    if (N == 8)
      mfn_op<8>(op - 20, a + 8 * i, b + 8 * i, o + 8 * i);
    else
      mfn_op<4>(op - 30, a + 4 * i, b + 4 * i, o + 4 * i);
  }
}
// Many ops at once (count entries of 2 or 4 limbs each).
void sh_batch(int op, const double* a, const double* b, double* o, long count) {
  for (long i = 0; i < count; i++) {
    switch (op) {
      case 0: sh_dd_add(a + 2 * i, b + 2 * i, o + 2 * i); break;
      case 1: sh_dd_mul(a + 2 * i, b + 2 * i, o + 2 * i); break;
      case 2: sh_dd_div(a + 2 * i, b + 2 * i, o + 2 * i); break;
      case 3: sh_dd_sqrt(a + 2 * i, o + 2 * i); break;
      case 4: sh_dd_recip(a + 2 * i, o + 2 * i); break;
      case 5: sh_dd_exp(a + 2 * i, o + 2 * i); break;
      case 6: {  // chosen-path reciprocal (error bound checked, not bits)
        const dd r = dd_recip_fast(dd{a[2 * i], a[2 * i + 1]});
        o[2 * i] = r.hi;
        o[2 * i + 1] = r.lo;
        break;
      }
      case 10: sh_qd_add(a + 4 * i, b + 4 * i, o + 4 * i); break;
      case 11: sh_qd_mul(a + 4 * i, b + 4 * i, o + 4 * i); break;
      case 12: sh_qd_div(a + 4 * i, b + 4 * i, o + 4 * i); break;
      case 13: sh_qd_sqrt(a + 4 * i, o + 4 * i); break;
    }
  }
}
}
