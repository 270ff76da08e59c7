// Text exchange of f128 and MultiFloat<N> values in the reference's serde
// formats (host code; no device work):
//   f128           crates/quad/src/dd.rs:441-514: human-readable form
//                  format!("{:+.18e}+{:+.18e}", hi, lo), parsed back by
//                  parse_dd_string (the first '+' that is followed by a
//                  sign and not preceded by 'e' / 'E' splits hi from lo);
//   MultiFloat<N>  crates/quad/src/multifloat/traits.rs:7-155: the limbs as
//                  "{:+.14e}" joined by '+', parsed back by
//                  parse_limbs_string (the same boundary rule, exactly N
//                  limbs).
// The compact (non-human-readable) forms are the structs {hi, lo} and
// {limbs: [..]} of f64 fields: the same bytes as this library's in-memory
// layout, so binary exchange needs no conversion.
//
// Rust's {:e} writes the exponent without a '+' and without leading zeros
// ("e-5", "e0") and a NaN as "NaN"; printf's %e ("e-05", "e+00", "nan") is
// rewritten accordingly. Both produce the correctly rounded decimal digits.
// Parsing accepts what Rust's f64::from_str accepts for these strings: an
// optional sign, decimal digits with an optional point and exponent, or
// inf / infinity / nan (any case); anything else (hex floats, blanks,
// trailing characters) is an error, as in Rust.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "hp_runtime.cuh"

namespace hp {
namespace {

// One f64 as Rust's format!("{:+.<prec>e}", x).
std::string rust_exp(double x, int prec) {
  if (std::isnan(x)) return "NaN";
  if (std::isinf(x)) return x > 0 ? "+inf" : "-inf";
  char buf[64];
  std::snprintf(buf, sizeof buf, "%+.*e", prec, x);
  std::string s(buf);
  const size_t e = s.find('e');
  if (e == std::string::npos) return s;
  std::string mant = s.substr(0, e), ex = s.substr(e + 1);
  bool neg = false;
  size_t p = 0;
  if (p < ex.size() && (ex[p] == '+' || ex[p] == '-')) neg = ex[p++] == '-';
  while (p + 1 < ex.size() && ex[p] == '0') p++;
  return mant + "e" + (neg ? "-" : "") + ex.substr(p);
}

// Rust f64::from_str on [b, e): false on a string Rust rejects.
bool rust_parse(const char* b, const char* e, double* out) {
  if (b == e) return false;
  std::string t(b, e);
  const char* c = t.c_str();
  size_t i = 0;
  if (c[i] == '+' || c[i] == '-') i++;
  std::string rest = t.substr(i);
  std::string low;
  for (char ch : rest) low += (char)std::tolower((unsigned char)ch);
  if (low == "inf" || low == "infinity") {
    *out = t[0] == '-' ? -INFINITY : INFINITY;
    return true;
  }
  if (low == "nan") {
    *out = NAN;
    return true;
  }
  size_t digits = 0, k = i;
  while (std::isdigit((unsigned char)c[k])) k++, digits++;
  if (c[k] == '.') {
    k++;
    while (std::isdigit((unsigned char)c[k])) k++, digits++;
  }
  if (digits == 0) return false;
  if (c[k] == 'e' || c[k] == 'E') {
    k++;
    if (c[k] == '+' || c[k] == '-') k++;
    size_t ed = 0;
    while (std::isdigit((unsigned char)c[k])) k++, ed++;
    if (ed == 0) return false;
  }
  if (c[k] != '\0') return false;
  errno = 0;
  char* end = nullptr;
  const double v = std::strtod(c, &end);
  if (end != c + t.size()) return false;
  *out = v;  // overflow gives +-inf and underflow 0 or a subnormal, as in Rust
  return true;
}

// Positions of the separators: '+' at i >= 1 followed by '+' or '-' and not
// preceded by 'e' / 'E'.
bool is_boundary(const char* s, size_t len, size_t i) {
  return s[i] == '+' && i + 1 < len && (s[i + 1] == '+' || s[i + 1] == '-') && s[i - 1] != 'e' && s[i - 1] != 'E';
}

int copy_out(const std::string& s, char* out, size_t cap) {
  if (!out || cap < s.size() + 1) {
    set_error("output buffer needs %zu bytes", s.size() + 1);
    return HP_ERR_INVALID_ARG;
  }
  std::memcpy(out, s.c_str(), s.size() + 1);
  return HP_OK;
}

}  // namespace
}  // namespace hp

extern "C" {

int hp_f128_to_string(const double* v, char* out, size_t cap) {
  if (!v) return HP_ERR_INVALID_ARG;
  return hp::copy_out(hp::rust_exp(v[0], 18) + "+" + hp::rust_exp(v[1], 18), out, cap);
}

int hp_f128_from_string(const char* s, double* out) {
  if (!s || !out) return HP_ERR_INVALID_ARG;
  const size_t len = std::strlen(s);
  for (size_t i = 1; i + 1 < len; i++) {
    if (s[i] == '+' && (s[i + 1] == '+' || s[i + 1] == '-')) {
      if (s[i - 1] == 'e' || s[i - 1] == 'E') continue;
      double hi, lo;
      if (!hp::rust_parse(s, s + i, &hi) || !hp::rust_parse(s + i + 1, s + len, &lo)) break;
      out[0] = hi;  // f128::new(hi, lo): the limbs as given
      out[1] = lo;
      return HP_OK;
    }
  }
  hp::set_error("not an f128 string \"<hi>+<lo>\": %.64s", s);
  return HP_ERR_INVALID_ARG;
}

int hp_mf_to_string(int n_limbs, const double* v, char* out, size_t cap) {
  if (!v || n_limbs < 1) return HP_ERR_INVALID_ARG;
  std::string s;
  for (int i = 0; i < n_limbs; i++) {
    if (i > 0) s += '+';
    s += hp::rust_exp(v[i], 14);
  }
  return hp::copy_out(s, out, cap);
}

int hp_mf_from_string(int n_limbs, const char* s, double* out) {
  if (!s || !out || n_limbs < 1) return HP_ERR_INVALID_ARG;
  const size_t len = std::strlen(s);
  int count = 0;
  size_t start = 0;
  bool ok = true;
  for (size_t i = 1; i < len && ok;) {
    if (hp::is_boundary(s, len, i)) {
      if (count >= n_limbs || !hp::rust_parse(s + start, s + i, &out[count])) ok = false;
      count++;
      start = i + 1;
      i = start + 1;
    } else {
      i++;
    }
  }
  if (ok) {
    if (count >= n_limbs || !hp::rust_parse(s + start, s + len, &out[count])) ok = false;
    count++;
  }
  if (!ok || count != n_limbs) {
    hp::set_error("not a string of %d limbs separated by '+': %.64s", n_limbs, s);
    return HP_ERR_INVALID_ARG;
  }
  return HP_OK;
}

}  // extern "C"
