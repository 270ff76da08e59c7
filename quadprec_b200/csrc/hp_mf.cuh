// MultiFloat<N> device arithmetic for any N (used for N = 8, the f512 of
// hyperprec: crates/quad/src/multifloat/{core,add,mul,div,math}.rs). The
// N = 4 kernels keep the hand-specialised qd_* of hp_arith.cuh; these
// templates follow the same rewrites, generalised:
//   * renormalize (core.rs:58-93) and renormalize_from (core.rs:100-168) use
//     the static-index sweep / compaction of hp_arith.cuh;
//   * add (add.rs:23-105): the stable insertion sort by |x| descending is a
//     Batcher odd-even merge sorting network over the key (|x| descending,
//     original index ascending), a total order whose sorted sequence is the
//     stable insertion sort's; the grow-expansion walks all 2N slots (the
//     slots past the live length hold zeros, and two_sum(0, c) = (c, 0));
//   * mul (mul.rs:16-110): the convolution over i + j < N in the reference's
//     (i, j) order with the cascaded accumulate of mul.rs:31-42 unrolled
//     (later slots are written only while the cascade is live);
//   * recip (div.rs:14-41, ceil(log2 N) + 2 Newton steps), div (div.rs:52-76),
//     sqrt (math.rs:22-40, ceil(log2 N) + 1 Heron steps).
// Every operation is an explicit round-to-nearest intrinsic, so the results
// are the reference's bits.
#pragma once
#include "hp_arith.cuh"

namespace hp {

template <int N>
struct mfn {
  double l[N];
};

template <int N>
__device__ __forceinline__ mfn<N> mfn_zero() {
  mfn<N> r;
#pragma unroll
  for (int i = 0; i < N; i++) r.l[i] = 0.0;
  return r;
}
template <int N>
__device__ __forceinline__ mfn<N> mfn_from(double x) {  // core.rs:185-189
  mfn<N> r = mfn_zero<N>();
  r.l[0] = x;
  return r;
}
template <int N>
__device__ __forceinline__ mfn<N> mfn_neg(const mfn<N>& a) {  // add.rs:4-17
  mfn<N> r;
#pragma unroll
  for (int i = 0; i < N; i++) r.l[i] = -a.l[i];
  return r;
}

// core.rs:58-93
template <int N>
__device__ __forceinline__ void mfn_renormalize(double* l) {
#pragma unroll
  for (int pass = 0; pass < 2; pass++) {
    sweep_bottom_up<N>(l);
    double out[N];
    compact_top_down<N, N>(l, out);
#pragma unroll
    for (int i = 0; i < N; i++) l[i] = out[i];
  }
}
// core.rs:100-168 (M inputs, N outputs)
template <int N, int M>
__device__ __forceinline__ void mfn_renormalize_from(const double* in, double* out) {
  double t[M];
#pragma unroll
  for (int i = 0; i < M; i++) t[i] = in[i];
  sweep_bottom_up<M>(t);
  double buf[M];
  compact_top_down<M, M>(t, buf);
  sweep_bottom_up<M>(buf);
  compact_top_down<M, N>(buf, out);
}

// Batcher odd-even merge sort of K (a power of two) keys by (|w| descending,
// id ascending); cmp_swap (hp_arith.cuh) orders one pair by that key.
template <int K>
__device__ __forceinline__ void sort_by_magnitude(double* w, int* id) {
#pragma unroll
  for (int p = 1; p < K; p <<= 1)
#pragma unroll
    for (int k = p; k >= 1; k >>= 1)
#pragma unroll
      for (int j = k % p; j + k < K; j += 2 * k)
#pragma unroll
        for (int i = 0; i < k; i++)
          if (i + j + k < K && (i + j) / (2 * p) == (i + j + k) / (2 * p))
            cmp_swap(w[i + j], id[i + j], w[i + j + k], id[i + j + k]);
}

// add.rs:23-105
template <int N>
__device__ __forceinline__ mfn<N> mfn_add(const mfn<N>& a, const mfn<N>& b) {
  constexpr int W = 2 * N;
  double w[W];
  int id[W];
#pragma unroll
  for (int i = 0; i < N; i++) {
    two_sum(a.l[i], b.l[i], w[2 * i], w[2 * i + 1]);
    id[2 * i] = 2 * i;
    id[2 * i + 1] = 2 * i + 1;
  }
  sort_by_magnitude<W>(w, id);
  double ex[W];
#pragma unroll
  for (int i = 0; i < W; i++) ex[i] = 0.0;
  int exp_len = 0;
#pragma unroll
  for (int i = 0; i < W; i++) {
    const double term = w[i];
    if (term != 0.0) {
      if (exp_len == 0) {
        ex[0] = term;
        exp_len = 1;
      } else {
        double carry = term;
#pragma unroll
        for (int j = W - 1; j >= 0; j--) {
          double s, e;
          two_sum(ex[j], carry, s, e);
          ex[j] = e;
          carry = s;
        }
        if (carry != 0.0) {
#pragma unroll
          for (int k = W - 1; k > 0; k--) ex[k] = ex[k - 1];
          ex[0] = carry;
          exp_len++;
        }
      }
    }
  }
  mfn<N> r;
#pragma unroll
  for (int i = 0; i < N; i++) r.l[i] = ex[i];  // slots >= exp_len are zero
  mfn_renormalize<N>(r.l);
  return r;
}
template <int N>
__device__ __forceinline__ mfn<N> mfn_sub(const mfn<N>& a, const mfn<N>& b) {  // add.rs:108-113
  return mfn_add<N>(a, mfn_neg<N>(b));
}

// mul.rs:31-42 accumulate(work, IDX, val, LIMIT)
template <int IDX, int LIMIT>
__device__ __forceinline__ void mfn_accumulate(double* work, double val) {
  double s, e;
  two_sum(work[IDX], val, s, e);
  work[IDX] = s;
  bool live = true;
#pragma unroll
  for (int k = IDX + 1; k < LIMIT; k++) {
    live = live && (e != 0.0);
    double s2, e2;
    two_sum(work[k], e, s2, e2);
    if (live) {
      work[k] = s2;
      e = e2;
    }
  }
}
template <int N, int I, int J>
__device__ __forceinline__ void mfn_mul_term(const mfn<N>& a, const mfn<N>& b, double* work) {
  if constexpr (I < N && J < N && I + J < N) {
    double p, e;
    two_prod(a.l[I], b.l[J], p, e);
    mfn_accumulate<I + J, 2 * N>(work, p);
    mfn_accumulate<I + J + 1, 2 * N>(work, e);
  }
}
template <int N, int I>
__device__ __forceinline__ void mfn_mul_row(const mfn<N>& a, const mfn<N>& b, double* work) {
  mfn_mul_term<N, I, 0>(a, b, work);
  mfn_mul_term<N, I, 1>(a, b, work);
  mfn_mul_term<N, I, 2>(a, b, work);
  mfn_mul_term<N, I, 3>(a, b, work);
  mfn_mul_term<N, I, 4>(a, b, work);
  mfn_mul_term<N, I, 5>(a, b, work);
  mfn_mul_term<N, I, 6>(a, b, work);
  mfn_mul_term<N, I, 7>(a, b, work);
}
// mul.rs:16-110 (N <= 8)
template <int N>
__device__ __forceinline__ mfn<N> mfn_mul(const mfn<N>& a, const mfn<N>& b) {
  static_assert(N <= 8, "convolution unrolled for up to 8 limbs");
  double work[2 * N];
#pragma unroll
  for (int i = 0; i < 2 * N; i++) work[i] = 0.0;
  mfn_mul_row<N, 0>(a, b, work);
  mfn_mul_row<N, 1>(a, b, work);
  mfn_mul_row<N, 2>(a, b, work);
  mfn_mul_row<N, 3>(a, b, work);
  mfn_mul_row<N, 4>(a, b, work);
  mfn_mul_row<N, 5>(a, b, work);
  mfn_mul_row<N, 6>(a, b, work);
  mfn_mul_row<N, 7>(a, b, work);
  mfn<N> r;
  mfn_renormalize_from<N, 2 * N>(work, r.l);
  return r;
}

// ceil(log2 n) at compile time
template <int n>
struct CeilLog2 {
  static constexpr int value = 1 + CeilLog2<(n + 1) / 2>::value;
};
template <>
struct CeilLog2<1> {
  static constexpr int value = 0;
};

// div.rs:14-41
template <int N>
__device__ __forceinline__ mfn<N> mfn_recip(const mfn<N>& a) {
  if (a.l[0] == 0.0) return mfn_from<N>(signbit(a.l[0]) ? -INFINITY : INFINITY);
  if (!isfinite(a.l[0])) return mfn_from<N>(0.0);
  mfn<N> x = mfn_from<N>(DIV(1.0, a.l[0]));
  const mfn<N> one = mfn_from<N>(1.0);
  constexpr int steps = N <= 1 ? 1 : CeilLog2<N>::value + 2;
  for (int s = 0; s < steps; s++) {
    const mfn<N> residual = mfn_sub<N>(one, mfn_mul<N>(a, x));
    x = mfn_add<N>(x, mfn_mul<N>(x, residual));
  }
  return x;
}
// div.rs:52-76
template <int N>
__device__ __forceinline__ mfn<N> mfn_div(const mfn<N>& a, const mfn<N>& b) {
  if (b.l[0] == 0.0) {
    const double sign = (signbit(a.l[0]) == signbit(b.l[0])) ? 1.0 : -1.0;
    return mfn_from<N>(a.l[0] == 0.0 ? __longlong_as_double(0x7ff8000000000000ll) : sign * INFINITY);
  }
  if (a.l[0] == 0.0) return mfn_zero<N>();
  if (!isfinite(a.l[0]) || !isfinite(b.l[0])) return mfn_from<N>(DIV(a.l[0], b.l[0]));
  return mfn_mul<N>(a, mfn_recip<N>(b));
}
// math.rs:22-40
template <int N>
__device__ __forceinline__ mfn<N> mfn_sqrt(const mfn<N>& a) {
  if (a.l[0] < 0.0) return mfn_from<N>(__longlong_as_double(0x7ff8000000000000ll));
  if (a.l[0] == 0.0) return mfn_zero<N>();
  if (!isfinite(a.l[0])) return mfn_from<N>(a.l[0]);
  mfn<N> x = mfn_from<N>(__dsqrt_rn(a.l[0]));
  const mfn<N> half = mfn_from<N>(0.5);
  constexpr int steps = CeilLog2<N>::value + 1;
  for (int s = 0; s < steps; s++) x = mfn_mul<N>(mfn_add<N>(x, mfn_div<N>(a, x)), half);
  return x;
}

}  // namespace hp
