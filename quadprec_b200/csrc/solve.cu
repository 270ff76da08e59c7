// Triangular solves, matvec, norms and small vector kernels for the f128
// solver path (crates/quad/src/linalg.rs:99-147, 185-194 and
// crates/solver/src/lib.rs:198-249).
//
// forward solve (linalg.rs:99-108): y_i is updated by y_i - L_ij y_j for
// j = 0..i-1 in order, then divided by L_ii. The kernel runs it
// right-looking (after y_j is final, every y_i with i > j takes its update),
// which applies each row's updates in the same order: bit-identical.
// backward solve (linalg.rs:111-120) accumulates x_i over j = i+1..n-1 in
// ascending order, but x_j becomes available in descending order, so a
// bit-identical version is a single sequential chain of n^2/2 dependent
// f128 adds. The kernel applies the updates right-looking instead
// (descending j): same operations, another order, normwise error of the
// same bound.
// matvec (linalg.rs:129-147) keeps the reference's sequential row sums
// (bit-identical); rows run in parallel and stream through shared memory.
#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {

struct VOpsF64 {
  using T = double;
  __device__ static T zero() { return 0.0; }
  __device__ static T sub(T a, T b) { return __dsub_rn(a, b); }
  __device__ static T mul(T a, T b) { return __dmul_rn(a, b); }
  __device__ static T div(T a, T b) { return __ddiv_rn(a, b); }
};
struct VOpsDD {
  using T = dd;
  __device__ static T zero() { return dd{0.0, 0.0}; }
  __device__ static T sub(T a, T b) { return dd_sub(a, b); }
  __device__ static T mul(T a, T b) { return dd_mul(a, b); }
  __device__ static T div(T a, T b) { return dd_div(a, b); }
};

namespace {

// One CTA of TH threads; thread t owns rows t, t + TH, ... (RMAX of them).
// The entries of L a step needs (its column below / row right of the
// diagonal, and the diagonal element) do not depend on y, so each step loads
// those of the step after next while its own multiply-adds run: the per-step chain
// is the owner's division, one barrier and one multiply-add. TH is one row
// per thread up to n = 1024 (no idle warps in each step's barrier). Measured
// at n = 512: 128 threads with four rows each is slower (the multiply-adds of
// a step are the larger cost), and so is a barrier-free hand-off through a
// shared-memory counter (the spinning threads slow the owner).
template <class O, int TH, int RMAX, bool UPPER_T>
__global__ void __launch_bounds__(TH) trsv_kernel(const typename O::T* __restrict__ L, typename O::T* y,
                                                  int64_t n) {
  using T = typename O::T;
  __shared__ T bc[2];
  const int t = threadIdx.x;
  T yr[RMAX], l0[RMAX], l1[RMAX];
  auto lval = [&](int64_t step, int r) {
    const int64_t j = UPPER_T ? n - 1 - step : step;
    const int64_t i = t + (int64_t)TH * r;
    const bool active = step < n && (UPPER_T ? (i < j) : (i > j && i < n));
    return active ? (UPPER_T ? L[j * n + i] : L[i * n + j]) : O::zero();
  };
  auto ldiag = [&](int64_t step) {
    const int64_t j = UPPER_T ? n - 1 - step : step;
    return (step < n && (int)(j % TH) == t) ? L[j * n + j] : O::zero();
  };
#pragma unroll
  for (int r = 0; r < RMAX; r++) {
    int64_t i = t + (int64_t)TH * r;
    yr[r] = i < n ? y[i] : O::zero();
    l0[r] = lval(0, r);
    l1[r] = lval(1, r);
  }
  T d0 = ldiag(0), d1 = ldiag(1);  // the diagonal entries of this step and the next
  for (int64_t step = 0; step < n; step++) {
    const int64_t j = UPPER_T ? n - 1 - step : step;
    const int owner = (int)(j % TH), rj = (int)(j / TH);
    if (t == owner) {
#pragma unroll
      for (int r = 0; r < RMAX; r++)
        if (r == rj) {
          yr[r] = O::div(yr[r], d0);
          bc[step & 1] = yr[r];
        }
    }
    __syncthreads();
    const T yj = bc[step & 1];
    // entries of step + 2, loaded two steps ahead (an L2 round trip is longer than a step's work)
    T l2[RMAX];
#pragma unroll
    for (int r = 0; r < RMAX; r++) l2[r] = lval(step + 2, r);
    const T d2 = ldiag(step + 2);
#pragma unroll
    for (int r = 0; r < RMAX; r++) {
      int64_t i = t + (int64_t)TH * r;
      bool active = UPPER_T ? (i < j) : (i > j && i < n);
      if (active) yr[r] = O::sub(yr[r], O::mul(l0[r], yj));
      l0[r] = l1[r];
      l1[r] = l2[r];
    }
    d0 = d1;
    d1 = d2;
  }
#pragma unroll
  for (int r = 0; r < RMAX; r++) {
    int64_t i = t + (int64_t)TH * r;
    if (i < n) y[i] = yr[r];
  }
}

// y = A x, one thread per row, sequential j order; A tiles of 128 rows x 16
// columns stream through shared memory.
__global__ void __launch_bounds__(128) matvec_dd_kernel(const dd* __restrict__ A, const dd* __restrict__ x, dd* y,
                                                        int64_t rows, int64_t cols) {
  __shared__ dd As[128][17];
  __shared__ dd xs[16];
  const int t = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * 128;
  dd s = dd{0.0, 0.0};
  for (int64_t c0 = 0; c0 < cols; c0 += 16) {
    __syncthreads();
    for (int e = t; e < 128 * 16; e += 128) {
      int rr = e / 16, cc = e % 16;
      int64_t gi = r0 + rr, gj = c0 + cc;
      As[rr][cc] = (gi < rows && gj < cols) ? A[gi * cols + gj] : dd{0.0, 0.0};
    }
    if (t < 16) xs[t] = (c0 + t < cols) ? x[c0 + t] : dd{0.0, 0.0};
    __syncthreads();
    const int cmax = (int)min((int64_t)16, cols - c0);
    for (int cc = 0; cc < cmax; cc++) s = dd_add(s, dd_mul(As[t][cc], xs[cc]));
  }
  if (r0 + t < rows) y[r0 + t] = s;
}

// solver/src/lib.rs:243-249: s = s + v*v in index order, sqrt, to_f64.
__global__ void norm_f128_kernel(const dd* __restrict__ v, int64_t n, double* out) {
  if (threadIdx.x != 0) return;
  dd s = dd{0.0, 0.0};
  for (int64_t i = 0; i < n; i++) s = dd_add(s, dd_mul(v[i], v[i]));
  dd r = dd_sqrt(s);
  *out = __dadd_rn(r.hi, r.lo);
}

// linalg.rs:185-194 / lib.rs:215-224: (max |d| / min |d|)^2 over the
// diagonal; max and min are exact, so a parallel reduction is bit-identical.
template <bool DD>
__global__ void cond_estimate_kernel(const double* L, int64_t n, double* out) {
  __shared__ double mx[256], mn[256];
  double dmax = 0.0, dmin = 1.7976931348623157e308;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    double d = DD ? fabs(__dadd_rn(L[2 * (i * n + i)], L[2 * (i * n + i) + 1])) : fabs(L[i * n + i]);
    dmax = fmax(dmax, d);
    dmin = fmin(dmin, d);
  }
  mx[threadIdx.x] = dmax;
  mn[threadIdx.x] = dmin;
  __syncthreads();
  for (int o = 128; o; o >>= 1) {
    if (threadIdx.x < o) {
      mx[threadIdx.x] = fmax(mx[threadIdx.x], mx[threadIdx.x + o]);
      mn[threadIdx.x] = fmin(mn[threadIdx.x], mn[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double r = __ddiv_rn(mx[0], mn[0]);
    *out = __dmul_rn(r, r);
  }
}

__global__ void vec_kernel(int op, const dd* a, const dd* b, dd* out, const double* f, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  switch (op) {
    case 0: out[i] = dd_sub(a[i], b[i]); break;   // r = b - ax
    case 1: out[i] = dd_add(a[i], b[i]); break;   // x = x + dx
    case 2: out[i] = dd{f[i], 0.0}; break;        // promote f64 -> f128
    case 3: reinterpret_cast<double*>(out)[i] = __dadd_rn(a[i].hi, a[i].lo); break;  // to_f64
  }
}

template <class O, bool UPPER_T>
int trsv_launch(const typename O::T* L, typename O::T* y, size_t n, cudaStream_t s) {
#define HP_TRSV(TH, RM) trsv_kernel<O, TH, RM, UPPER_T><<<1, TH, 0, s>>>(L, y, n)
  if (n <= 256) HP_TRSV(256, 1);
  else if (n <= 512) HP_TRSV(512, 1);
  else if (n <= 1024) HP_TRSV(1024, 1);
  else if (n <= 1024 * 2) HP_TRSV(1024, 2);
  else if (n <= 1024 * 4) HP_TRSV(1024, 4);
  else if (n <= 1024 * 8) HP_TRSV(1024, 8);
  else if (n <= 1024 * 16) HP_TRSV(1024, 16);
  else {
    set_error("triangular solve: n = %zu exceeds 16384", n);
    return HP_ERR_UNSUPPORTED;
  }
#undef HP_TRSV
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace

int dd_trsv(const double* L, double* y, size_t n, bool upper_t, cudaStream_t s) {
  if (n == 0) return HP_OK;
  return upper_t ? trsv_launch<VOpsDD, true>(reinterpret_cast<const dd*>(L), reinterpret_cast<dd*>(y), n, s)
                 : trsv_launch<VOpsDD, false>(reinterpret_cast<const dd*>(L), reinterpret_cast<dd*>(y), n, s);
}
int f64_trsv(const double* L, double* y, size_t n, bool upper_t, cudaStream_t s) {
  if (n == 0) return HP_OK;
  return upper_t ? trsv_launch<VOpsF64, true>(L, y, n, s) : trsv_launch<VOpsF64, false>(L, y, n, s);
}
// dot (linalg.rs:7-26): below 1024 entries one serial sum (dot_serial);
// otherwise each 1024-entry chunk is summed serially by one thread and the
// chunk sums are folded left to right from zero by one thread (rayon's
// reduce with the ZERO identity, in the order of a left fold).
__global__ void dot_chunks_kernel(const dd* __restrict__ a, const dd* __restrict__ b, int64_t len,
                                  dd* __restrict__ part) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c * 1024 >= len) return;
  const int64_t e = min(len, (c + 1) * 1024);
  dd s = {0.0, 0.0};
  for (int64_t i = c * 1024; i < e; i++) s = dd_add(s, dd_mul(a[i], b[i]));
  part[c] = s;
}
__global__ void dot_fold_kernel(const dd* __restrict__ part, int64_t nch, int fold, dd* __restrict__ out) {
  if (!fold) {
    *out = part[0];
    return;
  }
  dd t = {0.0, 0.0};
  for (int64_t c = 0; c < nch; c++) t = dd_add(t, part[c]);
  *out = t;
}
int dd_dot(const double* a, const double* b, size_t len, double* part, double* out, cudaStream_t s) {
  const int64_t nch = ((int64_t)len + 1023) / 1024;
  if (nch == 0) return HP_OK;
  dot_chunks_kernel<<<(unsigned)((nch + 127) / 128), 128, 0, s>>>(
      reinterpret_cast<const dd*>(a), reinterpret_cast<const dd*>(b), (int64_t)len, reinterpret_cast<dd*>(part));
  HP_LAUNCH_CHECK();
  dot_fold_kernel<<<1, 1, 0, s>>>(reinterpret_cast<const dd*>(part), nch, len >= 1024 ? 1 : 0,
                                  reinterpret_cast<dd*>(out));
  HP_LAUNCH_CHECK();
  return HP_OK;
}
int dd_matvec(const double* A, const double* x, double* y, size_t rows, size_t cols, cudaStream_t s) {
  if (rows == 0) return HP_OK;
  matvec_dd_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(
      reinterpret_cast<const dd*>(A), reinterpret_cast<const dd*>(x), reinterpret_cast<dd*>(y), rows, cols);
  HP_LAUNCH_CHECK();
  return HP_OK;
}
int dd_norm(const double* v, size_t n, double* out_dev, cudaStream_t s) {
  norm_f128_kernel<<<1, 32, 0, s>>>(reinterpret_cast<const dd*>(v), n, out_dev);
  HP_LAUNCH_CHECK();
  return HP_OK;
}
int cond_estimate(const double* L, size_t n, bool is_dd, double* out_dev, cudaStream_t s) {
  if (is_dd)
    cond_estimate_kernel<true><<<1, 256, 0, s>>>(L, n, out_dev);
  else
    cond_estimate_kernel<false><<<1, 256, 0, s>>>(L, n, out_dev);
  HP_LAUNCH_CHECK();
  return HP_OK;
}
int dd_vec(int op, const double* a, const double* b, double* out, const double* f, size_t n, cudaStream_t s) {
  if (n == 0) return HP_OK;
  vec_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(op, reinterpret_cast<const dd*>(a),
                                                          reinterpret_cast<const dd*>(b), reinterpret_cast<dd*>(out),
                                                          f, n);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace hp
