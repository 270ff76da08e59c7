// f512 (MultiFloat<8>) GEMM, Cholesky and Cholesky solve on CUDA cores:
//   hp_f512_gemm[_atb][_dev]  replace mf_gemm::<8> / mf_gemm_atb::<8>
//                             (crates/quad/src/multifloat/linalg.rs:39-85)
//   hp_f512_cholesky          replaces mf_cholesky::<8>       (linalg.rs:88-139)
//   hp_f512_cholesky_solve    replaces mf_cholesky_solve::<8> (linalg.rs:141-172)
// with the MultiFloat<8> arithmetic of hp_mf.cuh (the reference's operation
// sequences, bit for bit).
//
// GEMM: one C entry per thread, s = s + a_ip b_pj in p order from zero (the
// reference's loop), operands staged through shared memory in 8-deep
// k-slices; bit-identical.
// Cholesky: right-looking one column at a time with the running sums in a
// separate accumulator S: when column j is final, every sum s_iq of the
// trailing lower triangle adds L_ij L_qj. Each sum therefore receives the
// reference's products in the reference's order (k ascending, from zero),
// so the factor is bit-identical; per column, one launch forms the pivot
// (sqrt, recip: each block recomputes it, the same bits) and scales the
// column, and one launch updates the sums.
// Solve: one CTA, right-looking: forward bit-identical (each row's
// subtractions in j ascending order), backward with each row's
// subtractions in j descending order (the ascending order of the reference
// chains the whole sweep serially), f512-accurate rather than bit-identical.
#include <algorithm>

#include "hp_mf.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
namespace {

using mf8 = mfn<8>;

__device__ __forceinline__ mf8 ld8(const double* p) {
  const double4* q = reinterpret_cast<const double4*>(p);
  const double4 a = q[0], b = q[1];
  return mf8{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
}
__device__ __forceinline__ void st8(double* p, const mf8& v) {
  double4* q = reinterpret_cast<double4*>(p);
  q[0] = make_double4(v.l[0], v.l[1], v.l[2], v.l[3]);
  q[1] = make_double4(v.l[4], v.l[5], v.l[6], v.l[7]);
}

constexpr int G8_T = 16, G8_BK = 8;

template <bool ATB>
__global__ void __launch_bounds__(G8_T* G8_T) mf8_gemm_kernel(const double* __restrict__ A, const double* __restrict__ B,
                                                             double* __restrict__ C, int64_t m, int64_t n, int64_t k) {
  __shared__ double As[G8_BK][G8_T][9];  // [k][row][limb] (padded)
  __shared__ double Bs[G8_BK][G8_T][9];  // [k][col][limb]
  const int tx = threadIdx.x, ty = threadIdx.y, t = ty * G8_T + tx;
  const int64_t i0 = (int64_t)blockIdx.y * G8_T, j0 = (int64_t)blockIdx.x * G8_T;
  const int64_t gi = i0 + ty, gj = j0 + tx;
  mf8 acc = mfn_zero<8>();
  for (int64_t k0 = 0; k0 < k; k0 += G8_BK) {
    __syncthreads();
    // 8 k x 16 rows x 8 limbs of A and of B: 1024 doubles each, 4 per thread
    for (int e = t; e < G8_BK * G8_T * 8; e += G8_T * G8_T) {
      const int kk = e / (G8_T * 8), rem = e % (G8_T * 8), r = rem / 8, q = rem % 8;
      const int64_t p = k0 + kk;
      const int64_t ai = i0 + r, bj = j0 + r;
      As[kk][r][q] = (ai < m && p < k) ? (ATB ? A[(p * m + ai) * 8 + q] : A[(ai * k + p) * 8 + q]) : 0.0;
      Bs[kk][r][q] = (bj < n && p < k) ? B[(p * n + bj) * 8 + q] : 0.0;
    }
    __syncthreads();
    const int kmax = (int)min((int64_t)G8_BK, k - k0);
    for (int kk = 0; kk < kmax; kk++) {
      mf8 a, b;
#pragma unroll
      for (int q = 0; q < 8; q++) a.l[q] = As[kk][ty][q], b.l[q] = Bs[kk][tx][q];
      acc = mfn_add<8>(acc, mfn_mul<8>(a, b));
    }
  }
  if (gi < m && gj < n) st8(C + (gi * n + gj) * 8, acc);
}

struct Mf8Err {
  int flag;
  int pad;
  long long pivot;
};

// Column j: the pivot (recomputed by thread 0 of every block, the same bits),
// then L_ij = (A_ij - s_ij) recip(L_jj) for the block's rows i > j.
constexpr int C8_THREADS = 128;
__global__ void __launch_bounds__(C8_THREADS) mf8_chol_column_kernel(double* A, const double* S, int64_t n, int64_t j,
                                                                     Mf8Err* err) {
  __shared__ double inv_s[8];
  __shared__ int fail;
  if (err->flag) return;
  const int t = threadIdx.x;
  if (t == 0) {
    const mf8 d = mfn_sub<8>(ld8(A + (j * n + j) * 8), ld8(S + (j * n + j) * 8));
    if (d.l[0] <= 0.0) {  // multifloat/linalg.rs:105-107
      fail = 1;
      if (blockIdx.x == 0) {
        err->flag = 1;
        err->pivot = j;
      }
    } else {
      fail = 0;
      const mf8 l = mfn_sqrt<8>(d);
      const mf8 inv = mfn_recip<8>(l);
#pragma unroll
      for (int q = 0; q < 8; q++) inv_s[q] = inv.l[q];
      if (blockIdx.x == 0) st8(A + (j * n + j) * 8, l);
    }
  }
  __syncthreads();
  if (fail) return;
  const int64_t i = j + 1 + (int64_t)blockIdx.x * C8_THREADS + t;
  if (i >= n) return;
  mf8 inv;
#pragma unroll
  for (int q = 0; q < 8; q++) inv.l[q] = inv_s[q];
  st8(A + (i * n + j) * 8, mfn_mul<8>(mfn_sub<8>(ld8(A + (i * n + j) * 8), ld8(S + (i * n + j) * 8)), inv));
}

// s_iq += L_ij L_qj for j < q <= i < n: 16 x 16 tiles of the trailing lower
// triangle (tile rows >= tile columns), one sum per thread.
__global__ void __launch_bounds__(256) mf8_chol_update_kernel(const double* A, double* S, int64_t n, int64_t j,
                                                              const Mf8Err* err) {
  if (err->flag) return;
  const int64_t t0 = j + 1;
  int64_t idx = blockIdx.x;
  int64_t bi = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
  while (bi * (bi + 1) / 2 > idx) bi--;
  while ((bi + 1) * (bi + 2) / 2 <= idx) bi++;
  const int64_t bq = idx - bi * (bi + 1) / 2;
  const int64_t i = t0 + bi * 16 + threadIdx.x / 16, q = t0 + bq * 16 + threadIdx.x % 16;
  if (i >= n || q > i) return;
  const mf8 lij = ld8(A + (i * n + j) * 8);
  const mf8 prod = i == q ? mfn_mul<8>(lij, lij) : mfn_mul<8>(lij, ld8(A + (q * n + j) * 8));
  st8(S + (i * n + q) * 8, mfn_add<8>(ld8(S + (i * n + q) * 8), prod));
}

// In-place v <- L^-1 v (upper = 0) or L^-T v (upper = 1), one CTA.
constexpr int S8_THREADS = 256;
__global__ void __launch_bounds__(S8_THREADS) mf8_sweep_kernel(const double* __restrict__ L, double* __restrict__ v,
                                                               int64_t n, int upper) {
  __shared__ double vj[2][8];
  const int t = threadIdx.x;
  for (int64_t s = 0; s < n; s++) {
    const int64_t j = upper ? n - 1 - s : s;
    if (j % S8_THREADS == t) {
      const mf8 x = mfn_div<8>(ld8(v + j * 8), ld8(L + (j * n + j) * 8));
      st8(v + j * 8, x);
#pragma unroll
      for (int q = 0; q < 8; q++) vj[s & 1][q] = x.l[q];
    }
    __syncthreads();
    mf8 y;
#pragma unroll
    for (int q = 0; q < 8; q++) y.l[q] = vj[s & 1][q];
    for (int64_t i = t; i < n; i += S8_THREADS) {
      if (upper ? i < j : i > j) {
        const mf8 l = ld8(L + (upper ? j * n + i : i * n + j) * 8);
        st8(v + i * 8, mfn_sub<8>(ld8(v + i * 8), mfn_mul<8>(l, y)));
      }
    }
    // vj[s & 1] is rewritten two steps later, after the next barrier
  }
}

}  // namespace

int mf8_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, bool atb, cudaStream_t s) {
  if (m == 0 || n == 0) return HP_OK;
  if (k == 0) {
    HP_CUDA_TRY(cudaMemsetAsync(c, 0, m * n * 64, s));
    return HP_OK;
  }
  if ((m + G8_T - 1) / G8_T > 65535) {
    set_error("f512 gemm: m = %zu exceeds the grid limit", m);
    return HP_ERR_INVALID_ARG;
  }
  dim3 grid((unsigned)((n + G8_T - 1) / G8_T), (unsigned)((m + G8_T - 1) / G8_T)), block(G8_T, G8_T);
  if (atb)
    mf8_gemm_kernel<true><<<grid, block, 0, s>>>(a, b, c, (int64_t)m, (int64_t)n, (int64_t)k);
  else
    mf8_gemm_kernel<false><<<grid, block, 0, s>>>(a, b, c, (int64_t)m, (int64_t)n, (int64_t)k);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

// Factor in place; synchronises s and returns HP_ERR_NOT_SPD with *pivot.
int mf8_cholesky(double* a, size_t n, int64_t* pivot, cudaStream_t s) {
  if (n == 0) return HP_OK;
  DevBuf S(n * n * 64, s), err(sizeof(Mf8Err), s);
  if (!S.p || !err.p) {
    set_error("f512 cholesky: workspace allocation failed");
    return HP_ERR_CUDA;
  }
  HP_CUDA_TRY(cudaMemsetAsync(S.p, 0, n * n * 64, s));
  HP_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(Mf8Err), s));
  for (size_t j = 0; j < n; j++) {
    const size_t rows = n - j - 1;
    const unsigned blocks = (unsigned)std::max<size_t>(1, (rows + C8_THREADS - 1) / C8_THREADS);
    mf8_chol_column_kernel<<<blocks, C8_THREADS, 0, s>>>(a, S.as<double>(), (int64_t)n, (int64_t)j, err.as<Mf8Err>());
    HP_LAUNCH_CHECK();
    if (rows == 0) break;
    const size_t tiles = (rows + 15) / 16;
    mf8_chol_update_kernel<<<(unsigned)(tiles * (tiles + 1) / 2), 256, 0, s>>>(a, S.as<double>(), (int64_t)n,
                                                                               (int64_t)j, err.as<Mf8Err>());
    HP_LAUNCH_CHECK();
  }
  Mf8Err h;
  HP_CUDA_TRY(cudaMemcpyAsync(&h, err.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (h.flag) {
    if (pivot) *pivot = h.pivot;
    set_error("Cholesky failed: matrix is not positive definite (pivot %lld)", h.pivot);
    return HP_ERR_NOT_SPD;
  }
  return HP_OK;
}

int mf8_cholesky_solve(const double* L, double* v, size_t n, cudaStream_t s) {
  if (n == 0) return HP_OK;
  mf8_sweep_kernel<<<1, S8_THREADS, 0, s>>>(L, v, (int64_t)n, 0);
  HP_LAUNCH_CHECK();
  mf8_sweep_kernel<<<1, S8_THREADS, 0, s>>>(L, v, (int64_t)n, 1);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace hp

namespace {
int f512_check(size_t a, size_t b, size_t* bytes) {
  size_t t;
  if (hp::mul_overflows(a, b, &t) || hp::mul_overflows(t, 64, bytes)) {
    hp::set_error("matrix size overflows size_t");
    return HP_ERR_INVALID_ARG;
  }
  return HP_OK;
}
}  // namespace

extern "C" {

int hp_f512_gemm_dev(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, int atb,
                     void* stream) {
  using namespace hp;
  size_t ba, bb, bc;
  HP_TRY(f512_check(m, k, &ba));
  HP_TRY(f512_check(k, n, &bb));
  HP_TRY(f512_check(m, n, &bc));
  if ((ba && !a) || (bb && !b) || (bc && !c)) {
    set_error("null pointer with non-zero size");
    return HP_ERR_INVALID_ARG;
  }
  if (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c) % 32) {
    set_error("device pointers must be 32-byte aligned");
    return HP_ERR_INVALID_ARG;
  }
  return mf8_gemm(a, b, c, m, n, k, atb != 0, (cudaStream_t)stream);
}

static int f512_gemm_host(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, bool atb) {
  using namespace hp;
  size_t ba, bb, bc;
  HP_TRY(f512_check(m, k, &ba));
  HP_TRY(f512_check(k, n, &bb));
  HP_TRY(f512_check(m, n, &bc));
  if ((ba && !a) || (bb && !b) || (bc && !c)) {
    set_error("null pointer with non-zero size");
    return HP_ERR_INVALID_ARG;
  }
  if (bc == 0) return HP_OK;
  cudaStream_t s = library_stream();
  DevBuf da(ba, s), db(bb, s), dc(bc, s);
  if ((ba && !da.p) || (bb && !db.p) || !dc.p) return HP_ERR_CUDA;
  if (ba) HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, ba, cudaMemcpyHostToDevice, s));
  if (bb) HP_CUDA_TRY(cudaMemcpyAsync(db.p, b, bb, cudaMemcpyHostToDevice, s));
  HP_TRY(mf8_gemm(da.as<double>(), db.as<double>(), dc.as<double>(), m, n, k, atb, s));
  HP_CUDA_TRY(cudaMemcpyAsync(c, dc.p, bc, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_f512_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k) {
  return f512_gemm_host(a, b, c, m, n, k, false);
}
int hp_f512_gemm_atb(const double* a, const double* b, double* c, size_t m, size_t n, size_t k) {
  return f512_gemm_host(a, b, c, m, n, k, true);
}

int hp_f512_cholesky(double* a, size_t n, int64_t* pivot) {
  using namespace hp;
  size_t bytes;
  HP_TRY(f512_check(n, n, &bytes));
  if (n == 0) return HP_OK;
  if (!a) {
    set_error("null matrix");
    return HP_ERR_INVALID_ARG;
  }
  cudaStream_t s = library_stream();
  DevBuf da(bytes, s);
  if (!da.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, bytes, cudaMemcpyHostToDevice, s));
  HP_TRY(mf8_cholesky(da.as<double>(), n, pivot, s));
  HP_CUDA_TRY(cudaMemcpyAsync(a, da.p, bytes, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_f512_cholesky_solve(const double* l, const double* b, double* x, size_t n) {
  using namespace hp;
  size_t bytes;
  HP_TRY(f512_check(n, n, &bytes));
  if (n == 0) return HP_OK;
  if (!l || !b || !x) {
    set_error("null pointer");
    return HP_ERR_INVALID_ARG;
  }
  cudaStream_t s = library_stream();
  DevBuf dl(bytes, s), dv(n * 64, s);
  if (!dl.p || !dv.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dl.p, l, bytes, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dv.p, b, n * 64, cudaMemcpyHostToDevice, s));
  HP_TRY(mf8_cholesky_solve(dl.as<double>(), dv.as<double>(), n, s));
  HP_CUDA_TRY(cudaMemcpyAsync(x, dv.p, n * 64, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

}  // extern "C"
