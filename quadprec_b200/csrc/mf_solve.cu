// f256 (MultiFloat<4>) Cholesky factor and solves behind the C ABI:
//   hp_f256_cholesky[_dev]   replaces mf_cholesky::<4>   (crates/quad/src/multifloat/linalg.rs:88-139)
//   hp_f256_cholesky_solve   replaces mf_cholesky_solve::<4> (linalg.rs:141-172)
//   hp_f256_gemv, hp_f256_dot replace mf_gemv::<4>, mf_dot::<4> (linalg.rs:7-37):
//   bit-identical, each row summed s = s + a_ij x_j in j order by one thread
// The factor is the blocked kernel set of cholesky.cu with MultiFloat<4>
// arithmetic, bit-identical to the reference. The solve runs on one CTA,
// right-looking: at step j the owner of row j finishes it (v_j / l_jj, the
// reference's division) and every later row subtracts its product with v_j.
// Forward, that applies each row's subtractions in the reference's order
// (j ascending), so it is bit-identical; backward, the rows receive them
// for j descending instead of ascending (the ascending order chains the
// whole sweep serially), so that sweep is f256-accurate, not bit-identical.
#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
int qd_cholesky(double* a, size_t n, int64_t* pivot, cudaStream_t s);

namespace {

constexpr int MS_THREADS = 1024;

// In-place v <- L^-1 v (upper = 0) or L^-T v (upper = 1).
__global__ void __launch_bounds__(MS_THREADS) qd_chol_sweep_kernel(const qd* __restrict__ L, qd* __restrict__ v,
                                                                   int64_t n, int upper) {
  __shared__ qd vj[2];
  const int t = threadIdx.x;
  for (int64_t s = 0; s < n; s++) {
    const int64_t j = upper ? n - 1 - s : s;
    if (j % MS_THREADS == t) {
      const qd x = qd_div(v[j], L[j * n + j]);
      v[j] = x;
      vj[s & 1] = x;
    }
    __syncthreads();
    const qd y = vj[s & 1];
    for (int64_t i = t; i < n; i += MS_THREADS) {
      if (upper ? i < j : i > j) v[i] = qd_sub(v[i], qd_mul(upper ? L[j * n + i] : L[i * n + j], y));
    }
    // vj[s & 1] is rewritten two steps later, after the next barrier
  }
}

// y_i = sum_j a_ij x_j in MultiFloat<4>, j ascending (the reference's order),
// one thread per row; x is read by every thread of a warp at once.
__global__ void qd_gemv_kernel(const qd* __restrict__ A, const qd* __restrict__ x, qd* __restrict__ y, int64_t n,
                               int64_t m) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const qd* row = A + i * m;
  qd s = qd_zero();
  for (int64_t j = 0; j < m; j++) s = qd_add(s, qd_mul(row[j], x[j]));
  y[i] = s;
}

}  // namespace

int qd_gemv(const double* A, const double* x, double* y, size_t n, size_t m, cudaStream_t s) {
  if (n == 0) return HP_OK;
  qd_gemv_kernel<<<(unsigned)((n + 63) / 64), 64, 0, s>>>(reinterpret_cast<const qd*>(A), reinterpret_cast<const qd*>(x),
                                                          reinterpret_cast<qd*>(y), (int64_t)n, (int64_t)m);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

int qd_cholesky_solve(const double* L, double* v, size_t n, cudaStream_t s) {
  if (n == 0) return HP_OK;
  const qd* Lq = reinterpret_cast<const qd*>(L);
  qd* vq = reinterpret_cast<qd*>(v);
  qd_chol_sweep_kernel<<<1, MS_THREADS, 0, s>>>(Lq, vq, (int64_t)n, 0);
  HP_LAUNCH_CHECK();
  qd_chol_sweep_kernel<<<1, MS_THREADS, 0, s>>>(Lq, vq, (int64_t)n, 1);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace hp

extern "C" {

int hp_f256_cholesky_dev(double* a, size_t n, int64_t* pivot, void* stream) {
  if (n && !a) return HP_ERR_INVALID_ARG;
  if ((uintptr_t)a % 32) {
    hp::set_error("device pointer must be 32-byte aligned");
    return HP_ERR_INVALID_ARG;
  }
  return hp::qd_cholesky(a, n, pivot, (cudaStream_t)stream);
}

int hp_f256_cholesky(double* a, size_t n, int64_t* pivot) {
  using namespace hp;
  if (n == 0) return HP_OK;
  size_t bytes;
  if (!a || mul_overflows(n, n, &bytes) || mul_overflows(bytes, 32, &bytes)) return HP_ERR_INVALID_ARG;
  cudaStream_t s = library_stream();
  DevBuf d(bytes, s);
  if (!d.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(d.p, a, bytes, cudaMemcpyHostToDevice, s));
  HP_TRY(qd_cholesky(d.as<double>(), n, pivot, s));
  HP_CUDA_TRY(cudaMemcpyAsync(a, d.p, bytes, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_f256_gemv(const double* a, const double* x, double* y, size_t n, size_t m) {
  using namespace hp;
  if (n == 0) return HP_OK;
  size_t bytes;
  if (!a || !y || (m && !x) || mul_overflows(n, m, &bytes) || mul_overflows(bytes, 32, &bytes))
    return HP_ERR_INVALID_ARG;
  cudaStream_t s = library_stream();
  DevBuf da(bytes ? bytes : 32, s), dx(m ? m * 32 : 32, s), dy(n * 32, s);
  if (!da.p || !dx.p || !dy.p) return HP_ERR_CUDA;
  if (bytes) HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, bytes, cudaMemcpyHostToDevice, s));
  if (m) HP_CUDA_TRY(cudaMemcpyAsync(dx.p, x, m * 32, cudaMemcpyHostToDevice, s));
  HP_TRY(qd_gemv(da.as<double>(), dx.as<double>(), dy.as<double>(), n, m, s));
  HP_CUDA_TRY(cudaMemcpyAsync(y, dy.p, n * 32, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_f256_dot(const double* a, const double* b, size_t len, double* out) {
  if (!out) return HP_ERR_INVALID_ARG;
  return hp_f256_gemv(a, b, out, 1, len);
}

int hp_f256_cholesky_solve(const double* l, const double* b, double* x, size_t n) {
  using namespace hp;
  if (n == 0) return HP_OK;
  size_t bytes;
  if (!l || !b || !x || mul_overflows(n, n, &bytes) || mul_overflows(bytes, 32, &bytes)) return HP_ERR_INVALID_ARG;
  cudaStream_t s = library_stream();
  DevBuf dl(bytes, s), dv(n * 32, s);
  if (!dl.p || !dv.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dl.p, l, bytes, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dv.p, b, n * 32, cudaMemcpyHostToDevice, s));
  HP_TRY(qd_cholesky_solve(dl.as<double>(), dv.as<double>(), n, s));
  HP_CUDA_TRY(cudaMemcpyAsync(x, dv.p, n * 32, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

}  // extern "C"
