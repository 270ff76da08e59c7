// Canonical orthogonalisation of an overlap matrix, behind the C ABI:
//   hp_canonical_orthogonalize replaces canonical_orthogonalize
//   (crates/solver/src/ortho.rs:147-183): diagonalise S, keep the
//   eigenvalues whose f64 value (hi + lo) exceeds the threshold, sorted
//   ascending (stable), and return X = U diag(1 / sqrt(lambda)) (n x m,
//   row-major) with 1/sqrt(lambda) = lambda.sqrt().recip() in f128.
// The eigenpairs come from the GPU Jacobi solver (parallel round-robin
// rotations, n <= 128) instead of the reference's private max-pivot Jacobi
// (ortho.rs:58-143): eigenvalues agree to f128 rounding and each column of X
// to rounding and sign (eigenvectors are defined up to sign).
#include <algorithm>
#include <numeric>
#include <vector>

#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
namespace {

// X[i][k] = V[idx[k]][i] * recip(sqrt(lambda[idx[k]])), V's rows the eigenvectors.
__global__ void ortho_x_kernel(const dd* __restrict__ V, const dd* __restrict__ lam, const int32_t* __restrict__ idx,
                               int64_t n, int64_t m, dd* __restrict__ X) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n * m) return;
  const int64_t i = q / m, k = q % m;
  const int64_t e = idx[k];
  const dd inv_sqrt = dd_recip(dd_sqrt(lam[e]));  // ortho.rs:175
  X[q] = dd_mul(V[e * n + i], inv_sqrt);
}

}  // namespace
}  // namespace hp

extern "C" int hp_canonical_orthogonalize(const double* s, size_t n, double threshold, double* x,
                                          size_t* n_orth) {
  using namespace hp;
  if (!n_orth) return HP_ERR_INVALID_ARG;
  *n_orth = 0;
  if (n == 0) return HP_OK;
  if (!s || !x) return HP_ERR_INVALID_ARG;
  if (n > 128) {
    set_error("canonical_orthogonalize: n = %zu exceeds the Jacobi solver's 128", n);
    return HP_ERR_UNSUPPORTED;
  }
  cudaStream_t st = library_stream();
  DevBuf dS(n * n * 16, st), dl(n * 16, st), dV(n * n * 16, st), dsw(8, st), didx(n * 4, st), dX(n * n * 16, st);
  if (!dS.p || !dl.p || !dV.p || !dsw.p || !didx.p || !dX.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dS.p, s, n * n * 16, cudaMemcpyHostToDevice, st));
  int64_t noff[2] = {0, (int64_t)n};
  int32_t* dsweeps = dsw.as<int32_t>();
  HP_TRY(hp_f128_jacobi_eigen_batched_dev(1, noff, dS.as<double>(), 1000, dl.as<double>(), dV.as<double>(), dsweeps,
                                          dsweeps + 1, st));
  int32_t h[2];
  std::vector<double> lam(2 * n);
  HP_CUDA_TRY(cudaMemcpyAsync(h, dsw.p, 8, cudaMemcpyDeviceToHost, st));
  HP_CUDA_TRY(cudaMemcpyAsync(lam.data(), dl.p, n * 16, cudaMemcpyDeviceToHost, st));
  HP_CUDA_TRY(cudaStreamSynchronize(st));
  if (h[1] != HP_OK) {
    set_error("canonical_orthogonalize: Jacobi did not converge");
    return HP_ERR_NO_CONVERGE;
  }
  // ortho.rs:155-165: filter on to_f64() > threshold, stable sort ascending
  std::vector<int32_t> keep;
  for (size_t i = 0; i < n; i++)
    if (lam[2 * i] + lam[2 * i + 1] > threshold) keep.push_back((int32_t)i);
  std::stable_sort(keep.begin(), keep.end(), [&](int32_t a, int32_t b) {
    return lam[2 * a] + lam[2 * a + 1] < lam[2 * b] + lam[2 * b + 1];
  });
  const size_t m = keep.size();
  *n_orth = m;
  if (m == 0) return HP_OK;
  HP_CUDA_TRY(cudaMemcpyAsync(didx.p, keep.data(), m * 4, cudaMemcpyHostToDevice, st));
  ortho_x_kernel<<<(unsigned)((n * m + 127) / 128), 128, 0, st>>>(dV.as<dd>(), dl.as<dd>(), didx.as<int32_t>(),
                                                                 (int64_t)n, (int64_t)m, dX.as<dd>());
  HP_LAUNCH_CHECK();
  HP_CUDA_TRY(cudaMemcpyAsync(x, dX.p, n * m * 16, cudaMemcpyDeviceToHost, st));
  HP_CUDA_TRY(cudaStreamSynchronize(st));
  return HP_OK;
}
