// Canonical orthogonalisation and the generalised symmetric eigenproblem,
// behind the C ABI:
//   hp_canonical_orthogonalize replaces canonical_orthogonalize
//   (crates/solver/src/ortho.rs:147-183): diagonalise S, keep the
//   eigenvalues whose f64 value (hi + lo) exceeds the threshold, sorted
//   ascending (stable), and return X = U diag(1 / sqrt(lambda)) (n x m,
//   row-major) with 1/sqrt(lambda) = lambda.sqrt().recip() in f128.
//   hp_solve_gen_eigen replaces solve_gen_eigen (ortho.rs:185-239):
//   F' = X^T (F X) with the reference's f128 GEMMs (gemm_rect,
//   ortho.rs:41-55, and gemm_atb, linalg.rs:168-182: both accumulate each
//   entry in k order, as the plain GPU GEMM does bit for bit), F'
//   symmetrised by (F'_ij + F'_ji) * 0.5, diagonalised, eigenpairs sorted
//   ascending (stable) and C = X C'.
// The eigenpairs come from the GPU Jacobi solver (parallel round-robin
// rotations, n <= 128) instead of the reference's private max-pivot Jacobi
// (ortho.rs:58-143): eigenvalues agree to f128 rounding and each column of X
// (and of C) to rounding and sign (eigenvectors are defined up to sign).
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

// F' := (F'_ij + F'_ji) * 0.5 above and below the diagonal (ortho.rs:205-212).
__global__ void symmetrize_kernel(dd* __restrict__ A, int64_t m) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m * m) return;
  const int64_t i = q / m, j = q % m;
  if (j <= i) return;
  const dd avg = dd_mul(dd_add(A[i * m + j], A[j * m + i]), dd_from(0.5));
  A[i * m + j] = avg;
  A[j * m + i] = avg;
}

// C'[i][k] = V[order[k]][i]: eigenvector order[k] (a row of V) as column k.
__global__ void sorted_columns_kernel(const dd* __restrict__ V, const int32_t* __restrict__ order, int64_t m,
                                      dd* __restrict__ C) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m * m) return;
  const int64_t i = q / m, k = q % m;
  C[q] = V[(int64_t)order[k] * m + i];
}

// Eigenpairs of the symmetric n x n f128 matrix dA (device) on the GPU:
// eigenvalues to the host (lam, 2 doubles each), eigenvectors as rows of dV.
int jacobi_host_evals(const dd* dA, size_t n, dd* dl, dd* dV, std::vector<double>& lam, cudaStream_t st) {
  DevBuf dsw(8, st);
  if (!dsw.p) return HP_ERR_CUDA;
  int64_t noff[2] = {0, (int64_t)n};
  int32_t* dsweeps = dsw.as<int32_t>();
  HP_TRY(hp_f128_jacobi_eigen_batched_dev(1, noff, reinterpret_cast<const double*>(dA), 1000,
                                          reinterpret_cast<double*>(dl), reinterpret_cast<double*>(dV), dsweeps,
                                          dsweeps + 1, st));
  int32_t h[2];
  lam.assign(2 * n, 0.0);
  HP_CUDA_TRY(cudaMemcpyAsync(h, dsw.p, 8, cudaMemcpyDeviceToHost, st));
  HP_CUDA_TRY(cudaMemcpyAsync(lam.data(), dl, n * 16, cudaMemcpyDeviceToHost, st));
  HP_CUDA_TRY(cudaStreamSynchronize(st));
  if (h[1] != HP_OK) {
    set_error("Jacobi did not converge");
    return HP_ERR_NO_CONVERGE;
  }
  return HP_OK;
}

// X (n x m, device) of the canonical orthogonalisation of the device matrix dS.
int ortho_basis(const dd* dS, size_t n, double threshold, dd* dX, size_t* m_out, cudaStream_t st) {
  DevBuf dl(n * 16, st), dV(n * n * 16, st), didx(n * 4, st);
  if (!dl.p || !dV.p || !didx.p) return HP_ERR_CUDA;
  std::vector<double> lam;
  HP_TRY(jacobi_host_evals(dS, n, dl.as<dd>(), dV.as<dd>(), lam, st));
  // ortho.rs:155-165: filter on to_f64() > threshold, stable sort ascending
  std::vector<int32_t> keep;
  for (size_t i = 0; i < n; i++)
    if (lam[2 * i] + lam[2 * i + 1] > threshold) keep.push_back((int32_t)i);
  std::stable_sort(keep.begin(), keep.end(), [&](int32_t a, int32_t b) {
    return lam[2 * a] + lam[2 * a + 1] < lam[2 * b] + lam[2 * b + 1];
  });
  const size_t m = keep.size();
  *m_out = m;
  if (m == 0) return HP_OK;
  HP_CUDA_TRY(cudaMemcpyAsync(didx.p, keep.data(), m * 4, cudaMemcpyHostToDevice, st));
  ortho_x_kernel<<<(unsigned)((n * m + 127) / 128), 128, 0, st>>>(dV.as<dd>(), dl.as<dd>(), didx.as<int32_t>(),
                                                                 (int64_t)n, (int64_t)m, dX);
  HP_LAUNCH_CHECK();
  return HP_OK;
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
  DevBuf dS(n * n * 16, st), dX(n * n * 16, st);
  if (!dS.p || !dX.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dS.p, s, n * n * 16, cudaMemcpyHostToDevice, st));
  size_t m = 0;
  const int rc = ortho_basis(dS.as<dd>(), n, threshold, dX.as<dd>(), &m, st);
  if (rc != HP_OK) {
    if (rc == HP_ERR_NO_CONVERGE) set_error("canonical_orthogonalize: Jacobi did not converge");
    return rc;
  }
  *n_orth = m;
  if (m == 0) return HP_OK;
  HP_CUDA_TRY(cudaMemcpyAsync(x, dX.p, n * m * 16, cudaMemcpyDeviceToHost, st));
  HP_CUDA_TRY(cudaStreamSynchronize(st));
  return HP_OK;
}

extern "C" int hp_solve_gen_eigen(const double* f, const double* s, size_t n, double threshold, double* eigenvalues,
                                  double* eigenvectors, size_t* n_basis) {
  using namespace hp;
  if (!n_basis) return HP_ERR_INVALID_ARG;
  *n_basis = 0;
  if (n == 0) return HP_OK;
  if (!f || !s || !eigenvalues || !eigenvectors) return HP_ERR_INVALID_ARG;
  if (n > 128) {
    set_error("solve_gen_eigen: n = %zu exceeds the Jacobi solver's 128", n);
    return HP_ERR_UNSUPPORTED;
  }
  cudaStream_t st = library_stream();
  DevBuf dF(n * n * 16, st), dS(n * n * 16, st), dX(n * n * 16, st), dT(n * n * 16, st), dFp(n * n * 16, st),
      dl(n * 16, st), dV(n * n * 16, st), dC1(n * n * 16, st), dord(n * 4, st), dC(n * n * 16, st);
  if (!dF.p || !dS.p || !dX.p || !dT.p || !dFp.p || !dl.p || !dV.p || !dC1.p || !dord.p || !dC.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dF.p, f, n * n * 16, cudaMemcpyHostToDevice, st));
  HP_CUDA_TRY(cudaMemcpyAsync(dS.p, s, n * n * 16, cudaMemcpyHostToDevice, st));
  size_t m = 0;
  int rc = ortho_basis(dS.as<dd>(), n, threshold, dX.as<dd>(), &m, st);
  if (rc != HP_OK) {
    if (rc == HP_ERR_NO_CONVERGE) set_error("solve_gen_eigen: Jacobi (S) did not converge");
    return rc;
  }
  if (m == 0) return HP_OK;
  // tmp = F X (n x m, gemm_rect), F' = X^T tmp (m x m, gemm_atb)
  HP_TRY(dd_gemm_plain(dF.as<double>(), dX.as<double>(), dT.as<double>(), n, m, n, false, st));
  HP_TRY(dd_gemm_plain(dX.as<double>(), dT.as<double>(), dFp.as<double>(), m, m, n, true, st));
  symmetrize_kernel<<<(unsigned)((m * m + 127) / 128), 128, 0, st>>>(dFp.as<dd>(), (int64_t)m);
  HP_LAUNCH_CHECK();
  std::vector<double> lam;
  rc = jacobi_host_evals(dFp.as<dd>(), m, dl.as<dd>(), dV.as<dd>(), lam, st);
  if (rc != HP_OK) {
    if (rc == HP_ERR_NO_CONVERGE) set_error("solve_gen_eigen: Jacobi (F') did not converge");
    return rc;
  }
  // ortho.rs:218-229: ascending by to_f64(), stable; eigenvectors reordered as columns
  std::vector<int32_t> order(m);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return lam[2 * a] + lam[2 * a + 1] < lam[2 * b] + lam[2 * b + 1];
  });
  HP_CUDA_TRY(cudaMemcpyAsync(dord.p, order.data(), m * 4, cudaMemcpyHostToDevice, st));
  sorted_columns_kernel<<<(unsigned)((m * m + 127) / 128), 128, 0, st>>>(dV.as<dd>(), dord.as<int32_t>(),
                                                                         (int64_t)m, dC1.as<dd>());
  HP_LAUNCH_CHECK();
  // C = X C' (n x m, gemm_rect)
  HP_TRY(dd_gemm_plain(dX.as<double>(), dC1.as<double>(), dC.as<double>(), n, m, m, false, st));
  HP_CUDA_TRY(cudaMemcpyAsync(eigenvectors, dC.p, n * m * 16, cudaMemcpyDeviceToHost, st));
  HP_CUDA_TRY(cudaStreamSynchronize(st));
  for (size_t k = 0; k < m; k++) {
    eigenvalues[2 * k] = lam[2 * order[k]];
    eigenvalues[2 * k + 1] = lam[2 * order[k] + 1];
  }
  *n_basis = m;
  return HP_OK;
}
