// Adjoint of overlap assembly + SPD solve: the gradient of
//     L = b^T S^-1 b,   S_uv = (4 a_u a_v/(a_u+a_v)^2)^{3/4} exp(-p_uv r_uv^2),
//     p_uv = a_u a_v / (a_u + a_v),  r_uv = |R_u - R_v|,
// with respect to the centre coordinates and the log-exponents:
//     dL/dtheta = -lambda^T (dS/dtheta) lambda,  lambda = S^-1 b,
//     dS_uv/dR_u      = -2 p_uv (R_u - R_v) S_uv,
//     dS_uv/d ln a_u  = S_uv [ (3/4)(a_v - a_u)/(a_u + a_v) - r^2 a_u a_v^2/(a_u + a_v)^2 ].
// By symmetry of S:
//     dL/dR_C     = 4 sum_{u in C} lambda_u sum_v lambda_v p_uv (R_u - R_v) S_uv,
//     dL/d ln a_u = -2 lambda_u sum_{v != u} lambda_v S_uv f_uv.
// dS is never formed: each warp sweeps one row of the stored S (the matrix
// the solve already used) and forms the factors on the fly in f128, so the
// adjoint costs one pass over S after the solve. lambda comes from the
// refined solve (hp_spd_solve_refined), accurate to ~1e-30.
#include <vector>

#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
int spd_refined(const double* S, const double* b, size_t n, int mode, double tol, int max_iter, double* x,
                hp_refine_info_t* info, int64_t* pivot, cudaStream_t s);

namespace {

__device__ __forceinline__ dd warp_sum_dd(dd a) {
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    dd t;
    t.hi = __shfl_down_sync(0xffffffffu, a.hi, o);
    t.lo = __shfl_down_sync(0xffffffffu, a.lo, o);
    a = dd_add(a, t);
  }
  return a;
}

// per basis function u: gRb[u][0..2] = 4 lambda_u sum_v lambda_v p (R_u - R_v) S_uv,
//                       ga[u]       = -2 lambda_u sum_{v != u} lambda_v S_uv f_uv.
__global__ void __launch_bounds__(256) adjoint_rows_kernel(int64_t n, const double* __restrict__ centers,
                                                           const double* __restrict__ alpha,
                                                           const dd* __restrict__ S, const dd* __restrict__ lam,
                                                           dd* __restrict__ gRb, dd* __restrict__ ga) {
  const int64_t u = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const int lane = threadIdx.x % 32;
  if (u >= n) return;
  const dd a = dd_from(alpha[u]);
  const double* Ru = centers + 3 * u;
  dd accR[3] = {{0, 0}, {0, 0}, {0, 0}}, acca = {0, 0};
  for (int64_t v = lane; v < n; v += 32) {
    if (v == u) continue;
    const dd bb = dd_from(alpha[v]);
    const dd sum = dd_add(a, bb);
    const dd p = dd_div(dd_mul(a, bb), sum);
    dd d[3], r2 = {0, 0};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      d[c] = dd_sub(dd_from(Ru[c]), dd_from(centers[3 * v + c]));
      r2 = dd_add(r2, dd_mul(d[c], d[c]));
    }
    const dd w = dd_mul(lam[v], S[u * n + v]);
    const dd wp = dd_mul(w, p);
#pragma unroll
    for (int c = 0; c < 3; c++) accR[c] = dd_add(accR[c], dd_mul(wp, d[c]));
    const dd f = dd_sub(dd_div(dd_mul(dd_from(0.75), dd_sub(bb, a)), sum),
                        dd_div(dd_mul(r2, dd_mul(a, dd_mul(bb, bb))), dd_mul(sum, sum)));
    acca = dd_add(acca, dd_mul(w, f));
  }
#pragma unroll
  for (int c = 0; c < 3; c++) accR[c] = warp_sum_dd(accR[c]);
  acca = warp_sum_dd(acca);
  if (lane == 0) {
    const dd l4 = dd_mul(dd_from(4.0), lam[u]);
#pragma unroll
    for (int c = 0; c < 3; c++) gRb[3 * u + c] = dd_mul(l4, accR[c]);
    ga[u] = dd_mul(dd_from(-2.0), dd_mul(lam[u], acca));
  }
}

// grad_R[c] = sum over basis functions u of centre c (ascending u) of gRb[u]
__global__ void centre_sum_kernel(int64_t n, const int32_t* __restrict__ center_of, int64_t n_centers,
                                  const dd* __restrict__ gRb, dd* __restrict__ gR) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n_centers) return;
  const int64_t c = t / 3, comp = t % 3;
  dd s = {0, 0};
  for (int64_t u = 0; u < n; u++)
    if (center_of[u] == c) s = dd_add(s, gRb[3 * u + comp]);
  gR[t] = s;
}

// loss = b^T lambda (f128 sum of error-free products)
__global__ void loss_kernel(int64_t n, const dd* __restrict__ b, const dd* __restrict__ lam, dd* out) {
  const int lane = threadIdx.x;
  dd acc = {0, 0};
  for (int64_t i = lane; i < n; i += 32) acc = dd_add(acc, dd_mul(b[i], lam[i]));
  acc = warp_sum_dd(acc);
  if (lane == 0) *out = acc;
}

}  // namespace

int overlap_adjoint(size_t n, const double* centers, const double* alpha, const double* b2,
                    const int32_t* center_of, size_t n_centers, int mode, double* loss, double* grad_R,
                    double* grad_lnalpha, hp_refine_info_t* info, int64_t* pivot, cudaStream_t s) {
  if (n == 0) return HP_OK;
  DevBuf S(n * n * 16, s), lam(n * 16, s), gRb(3 * n * 16, s);
  if (!S.p || !lam.p || !gRb.p) return HP_ERR_CUDA;
  HP_TRY(overlap_norm_dd(n, centers, alpha, S.as<double>(), s));
  HP_TRY(spd_refined(S.as<double>(), b2, n, mode, 1e-28, 10, lam.as<double>(), info, pivot, s));
  loss_kernel<<<1, 32, 0, s>>>(n, reinterpret_cast<const dd*>(b2), lam.as<dd>(), reinterpret_cast<dd*>(loss));
  HP_LAUNCH_CHECK();
  adjoint_rows_kernel<<<(unsigned)((n + 7) / 8), 256, 0, s>>>(n, centers, alpha, S.as<dd>(), lam.as<dd>(), gRb.as<dd>(),
                                                              reinterpret_cast<dd*>(grad_lnalpha));
  HP_LAUNCH_CHECK();
  centre_sum_kernel<<<(unsigned)((3 * n_centers + 127) / 128), 128, 0, s>>>(n, center_of, n_centers, gRb.as<dd>(),
                                                                            reinterpret_cast<dd*>(grad_R));
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace hp

extern "C" {

int hp_overlap_adjoint_dev(size_t n, const double* centers, const double* alpha, const double* b,
                           const int32_t* center_of, size_t n_centers, int mode, double* loss, double* grad_R,
                           double* grad_lnalpha, hp_refine_info_t* info, void* stream) {
  if (n && (!centers || !alpha || !b || !center_of || !loss || !grad_R || !grad_lnalpha)) return HP_ERR_INVALID_ARG;
  if (mode != HP_MODE_PLAIN && mode != HP_MODE_OZAKI) return HP_ERR_INVALID_ARG;
  int64_t pivot = -1;
  return hp::overlap_adjoint(n, centers, alpha, b, center_of, n_centers, mode, loss, grad_R, grad_lnalpha, info, &pivot,
                             (cudaStream_t)stream);
}

int hp_overlap_adjoint(size_t n, const double* centers, const double* alpha, const double* b_f64,
                       const int32_t* center_of, size_t n_centers, int mode, double* loss, double* grad_R,
                       double* grad_lnalpha, hp_refine_info_t* info) {
  using namespace hp;
  if (n == 0) return HP_OK;
  if (!centers || !alpha || !b_f64 || !center_of || !loss || !grad_R || !grad_lnalpha) return HP_ERR_INVALID_ARG;
  if (mode != HP_MODE_PLAIN && mode != HP_MODE_OZAKI) return HP_ERR_INVALID_ARG;
  for (size_t u = 0; u < n; u++)
    if (center_of[u] < 0 || (size_t)center_of[u] >= n_centers) {
      set_error("center_of[%zu] out of range", u);
      return HP_ERR_INVALID_ARG;
    }
  cudaStream_t s = library_stream();
  DevBuf dc(n * 24, s), da(n * 8, s), db(n * 16, s), dco(n * 4, s), dl(16, s), dgR(n_centers * 48, s), dga(n * 16, s);
  if (!dc.p || !da.p || !db.p || !dco.p || !dl.p || !dgR.p || !dga.p) return HP_ERR_CUDA;
  std::vector<double> b2(2 * n, 0.0);
  for (size_t i = 0; i < n; i++) b2[2 * i] = b_f64[i];
  HP_CUDA_TRY(cudaMemcpyAsync(dc.p, centers, n * 24, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(da.p, alpha, n * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(db.p, b2.data(), n * 16, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dco.p, center_of, n * 4, cudaMemcpyHostToDevice, s));
  int64_t pivot = -1;
  HP_TRY(overlap_adjoint(n, dc.as<double>(), da.as<double>(), db.as<double>(), dco.as<int32_t>(), n_centers, mode,
                         dl.as<double>(), dgR.as<double>(), dga.as<double>(), info, &pivot, s));
  HP_CUDA_TRY(cudaMemcpyAsync(loss, dl.p, 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(grad_R, dgR.p, n_centers * 48, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(grad_lnalpha, dga.p, n * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

}  // extern "C"
