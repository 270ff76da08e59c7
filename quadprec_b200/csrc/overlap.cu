// Gaussian overlap-matrix assembly for s-type basis functions.
//
// overlap_s_kernel: crates/overlap/src/assemble.rs:35-85 for a basis of s
// shells: every lower-triangle shell pair is screened (screen.rs:57-101),
// contracted in f64 (integral.rs:15-25, 175-187) or f128 (integral.rs:29-56,
// 202-215) and written to both triangles of the f64 matrix; tier counts are
// accumulated. exp/log here are CUDA's, so values agree with the reference to
// the last few ulps of f64 (the reference's own f128 tier also rounds through
// an f64 exp, integral.rs:125-130).
//
// overlap_norm_dd_kernel: the f128 problem matrix of the overlap SPD
// workloads, S = (4ab/(a+b)^2)^{3/4} exp(-ab/(a+b) |R-R'|^2), evaluated with
// the reference's f128 operations only (dd.rs:61-121: sqrt, division and its
// Taylor exp), so the matrix is bit-identical to the CPU evaluation.
#include <cmath>

#include "hp_arith.cuh"
#include "hp_overlap.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
namespace {

__device__ __forceinline__ double dist2(const double* a, const double* b) {
  double dx = __dsub_rn(a[0], b[0]), dy = __dsub_rn(a[1], b[1]), dz = __dsub_rn(a[2], b[2]);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ double prim_f64(double ai, const double* ci, double aj, const double* cj) {  // integral.rs:15-25
  double gamma = __dadd_rn(ai, aj);
  double mu = __ddiv_rn(__dmul_rn(ai, aj), gamma);
  double r2 = dist2(ci, cj);
  double t = __dsqrt_rn(__ddiv_rn(3.141592653589793, gamma));
  double pref = __dmul_rn(__dmul_rn(t, t), t);
  return __dmul_rn(pref, exp(__dmul_rn(-mu, r2)));
}

__device__ dd prim_f128(double ai_, const double* ci, double aj_, const double* cj) {  // integral.rs:29-56
  dd ai = dd_from(ai_), aj = dd_from(aj_);
  dd gamma = dd_add(ai, aj);
  dd mu = dd_div(dd_mul(ai, aj), gamma);
  dd dx = dd_from(__dsub_rn(ci[0], cj[0])), dy = dd_from(__dsub_rn(ci[1], cj[1])),
     dz = dd_from(__dsub_rn(ci[2], cj[2]));
  dd r2 = dd_add(dd_add(dd_mul(dx, dx), dd_mul(dy, dy)), dd_mul(dz, dz));
  dd ratio = dd_div(dd_from(3.141592653589793), gamma);
  dd pref = dd_mul(ratio, dd_sqrt(ratio));
  dd neg_mu_r2 = dd_mul(dd_sub(dd{0.0, 0.0}, mu), r2);
  dd exp_hi = dd_from(exp(neg_mu_r2.hi));
  dd exp_val = dd_mul(exp_hi, dd_add(dd_from(1.0), dd_from(neg_mu_r2.lo)));
  return dd_mul(pref, exp_val);
}

// One thread per shell pair (i >= j), pairs enumerated row-major.
__global__ void overlap_s_kernel(int64_t nsh, const double* __restrict__ centers, const int64_t* __restrict__ poff,
                                 const double* __restrict__ alpha, const double* __restrict__ coeff, double diffuse,
                                 double ratio_thr, double neg_ln_eps, double safe_dist, double* __restrict__ S,
                                 unsigned long long* __restrict__ counts) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t npairs = nsh * (nsh + 1) / 2;
  if (p >= npairs) return;
  int64_t i = (int64_t)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while (i * (i + 1) / 2 > p) i--;
  while ((i + 1) * (i + 2) / 2 <= p) i++;
  const int64_t j = p - i * (i + 1) / 2;
  const double *ci = centers + 3 * i, *cj = centers + 3 * j;
  const int64_t a0 = poff[i], a1 = poff[i + 1], b0 = poff[j], b1 = poff[j + 1];
  // screen.rs:57-101
  double amin_a = INFINITY, amin_b = INFINITY, amax_a = 0.0, amax_b = 0.0;
  for (int64_t q = a0; q < a1; q++) {
    amin_a = fmin(amin_a, alpha[q]);
    amax_a = fmax(amax_a, alpha[q]);
  }
  for (int64_t q = b0; q < b1; q++) {
    amin_b = fmin(amin_b, alpha[q]);
    amax_b = fmax(amax_b, alpha[q]);
  }
  const double r2 = dist2(ci, cj);
  const double gam = __ddiv_rn(__dmul_rn(amin_a, amin_b), __dadd_rn(amin_a, amin_b));
  int tier;
  if (__dmul_rn(gam, r2) > neg_ln_eps) {
    tier = 2;
  } else {
    bool ad = amin_a < diffuse, bd = amin_b < diffuse;
    if (!ad && !bd) {
      tier = 0;
    } else {
      double ratio = fmax(__ddiv_rn(amax_a, amin_b), __ddiv_rn(amax_b, amin_a));
      double r = __dsqrt_rn(r2);
      if (ratio > ratio_thr && r < safe_dist)
        tier = 1;
      else if (ad && bd && r < safe_dist)
        tier = 1;
      else
        tier = 0;
    }
  }
  atomicAdd(counts + tier, 1ull);
  if (tier == 2) return;  // matrix entries stay 0 (assemble.rs:70)
  double v;
  if (tier == 0) {
    double sum = 0.0;
    for (int64_t x = a0; x < a1; x++)
      for (int64_t y = b0; y < b1; y++)
        sum = __dadd_rn(sum, __dmul_rn(__dmul_rn(coeff[x], coeff[y]), prim_f64(alpha[x], ci, alpha[y], cj)));
    v = sum;
  } else {
    dd sum = dd{0.0, 0.0};
    for (int64_t x = a0; x < a1; x++)
      for (int64_t y = b0; y < b1; y++)
        sum = dd_add(sum, dd_mul(dd_mul(dd_from(coeff[x]), dd_from(coeff[y])), prim_f128(alpha[x], ci, alpha[y], cj)));
    v = __dadd_rn(sum.hi, sum.lo);
  }
  S[i * nsh + j] = v;
  S[j * nsh + i] = v;
}

}  // namespace

namespace {
// 16 x 16 tiles on and below the diagonal; writes both triangles.
__global__ void overlap_norm_dd_kernel(int64_t n, const double* __restrict__ centers, const double* __restrict__ alpha,
                                       int64_t ld, dd* __restrict__ S) {
  int64_t idx = blockIdx.x;
  int64_t bi = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
  while (bi * (bi + 1) / 2 > idx) bi--;
  while ((bi + 1) * (bi + 2) / 2 <= idx) bi++;
  const int64_t bj = idx - bi * (bi + 1) / 2;
  const int64_t i = bi * 16 + threadIdx.y, j = bj * 16 + threadIdx.x;
  if (i >= n || j >= n || j > i) return;
  dd v = overlap_norm_pair(alpha[i], centers + 3 * i, alpha[j], centers + 3 * j);
  S[i * ld + j] = v;
  S[j * ld + i] = v;
}
}  // namespace

int overlap_norm_dd(size_t n, const double* centers, const double* alpha, double* S, cudaStream_t s) {
  if (n == 0) return HP_OK;
  const size_t tiles = (n + 15) / 16;
  overlap_norm_dd_kernel<<<(unsigned)(tiles * (tiles + 1) / 2), dim3(16, 16), 0, s>>>(n, centers, alpha, n,
                                                                                     reinterpret_cast<dd*>(S));
  HP_LAUNCH_CHECK();
  return HP_OK;
}

int overlap_s(size_t nsh, const double* centers, const int64_t* poff, const double* alpha, const double* coeff,
              const double* params, double* S, unsigned long long* counts, cudaStream_t s) {
  if (nsh == 0) return HP_OK;
  const int64_t npairs = (int64_t)(nsh * (nsh + 1) / 2);
  overlap_s_kernel<<<(unsigned)((npairs + 127) / 128), 128, 0, s>>>(
      nsh, centers, poff, alpha, coeff, params[0], params[1], -std::log(params[2]), params[3], S, counts);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace hp

extern "C" {

int hp_overlap_norm_dd(size_t n, const double* centers, const double* alpha, double* s_out) {
  if (n == 0) return HP_OK;
  if (!centers || !alpha || !s_out) return HP_ERR_INVALID_ARG;
  cudaStream_t s = hp::library_stream();
  hp::DevBuf dc(n * 24, s), da(n * 8, s), dS(n * n * 16, s);
  if (!dc.p || !da.p || !dS.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dc.p, centers, n * 24, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(da.p, alpha, n * 8, cudaMemcpyHostToDevice, s));
  HP_TRY(hp::overlap_norm_dd(n, dc.as<double>(), da.as<double>(), dS.as<double>(), s));
  HP_CUDA_TRY(cudaMemcpyAsync(s_out, dS.p, n * n * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_overlap_norm_dd_dev(size_t n, const double* centers, const double* alpha, double* s_out, void* stream) {
  if (n && (!centers || !alpha || !s_out)) return HP_ERR_INVALID_ARG;
  return hp::overlap_norm_dd(n, centers, alpha, s_out, (cudaStream_t)stream);
}

int hp_assemble_overlap_s(size_t n_shells, const double* centers, const int64_t* prim_off, const double* alpha,
                          const double* coeff, const double* params, double* matrix, int64_t* tier_counts) {
  if (n_shells == 0) return HP_OK;
  if (!centers || !prim_off || !alpha || !coeff || !params || !matrix || !tier_counts) return HP_ERR_INVALID_ARG;
  const size_t nprim = (size_t)prim_off[n_shells];
  cudaStream_t s = hp::library_stream();
  hp::DevBuf dc(n_shells * 24, s), dp((n_shells + 1) * 8, s), dal(nprim * 8 + 8, s), dco(nprim * 8 + 8, s),
      dS(n_shells * n_shells * 8, s), dcnt(3 * sizeof(unsigned long long), s);
  if (!dc.p || !dp.p || !dal.p || !dco.p || !dS.p || !dcnt.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dc.p, centers, n_shells * 24, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dp.p, prim_off, (n_shells + 1) * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dal.p, alpha, nprim * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dco.p, coeff, nprim * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemsetAsync(dS.p, 0, n_shells * n_shells * 8, s));
  HP_CUDA_TRY(cudaMemsetAsync(dcnt.p, 0, 3 * sizeof(unsigned long long), s));
  HP_TRY(hp::overlap_s(n_shells, dc.as<double>(), dp.as<int64_t>(), dal.as<double>(), dco.as<double>(), params,
                       dS.as<double>(), dcnt.as<unsigned long long>(), s));
  unsigned long long cnt[3];
  HP_CUDA_TRY(cudaMemcpyAsync(matrix, dS.p, n_shells * n_shells * 8, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(cnt, dcnt.p, sizeof(cnt), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  for (int t = 0; t < 3; t++) tier_counts[t] = (int64_t)cnt[t];
  return HP_OK;
}

}  // extern "C"
