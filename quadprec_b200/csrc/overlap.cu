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
#include <vector>

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

// ---- Cartesian shells of any kind S, P, D, F (l = 0..3) ----
// Obara-Saika recurrence in one direction, integral.rs:156-186 (f64) and
// :188-219 (f128): S[i][j] for i <= la, j <= lb, row stride lb + 1.
__device__ void os1d_f64(int la, int lb, double pa, double pb, double gamma, double* s) {
  const int nb = lb + 1;
  const double oo2g = __ddiv_rn(0.5, gamma);
  for (int q = 0; q < (la + 1) * nb; q++) s[q] = 0.0;
  s[0] = 1.0;
  for (int i = 0; i < la; i++)
    s[(i + 1) * nb] = __dadd_rn(__dmul_rn(pa, s[i * nb]), __dmul_rn(__dmul_rn(oo2g, (double)i), i > 0 ? s[(i - 1) * nb] : 0.0));
  for (int j = 0; j < lb; j++)
    for (int i = 0; i <= la; i++) {
      const double tim1 = __dmul_rn(__dmul_rn(oo2g, (double)i), i > 0 ? s[(i - 1) * nb + j] : 0.0);
      const double tjm1 = __dmul_rn(__dmul_rn(oo2g, (double)j), j > 0 ? s[i * nb + j - 1] : 0.0);
      s[i * nb + j + 1] = __dadd_rn(__dadd_rn(__dmul_rn(pb, s[i * nb + j]), tim1), tjm1);
    }
}
__device__ void os1d_f128(int la, int lb, dd pa, dd pb, dd gamma, dd* s) {
  const int nb = lb + 1;
  const dd oo2g = dd_div(dd_from(0.5), gamma);
  for (int q = 0; q < (la + 1) * nb; q++) s[q] = dd{0.0, 0.0};
  s[0] = dd_from(1.0);
  for (int i = 0; i < la; i++) {
    const dd prev = i > 0 ? s[(i - 1) * nb] : dd{0.0, 0.0};
    s[(i + 1) * nb] = dd_add(dd_mul(pa, s[i * nb]), dd_mul(dd_mul(oo2g, dd_from((double)i)), prev));
  }
  for (int j = 0; j < lb; j++) {
    const dd fj = dd_from((double)j);
    for (int i = 0; i <= la; i++) {
      const dd fi = dd_from((double)i);
      const dd im1 = i > 0 ? s[(i - 1) * nb + j] : dd{0.0, 0.0};
      const dd jm1 = j > 0 ? s[i * nb + j - 1] : dd{0.0, 0.0};
      s[i * nb + j + 1] =
          dd_add(dd_add(dd_mul(pb, s[i * nb + j]), dd_mul(dd_mul(oo2g, fi), im1)), dd_mul(dd_mul(oo2g, fj), jm1));
    }
  }
}
// integral.rs:223-233: component k of shell kind l is (lx, ly, lz) with lx
// descending, then ly descending.
__device__ __forceinline__ void cart_component(int l, int k, int* c) {
  int idx = 0;
  for (int lx = l; lx >= 0; lx--)
    for (int ly = l - lx; ly >= 0; ly--, idx++)
      if (idx == k) c[0] = lx, c[1] = ly, c[2] = l - lx - ly;
}
__device__ __forceinline__ int n_cart(int l) { return (l + 1) * (l + 2) / 2; }

// screen.rs:57-101: 0 = F64, 1 = F128, 2 = Skip.
__device__ int screen_tier(const double* ci, const double* cj, const double* alpha, int64_t a0, int64_t a1, int64_t b0,
                           int64_t b1, double diffuse, double ratio_thr, double neg_ln_eps, double safe_dist) {
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
  if (__dmul_rn(gam, r2) > neg_ln_eps) return 2;
  const bool ad = amin_a < diffuse, bd = amin_b < diffuse;
  if (!ad && !bd) return 0;
  const double ratio = fmax(__ddiv_rn(amax_a, amin_b), __ddiv_rn(amax_b, amin_a));
  const double r = __dsqrt_rn(r2);
  if (ratio > ratio_thr && r < safe_dist) return 1;
  if (ad && bd && r < safe_dist) return 1;
  return 0;
}

// One thread per shell pair (i >= j): the block of overlap_shell_pair
// (integral.rs:66-138; s-s pairs as in overlap_s_kernel, others by the
// contracted Obara-Saika recurrence of :235-284 (f64) / :286-352 (f128)),
// written to both triangles of the n_ao x n_ao f64 matrix at the shells' AO
// offsets (assemble.rs:64-82).
__global__ void overlap_cart_kernel(int64_t nsh, const int* __restrict__ shell_l, const int64_t* __restrict__ ao_off,
                                    const double* __restrict__ centers, const int64_t* __restrict__ poff,
                                    const double* __restrict__ alpha, const double* __restrict__ coeff,
                                    double diffuse, double ratio_thr, double neg_ln_eps, double safe_dist,
                                    int64_t n_ao, double* __restrict__ S, unsigned long long* __restrict__ counts) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t npairs = nsh * (nsh + 1) / 2;
  if (p >= npairs) return;
  int64_t i = (int64_t)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while (i * (i + 1) / 2 > p) i--;
  while ((i + 1) * (i + 2) / 2 <= p) i++;
  const int64_t j = p - i * (i + 1) / 2;
  const double *ci = centers + 3 * i, *cj = centers + 3 * j;
  const int64_t a0 = poff[i], a1 = poff[i + 1], b0 = poff[j], b1 = poff[j + 1];
  const int tier = screen_tier(ci, cj, alpha, a0, a1, b0, b1, diffuse, ratio_thr, neg_ln_eps, safe_dist);
  atomicAdd(counts + tier, 1ull);
  if (tier == 2) return;  // matrix entries stay 0 (assemble.rs:70)
  const int li = shell_l[i], lj = shell_l[j], ni = n_cart(li), nj = n_cart(lj), nb = lj + 1;
  double blk[100];
  if (li == 0 && lj == 0) {
    if (tier == 0) {
      double sum = 0.0;
      for (int64_t x = a0; x < a1; x++)
        for (int64_t y = b0; y < b1; y++)
          sum = __dadd_rn(sum, __dmul_rn(__dmul_rn(coeff[x], coeff[y]), prim_f64(alpha[x], ci, alpha[y], cj)));
      blk[0] = sum;
    } else {
      dd sum = dd{0.0, 0.0};
      for (int64_t x = a0; x < a1; x++)
        for (int64_t y = b0; y < b1; y++)
          sum = dd_add(sum, dd_mul(dd_mul(dd_from(coeff[x]), dd_from(coeff[y])), prim_f128(alpha[x], ci, alpha[y], cj)));
      blk[0] = __dadd_rn(sum.hi, sum.lo);
    }
  } else if (tier == 0) {
    double sx[16], sy[16], sz[16];
    for (int q = 0; q < ni * nj; q++) blk[q] = 0.0;
    for (int64_t x = a0; x < a1; x++)
      for (int64_t y = b0; y < b1; y++) {
        const double ai = alpha[x], aj = alpha[y];
        const double gamma = __dadd_rn(ai, aj);
        const double mu = __ddiv_rn(__dmul_rn(ai, aj), gamma);
        const double r2 = dist2(ci, cj);
        const double t = __dsqrt_rn(__ddiv_rn(3.141592653589793, gamma));
        const double pref = __dmul_rn(__dmul_rn(__dmul_rn(t, t), t), exp(__dmul_rn(-mu, r2)));
        double pa[3], pb[3];
        for (int c = 0; c < 3; c++) {
          const double pc = __ddiv_rn(__dadd_rn(__dmul_rn(ai, ci[c]), __dmul_rn(aj, cj[c])), gamma);
          pa[c] = __dsub_rn(pc, ci[c]);
          pb[c] = __dsub_rn(pc, cj[c]);
        }
        os1d_f64(li, lj, pa[0], pb[0], gamma, sx);
        os1d_f64(li, lj, pa[1], pb[1], gamma, sy);
        os1d_f64(li, lj, pa[2], pb[2], gamma, sz);
        for (int u = 0; u < ni; u++) {
          int cu[3];
          cart_component(li, u, cu);
          for (int v = 0; v < nj; v++) {
            int cv[3];
            cart_component(lj, v, cv);
            const double val = __dmul_rn(
                __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(sx[cu[0] * nb + cv[0]], sy[cu[1] * nb + cv[1]]),
                                              sz[cu[2] * nb + cv[2]]),
                                    pref),
                          coeff[x]),
                coeff[y]);
            blk[u * nj + v] = __dadd_rn(blk[u * nj + v], val);
          }
        }
      }
  } else {
    dd sx[16], sy[16], sz[16], b128[100];
    for (int q = 0; q < ni * nj; q++) b128[q] = dd{0.0, 0.0};
    for (int64_t x = a0; x < a1; x++)
      for (int64_t y = b0; y < b1; y++) {
        const dd ai = dd_from(alpha[x]), aj = dd_from(alpha[y]);
        const dd gamma = dd_add(ai, aj);
        const dd mu = dd_div(dd_mul(ai, aj), gamma);
        const dd dx = dd_from(__dsub_rn(ci[0], cj[0])), dy = dd_from(__dsub_rn(ci[1], cj[1])),
                 dz = dd_from(__dsub_rn(ci[2], cj[2]));
        const dd r2 = dd_add(dd_add(dd_mul(dx, dx), dd_mul(dy, dy)), dd_mul(dz, dz));
        const dd ratio = dd_div(dd_from(3.141592653589793), gamma);
        const dd pref = dd_mul(ratio, dd_sqrt(ratio));
        const dd neg_mu_r2 = dd_mul(dd_sub(dd{0.0, 0.0}, mu), r2);
        const dd exp_val = dd_mul(dd_from(exp(neg_mu_r2.hi)), dd_add(dd_from(1.0), dd_from(neg_mu_r2.lo)));
        const dd total_pre = dd_mul(pref, exp_val);
        dd pa[3], pb[3];
        for (int c = 0; c < 3; c++) {
          const dd cic = dd_from(ci[c]), cjc = dd_from(cj[c]);
          const dd pc = dd_div(dd_add(dd_mul(ai, cic), dd_mul(aj, cjc)), gamma);
          pa[c] = dd_sub(pc, cic);
          pb[c] = dd_sub(pc, cjc);
        }
        os1d_f128(li, lj, pa[0], pb[0], gamma, sx);
        os1d_f128(li, lj, pa[1], pb[1], gamma, sy);
        os1d_f128(li, lj, pa[2], pb[2], gamma, sz);
        const dd k = dd_mul(dd_mul(dd_from(coeff[x]), dd_from(coeff[y])), total_pre);
        for (int u = 0; u < ni; u++) {
          int cu[3];
          cart_component(li, u, cu);
          for (int v = 0; v < nj; v++) {
            int cv[3];
            cart_component(lj, v, cv);
            const dd val =
                dd_mul(dd_mul(dd_mul(sx[cu[0] * nb + cv[0]], sy[cu[1] * nb + cv[1]]), sz[cu[2] * nb + cv[2]]), k);
            b128[u * nj + v] = dd_add(b128[u * nj + v], val);
          }
        }
      }
    for (int q = 0; q < ni * nj; q++) blk[q] = __dadd_rn(b128[q].hi, b128[q].lo);
  }
  const int64_t oi = ao_off[i], oj = ao_off[j];
  for (int u = 0; u < ni; u++)
    for (int v = 0; v < nj; v++) {
      S[(oi + u) * n_ao + oj + v] = blk[u * nj + v];
      if (i != j) S[(oj + v) * n_ao + oi + u] = blk[u * nj + v];
    }
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

int hp_assemble_overlap(size_t n_shells, const int32_t* shell_l, const double* centers, const int64_t* prim_off,
                        const double* alpha, const double* coeff, const double* params, double* matrix,
                        int64_t* tier_counts, size_t* n_ao_out) {
  using namespace hp;
  if (n_shells == 0) {
    if (n_ao_out) *n_ao_out = 0;
    return HP_OK;
  }
  if (!shell_l || !centers || !prim_off || !alpha || !coeff || !params || !matrix || !tier_counts) {
    set_error("null pointer");
    return HP_ERR_INVALID_ARG;
  }
  std::vector<int64_t> off(n_shells + 1, 0);
  for (size_t q = 0; q < n_shells; q++) {
    if (shell_l[q] < 0 || shell_l[q] > 3) {
      set_error("shell %zu: angular momentum %d is not one of S, P, D, F (0..3)", q, shell_l[q]);
      return HP_ERR_INVALID_ARG;
    }
    if (prim_off[q + 1] <= prim_off[q]) {
      set_error("shell %zu has no primitives", q);
      return HP_ERR_INVALID_ARG;
    }
    off[q + 1] = off[q] + (shell_l[q] + 1) * (shell_l[q] + 2) / 2;
  }
  const size_t n_ao = (size_t)off[n_shells];
  if (n_ao_out) *n_ao_out = n_ao;
  const size_t nprim = (size_t)prim_off[n_shells];
  cudaStream_t s = library_stream();
  DevBuf dl(n_shells * 4, s), doff((n_shells + 1) * 8, s), dc(n_shells * 24, s), dp((n_shells + 1) * 8, s),
      dal(nprim * 8, s), dco(nprim * 8, s), dS(n_ao * n_ao * 8, s), dcnt(3 * sizeof(unsigned long long), s);
  if (!dl.p || !doff.p || !dc.p || !dp.p || !dal.p || !dco.p || !dS.p || !dcnt.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dl.p, shell_l, n_shells * 4, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(doff.p, off.data(), (n_shells + 1) * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dc.p, centers, n_shells * 24, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dp.p, prim_off, (n_shells + 1) * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dal.p, alpha, nprim * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dco.p, coeff, nprim * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemsetAsync(dS.p, 0, n_ao * n_ao * 8, s));
  HP_CUDA_TRY(cudaMemsetAsync(dcnt.p, 0, 3 * sizeof(unsigned long long), s));
  const int64_t npairs = (int64_t)(n_shells * (n_shells + 1) / 2);
  overlap_cart_kernel<<<(unsigned)((npairs + 127) / 128), 128, 0, s>>>(
      (int64_t)n_shells, dl.as<int>(), doff.as<int64_t>(), dc.as<double>(), dp.as<int64_t>(), dal.as<double>(),
      dco.as<double>(), params[0], params[1], -std::log(params[2]), params[3], (int64_t)n_ao, dS.as<double>(),
      dcnt.as<unsigned long long>());
  HP_LAUNCH_CHECK();
  unsigned long long cnt[3];
  HP_CUDA_TRY(cudaMemcpyAsync(matrix, dS.p, n_ao * n_ao * 8, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(cnt, dcnt.p, sizeof(cnt), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  for (int t = 0; t < 3; t++) tier_counts[t] = (int64_t)cnt[t];
  return HP_OK;
}

}  // extern "C"
