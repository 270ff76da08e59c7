// SPD solve to 1e-25 relative accuracy for ill-conditioned f128 matrices
// (kappa up to ~1e28): f128 Cholesky factor + iterative refinement with
// residuals accurate to ~2^-159, the procedure of crates/solver/src/lib.rs
// :75-125 with the residual precision raised from f128 to f256 so that the
// attainable error is kappa * 2^-159 instead of kappa * 2^-104.
//
// Two residual kernels:
//  * resid_qd_kernel: MultiFloat<4> arithmetic (the reference's mf_gemv,
//    crates/quad/src/multifloat/linalg.rs:17-36), each row split into 32
//    k-ordered chunks combined in order (plain mode);
//  * resid_sumk_kernel: error-free products of the f128 limbs (TwoProd)
//    accumulated by a 3-level TwoSum cascade (Ogita-Rump-Oishi SumK, K = 3),
//    warp per row (chosen mode). Both are accurate to well below 1e-40
//    relative to |S||x|.
#include <cfloat>

#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
namespace {

struct Casc3 {
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  __device__ __forceinline__ void add(double t) {
    double a, e1, e2;
    two_sum(s1, t, a, e1);
    s1 = a;
    two_sum(s2, e1, a, e2);
    s2 = a;
    s3 = __dadd_rn(s3, e2);
  }
  __device__ __forceinline__ dd result() const {  // s1 + s2 + s3 rounded to f128
    double h, l;
    two_sum(s1, s2, h, l);
    return dd_renorm(h, __dadd_rn(l, s3));
  }
};

// r = b - S x, four warps per row (each a quarter of the columns, k-ordered
// within it); the row's four partial cascades are combined in segment order
// through shared memory. Two rows per CTA.
constexpr int RS_SEG = 4;
__global__ void __launch_bounds__(256) resid_sumk_kernel(const dd* __restrict__ S, const dd* __restrict__ x,
                                                         const dd* __restrict__ b, dd* __restrict__ r, int64_t n) {
  __shared__ double part[2][RS_SEG][3];
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int rloc = w / RS_SEG, seg = w % RS_SEG;
  const int64_t row = (int64_t)blockIdx.x * 2 + rloc;
  Casc3 c;
  if (row < n) {
    if (seg == 0 && lane == 0) {
      c.add(-b[row].hi);
      c.add(-b[row].lo);
    }
    const dd* srow = S + row * n;
    const int64_t j1 = n * (seg + 1) / RS_SEG;
    for (int64_t j = n * seg / RS_SEG + lane; j < j1; j += 32) {
      const dd sv = srow[j], v = x[j];
      double p, e;
      two_prod(sv.hi, v.hi, p, e);
      c.add(p);
      c.add(e);
      two_prod(sv.hi, v.lo, p, e);
      c.add(p);
      c.add(e);
      two_prod(sv.lo, v.hi, p, e);
      c.add(p);
      c.add(e);
      c.add(__dmul_rn(sv.lo, v.lo));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      double t1 = __shfl_down_sync(0xffffffffu, c.s1, o);
      double t2 = __shfl_down_sync(0xffffffffu, c.s2, o);
      double t3 = __shfl_down_sync(0xffffffffu, c.s3, o);
      if (lane < o) {
        c.add(t1);
        c.add(t2);
        c.add(t3);
      }
    }
    if (lane == 0) {
      part[rloc][seg][0] = c.s1;
      part[rloc][seg][1] = c.s2;
      part[rloc][seg][2] = c.s3;
    }
  }
  __syncthreads();
  if (row < n && seg == 0 && lane == 0) {
    for (int q = 1; q < RS_SEG; q++) {
      c.add(part[rloc][q][0]);
      c.add(part[rloc][q][1]);
      c.add(part[rloc][q][2]);
    }
    r[row] = dd_neg(c.result());
  }
}

// r = b - S x in MultiFloat<4> arithmetic; lane k of the row's warp sums
// columns [k*n/32, (k+1)*n/32) in order, lane 0 adds the 32 partials in order.
__global__ void __launch_bounds__(64) resid_qd_kernel(const dd* __restrict__ S, const dd* __restrict__ x,
                                                      const dd* __restrict__ b, dd* __restrict__ r, int64_t n) {
  __shared__ qd part[2][32];
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int64_t row = (int64_t)blockIdx.x * 2 + w;
  if (row >= n) return;
  const int64_t j0 = n * lane / 32, j1 = n * (lane + 1) / 32;
  qd acc = qd_zero();
  const dd* srow = S + row * n;
  for (int64_t j = j0; j < j1; j++) {
    const dd s = srow[j], v = x[j];
    acc = qd_add(acc, qd_mul(qd{{s.hi, s.lo, 0.0, 0.0}}, qd{{v.hi, v.lo, 0.0, 0.0}}));
  }
  part[w][lane] = acc;
  __syncwarp();
  if (lane == 0) {
    qd tot = qd_zero();
    for (int k = 0; k < 32; k++) tot = qd_add(tot, part[w][k]);
    qd res = qd_sub(qd{{b[row].hi, b[row].lo, 0.0, 0.0}}, tot);
    r[row] = dd_renorm(res.l[0], __dadd_rn(res.l[1], res.l[2]));
  }
}

// out[0] = max |v_i.hi| (exact, order independent)
__global__ void maxabs_kernel(const dd* __restrict__ v, int64_t n, double* out) {
  __shared__ double m[256];
  double a = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 256) a = fmax(a, fabs(v[i].hi));
  m[threadIdx.x] = a;
  __syncthreads();
  for (int o = 128; o; o >>= 1) {
    if (threadIdx.x < o) m[threadIdx.x] = fmax(m[threadIdx.x], m[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = m[0];
}

// x += dx, then out[0] = max |dx_i.hi| and out[1] = max |x_i.hi| of the
// updated x (exact, order independent), in one CTA.
__global__ void __launch_bounds__(1024) update_norms_kernel(dd* __restrict__ x, const dd* __restrict__ dx, int64_t n,
                                                            double* out) {
  __shared__ double md_s[32], mx_s[32];
  double md = 0.0, mx = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const dd d = dx[i];
    const dd v = dd_add(x[i], d);
    x[i] = v;
    md = fmax(md, fabs(d.hi));
    mx = fmax(mx, fabs(v.hi));
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if (threadIdx.x % 32 == 0) {
    md_s[threadIdx.x / 32] = md;
    mx_s[threadIdx.x / 32] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x / 32); w++) {
      md = fmax(md, md_s[w]);
      mx = fmax(mx, mx_s[w]);
    }
    out[0] = md;
    out[1] = mx;
  }
}

}  // namespace

int dd_update_norms(double* x, const double* dx, size_t n, double* out_dev, cudaStream_t s) {
  if (n == 0) return HP_OK;
  update_norms_kernel<<<1, 1024, 0, s>>>(reinterpret_cast<dd*>(x), reinterpret_cast<const dd*>(dx), (int64_t)n,
                                         out_dev);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

int dd_residual(const double* S, const double* x, const double* b, double* r, size_t n, bool accurate_qd,
                cudaStream_t s) {
  if (n == 0) return HP_OK;
  if (accurate_qd)
    resid_qd_kernel<<<(unsigned)((n + 1) / 2), 64, 0, s>>>(reinterpret_cast<const dd*>(S), reinterpret_cast<const dd*>(x),
                                                            reinterpret_cast<const dd*>(b), reinterpret_cast<dd*>(r), n);
  else
    resid_sumk_kernel<<<(unsigned)((n + 1) / 2), 256, 0, s>>>(reinterpret_cast<const dd*>(S),
                                                               reinterpret_cast<const dd*>(x),
                                                               reinterpret_cast<const dd*>(b), reinterpret_cast<dd*>(r), n);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

int dd_maxabs(const double* v, size_t n, double* out_dev, cudaStream_t s) {
  maxabs_kernel<<<1, 256, 0, s>>>(reinterpret_cast<const dd*>(v), n, out_dev);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace hp

// ---------------------------------------------------------------------------
// Refined SPD solve driver (C ABI below).
// ---------------------------------------------------------------------------
namespace hp {

int spd_refined(const double* S, const double* b, size_t n, int mode, double tol, int max_iter, double* x,
                hp_refine_info_t* info, int64_t* pivot, cudaStream_t s) {
  if (n == 0) return HP_OK;
  // scal: max|dx|, max|x| (doubles 0, 1) and the factorisation's outcome
  // (chosen mode), all read back with each iteration's one synchronisation
  struct Readback {
    double dx_max, x_max;
    FactorErr ferr;
  };
  DevBuf L(n * n * 16, s), r(n * 16, s), scal(sizeof(Readback), s);
  if (!L.p || !r.p || !scal.p) return HP_ERR_CUDA;
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&e2);
  cudaEventRecord(e0, s);
  int rc;
  if (mode == HP_MODE_PLAIN) {
    HP_CUDA_TRY(cudaMemcpyAsync(L.p, S, n * n * 16, cudaMemcpyDeviceToDevice, s));
    rc = dd_cholesky(L.as<double>(), n, 0, false, pivot, nullptr, s, true);
  } else {
    // no synchronisation here: a failed pivot is reported with the first
    // readback below (the solves in between run on a partial factor)
    rc = rns_cholesky(S, L.as<double>(), n, pivot, s, &scal.as<Readback>()->ferr);
  }
  if (rc != HP_OK) return rc;
  cudaEventRecord(e1, s);
  DevBuf Xinv(dd_block_inverses_bytes(n), s);
  if (!Xinv.p) return HP_ERR_CUDA;
  HP_TRY(dd_block_inverses(L.as<double>(), n, Xinv.as<double>(), s));
  HP_CUDA_TRY(cudaMemcpyAsync(x, b, n * 16, cudaMemcpyDeviceToDevice, s));
  HP_TRY(dd_trsv_blocked(L.as<double>(), Xinv.as<double>(), x, n, false, s));
  HP_TRY(dd_trsv_blocked(L.as<double>(), Xinv.as<double>(), x, n, true, s));
  const unsigned* trsv_status = dd_trsv_status_word(Xinv.as<double>(), n);
  uint32_t* dev_status = device_status(s);  // the residue GEMMs' bounded waits
  if (!dev_status) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  // a device-side wait that gave up: clear the word, report HP_ERR_TIMEOUT
  auto timed_out = [&](unsigned trsv_bits, uint32_t dev_bits) -> bool {
    if (dev_bits) cudaMemsetAsync(dev_status, 0, sizeof(uint32_t), s);
    if ((trsv_bits | dev_bits) & DEV_STATUS_TIMEOUT) {
      set_error(trsv_bits & DEV_STATUS_TIMEOUT ? "triangular solve: a block wait timed out"
                                               : "residue GEMM: a bounded wait gave up");
      return true;
    }
    return false;
  };
  int it = 0, converged = 0;
  double ratio = 0.0;
  for (it = 1; it <= max_iter; it++) {
    HP_TRY(dd_residual(S, x, b, r.as<double>(), n, mode == HP_MODE_PLAIN, s));
    HP_TRY(dd_trsv_blocked(L.as<double>(), Xinv.as<double>(), r.as<double>(), n, false, s));
    HP_TRY(dd_trsv_blocked(L.as<double>(), Xinv.as<double>(), r.as<double>(), n, true, s));
    HP_TRY(dd_update_norms(x, r.as<double>(), n, &scal.as<Readback>()->dx_max, s));  // dx_max, x_max
    Readback h;
    unsigned st = 0;
    uint32_t ds = 0;
    HP_CUDA_TRY(cudaMemcpyAsync(&h, scal.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaMemcpyAsync(&st, trsv_status, sizeof(st), cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaMemcpyAsync(&ds, dev_status, sizeof(ds), cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    if (timed_out(st, ds)) return HP_ERR_TIMEOUT;
    if (mode != HP_MODE_PLAIN && h.ferr.flag) {
      if (pivot) *pivot = h.ferr.pivot;
      set_error("Cholesky failed at pivot %lld", (long long)h.ferr.pivot);
      return HP_ERR_NOT_SPD;
    }
    ratio = h.x_max > 0 ? h.dx_max / h.x_max : 0.0;
    if (ratio <= tol) {
      converged = 1;
      break;
    }
  }
  if (max_iter < 1) {  // no iteration read the outcomes back
    FactorErr fe;
    unsigned st = 0;
    uint32_t ds = 0;
    HP_CUDA_TRY(cudaMemcpyAsync(&fe, &scal.as<Readback>()->ferr, sizeof(fe), cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaMemcpyAsync(&st, trsv_status, sizeof(st), cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaMemcpyAsync(&ds, dev_status, sizeof(ds), cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    if (timed_out(st, ds)) return HP_ERR_TIMEOUT;
    if (mode != HP_MODE_PLAIN && fe.flag) {
      if (pivot) *pivot = fe.pivot;
      set_error("Cholesky failed at pivot %lld", (long long)fe.pivot);
      return HP_ERR_NOT_SPD;
    }
  }
  cudaEventRecord(e2, s);
  cudaEventSynchronize(e2);
  float fm = 0, tm = 0;
  cudaEventElapsedTime(&fm, e0, e1);
  cudaEventElapsedTime(&tm, e0, e2);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  if (info) {
    info->iterations = converged ? it : max_iter;
    info->converged = converged;
    info->last_correction = ratio;
    info->factor_ms = fm;
    info->total_ms = tm;
  }
  return HP_OK;
}

}  // namespace hp

extern "C" {

int hp_spd_solve_refined_dev(const double* S, const double* b, size_t n, int mode, double tol, int max_iter,
                             double* x, hp_refine_info_t* info, int64_t* pivot, void* stream) {
  if (mode != HP_MODE_PLAIN && mode != HP_MODE_OZAKI) return HP_ERR_INVALID_ARG;
  if (n && (!S || !b || !x)) return HP_ERR_INVALID_ARG;
  return hp::spd_refined(S, b, n, mode, tol, max_iter, x, info, pivot, (cudaStream_t)stream);
}

int hp_spd_solve_refined(const double* S, const double* b, size_t n, int mode, double tol, int max_iter, double* x,
                         hp_refine_info_t* info, int64_t* pivot) {
  if (mode != HP_MODE_PLAIN && mode != HP_MODE_OZAKI) return HP_ERR_INVALID_ARG;
  if (n == 0) return HP_OK;
  if (!S || !b || !x) return HP_ERR_INVALID_ARG;
  cudaStream_t s = hp::library_stream();
  hp::DevBuf dS(n * n * 16, s), db(n * 16, s), dx(n * 16, s);
  if (!dS.p || !db.p || !dx.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dS.p, S, n * n * 16, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(db.p, b, n * 16, cudaMemcpyHostToDevice, s));
  HP_TRY(hp::spd_refined(dS.as<double>(), db.as<double>(), n, mode, tol, max_iter, dx.as<double>(), info, pivot, s));
  HP_CUDA_TRY(cudaMemcpyAsync(x, dx.p, n * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

}  // extern "C"
