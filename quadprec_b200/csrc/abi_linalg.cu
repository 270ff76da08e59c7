// C ABI: f128 Cholesky, triangular solves, matvec and the SPD solver driver
// (crates/quad/src/linalg.rs, crates/solver/src/lib.rs). The solver's
// control flow (strategy choice, refinement stopping rules) runs on the host
// exactly as in lib.rs:38-144; every vector and matrix operation runs on the
// GPU.
#include <cfloat>
#include <vector>

#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
namespace {

int check_sq(size_t n, size_t limbs, size_t* bytes) {
  size_t t;
  if (mul_overflows(n, n, &t) || mul_overflows(t, 8 * limbs, bytes)) {
    set_error("matrix size overflows size_t");
    return HP_ERR_INVALID_ARG;
  }
  return HP_OK;
}

struct Stream {
  cudaStream_t s = library_stream();
};

int d2h_double(double* host, const double* dev, cudaStream_t s) {
  HP_CUDA_TRY(cudaMemcpyAsync(host, dev, sizeof(double), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int cholesky_host(double* a, size_t n, size_t nb, bool blocked, int64_t* pivot, double* value) {
  size_t bytes;
  HP_TRY(check_sq(n, 2, &bytes));
  if (n == 0) return HP_OK;
  if (!a) {
    set_error("null matrix");
    return HP_ERR_INVALID_ARG;
  }
  cudaStream_t s = library_stream();
  DevBuf da(bytes, s);
  if (!da.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, bytes, cudaMemcpyHostToDevice, s));
  HP_TRY(dd_cholesky(da.as<double>(), n, nb, blocked, pivot, value, s, true));
  HP_CUDA_TRY(cudaMemcpyAsync(a, da.p, bytes, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

// Solves with an f128 factor already on the device: x = (L L^T)^-1 b.
int solve_chol_dev(const double* dL, const double* db, double* dx, size_t n, cudaStream_t s) {
  if (dx != db) HP_CUDA_TRY(cudaMemcpyAsync(dx, db, n * 16, cudaMemcpyDeviceToDevice, s));
  HP_TRY(dd_trsv(dL, dx, n, false, s));
  return dd_trsv(dL, dx, n, true, s);
}

int trsv_host(const double* l, const double* b, double* x, size_t n, int which) {
  size_t bytes;
  HP_TRY(check_sq(n, 2, &bytes));
  if (n == 0) return HP_OK;
  if (!l || !b || !x) {
    set_error("null pointer");
    return HP_ERR_INVALID_ARG;
  }
  cudaStream_t s = library_stream();
  DevBuf dl(bytes, s), dv(n * 16, s);
  if (!dl.p || !dv.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dl.p, l, bytes, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dv.p, b, n * 16, cudaMemcpyHostToDevice, s));
  if (which == 0 || which == 2) HP_TRY(dd_trsv(dl.as<double>(), dv.as<double>(), n, false, s));
  if (which == 1 || which == 2) HP_TRY(dd_trsv(dl.as<double>(), dv.as<double>(), n, true, s));
  HP_CUDA_TRY(cudaMemcpyAsync(x, dv.p, n * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

// residual_norm_f128_from_f128 (lib.rs:237-241), everything on the device.
int residual_norm_dev(const double* dA, const double* dx, const double* db, size_t n, double* work_r,
                      double* dnorm, double* out, cudaStream_t s) {
  HP_TRY(dd_matvec(dA, dx, work_r, n, n, s));
  HP_TRY(dd_vec(0, db, work_r, work_r, nullptr, n, s));
  HP_TRY(dd_norm(work_r, n, dnorm, s));
  return d2h_double(out, dnorm, s);
}

// solve_pure_f128 (lib.rs:127-144) on device buffers dA (kept), db.
int solve_pure_f128_dev(const double* dA, const double* db, size_t n, double* x, double* x_f64,
                        hp_solution_t* sol, int64_t* pivot, cudaStream_t s) {
  DevBuf dl(n * n * 16, s), dx(n * 16, s), dr(n * 16, s), scal(2 * sizeof(double), s);
  if (!dl.p || !dx.p || !dr.p || !scal.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dl.p, dA, n * n * 16, cudaMemcpyDeviceToDevice, s));
  int rc = dd_cholesky(dl.as<double>(), n, 0, false, pivot, nullptr, s, true);
  if (rc != HP_OK) return rc;
  HP_TRY(cond_estimate(dl.as<double>(), n, true, scal.as<double>(), s));
  double kappa;
  HP_TRY(d2h_double(&kappa, scal.as<double>(), s));
  HP_TRY(solve_chol_dev(dl.as<double>(), db, dx.as<double>(), n, s));
  double rn;
  HP_TRY(residual_norm_dev(dA, dx.as<double>(), db, n, dr.as<double>(), scal.as<double>() + 1, &rn, s));
  HP_CUDA_TRY(cudaMemcpyAsync(x, dx.p, n * 16, cudaMemcpyDeviceToHost, s));
  if (x_f64) {
    HP_TRY(dd_vec(3, dx.as<double>(), nullptr, dr.as<double>(), nullptr, n, s));
    HP_CUDA_TRY(cudaMemcpyAsync(x_f64, dr.p, n * 8, cudaMemcpyDeviceToHost, s));
  }
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (sol) *sol = hp_solution_t{kappa, rn, 2, 0};
  return HP_OK;
}

}  // namespace
}  // namespace hp

extern "C" {

int hp_f128_cholesky(double* a, size_t n, int64_t* pivot, double* value) {
  return hp::cholesky_host(a, n, 0, false, pivot, value);
}
int hp_f128_cholesky_blocked(double* a, size_t n, size_t nb, int64_t* pivot, double* value) {
  return hp::cholesky_host(a, n, nb == 0 ? 64 : nb, true, pivot, value);
}
int hp_f128_cholesky_dev(double* a, size_t n, int64_t* pivot, double* value, void* stream) {
  if (n && !a) return HP_ERR_INVALID_ARG;
  return hp::dd_cholesky(a, n, 0, false, pivot, value, (cudaStream_t)stream, true);
}
int hp_f128_forward_solve(const double* l, const double* b, double* y, size_t n) {
  return hp::trsv_host(l, b, y, n, 0);
}
int hp_f128_backward_solve(const double* l, const double* y, double* x, size_t n) {
  return hp::trsv_host(l, y, x, n, 1);
}
int hp_f128_solve_cholesky(const double* l, const double* b, double* x, size_t n) {
  return hp::trsv_host(l, b, x, n, 2);
}

int hp_f128_solve_cholesky_dev(const double* l, double* x, size_t n, void* stream) {
  size_t bytes;
  HP_TRY(hp::check_sq(n, 2, &bytes));
  if (n == 0) return HP_OK;
  if (!l || !x) {
    hp::set_error("null pointer");
    return HP_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  HP_TRY(hp::dd_trsv(l, x, n, false, s));
  return hp::dd_trsv(l, x, n, true, s);
}

int hp_f128_dot(const double* a, const double* b, size_t len, double* out) {
  size_t bytes;
  if (hp::mul_overflows(len, 16, &bytes)) {
    hp::set_error("length overflows size_t");
    return HP_ERR_INVALID_ARG;
  }
  if (!out || (len && (!a || !b))) {
    hp::set_error("null pointer");
    return HP_ERR_INVALID_ARG;
  }
  if (len == 0) {
    out[0] = out[1] = 0.0;
    return HP_OK;
  }
  cudaStream_t s = hp::library_stream();
  const size_t nch = (len + 1023) / 1024;
  hp::DevBuf da(bytes, s), db(bytes, s), dp(nch * 16, s), dout(16, s);
  if (!da.p || !db.p || !dp.p || !dout.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, bytes, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(db.p, b, bytes, cudaMemcpyHostToDevice, s));
  HP_TRY(hp::dd_dot(da.as<double>(), db.as<double>(), len, dp.as<double>(), dout.as<double>(), s));
  HP_CUDA_TRY(cudaMemcpyAsync(out, dout.p, 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_f128_gemv(const double* a, size_t rows, size_t cols, const double* x, double* y) {
  size_t t, bytes;
  if (hp::mul_overflows(rows, cols, &t) || hp::mul_overflows(t, 16, &bytes) || hp::mul_overflows(cols, 16, &t)) {
    hp::set_error("matrix size overflows size_t");
    return HP_ERR_INVALID_ARG;
  }
  if (rows == 0) return HP_OK;
  if (!y || (cols && (!a || !x))) {
    hp::set_error("null pointer");
    return HP_ERR_INVALID_ARG;
  }
  cudaStream_t s = hp::library_stream();
  hp::DevBuf da(bytes, s), dx(cols * 16, s), dy(rows * 16, s);
  if ((bytes && !da.p) || (cols && !dx.p) || !dy.p) return HP_ERR_CUDA;
  if (bytes) HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, bytes, cudaMemcpyHostToDevice, s));
  if (cols) HP_CUDA_TRY(cudaMemcpyAsync(dx.p, x, cols * 16, cudaMemcpyHostToDevice, s));
  HP_TRY(hp::dd_matvec(da.as<double>(), dx.as<double>(), dy.as<double>(), rows, cols, s));
  HP_CUDA_TRY(cudaMemcpyAsync(y, dy.p, rows * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_f128_matvec(const double* a, const double* x, double* y, size_t n) {
  size_t bytes;
  HP_TRY(hp::check_sq(n, 2, &bytes));
  if (n == 0) return HP_OK;
  if (!a || !x || !y) return HP_ERR_INVALID_ARG;
  cudaStream_t s = hp::library_stream();
  hp::DevBuf da(bytes, s), dx(n * 16, s), dy(n * 16, s);
  if (!da.p || !dx.p || !dy.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, bytes, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dx.p, x, n * 16, cudaMemcpyHostToDevice, s));
  HP_TRY(hp::dd_matvec(da.as<double>(), dx.as<double>(), dy.as<double>(), n, n, s));
  HP_CUDA_TRY(cudaMemcpyAsync(y, dy.p, n * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_f128_cond_estimate(const double* l, size_t n, double* kappa) {
  size_t bytes;
  HP_TRY(hp::check_sq(n, 2, &bytes));
  if (!l || !kappa) return HP_ERR_INVALID_ARG;
  cudaStream_t s = hp::library_stream();
  hp::DevBuf dl(bytes, s), out(8, s);
  if (!dl.p || !out.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dl.p, l, bytes, cudaMemcpyHostToDevice, s));
  HP_TRY(hp::cond_estimate(dl.as<double>(), n, true, out.as<double>(), s));
  return hp::d2h_double(kappa, out.as<double>(), s);
}

int hp_solve_spd_f128(const double* a, const double* b, size_t n, double* x, double* x_f64,
                      hp_solution_t* sol, int64_t* pivot) {
  size_t bytes;
  HP_TRY(hp::check_sq(n, 2, &bytes));
  if (n == 0) return HP_OK;
  if (!a || !b || !x) return HP_ERR_INVALID_ARG;
  cudaStream_t s = hp::library_stream();
  hp::DevBuf da(bytes, s), db(n * 16, s);
  if (!da.p || !db.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, bytes, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(db.p, b, n * 16, cudaMemcpyHostToDevice, s));
  return hp::solve_pure_f128_dev(da.as<double>(), db.as<double>(), n, x, x_f64, sol, pivot, s);
}

int hp_solve_spd(const double* a_f64, const double* b_f64, size_t n, double* x, double* x_f64,
                 hp_solution_t* sol, int64_t* pivot) {
  using namespace hp;
  size_t bytes;
  HP_TRY(check_sq(n, 1, &bytes));
  if (n == 0) return HP_OK;
  if (!a_f64 || !b_f64 || !x) return HP_ERR_INVALID_ARG;
  cudaStream_t s = library_stream();
  DevBuf a64(bytes, s), b64(n * 8, s), l64(bytes, s), y64(n * 8, s);
  DevBuf a128(2 * bytes, s), b128(n * 16, s), scal(4 * sizeof(double), s);
  if (!a64.p || !b64.p || !l64.p || !y64.p || !a128.p || !b128.p || !scal.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(a64.p, a_f64, bytes, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(b64.p, b_f64, n * 8, cudaMemcpyHostToDevice, s));
  // promote_matrix (lib.rs:228-230) and b128
  HP_TRY(dd_vec(2, nullptr, nullptr, a128.as<double>(), a64.as<double>(), n * n, s));
  HP_TRY(dd_vec(2, nullptr, nullptr, b128.as<double>(), b64.as<double>(), n, s));
  // factor_and_solve_f64 (lib.rs:149-166, non-Accelerate path)
  HP_CUDA_TRY(cudaMemcpyAsync(l64.p, a64.p, bytes, cudaMemcpyDeviceToDevice, s));
  int rc = f64_cholesky(l64.as<double>(), n, nullptr, s);
  if (rc == HP_ERR_NOT_SPD) {
    return solve_pure_f128_dev(a128.as<double>(), b128.as<double>(), n, x, x_f64, sol, pivot, s);
  }
  if (rc != HP_OK) return rc;
  HP_CUDA_TRY(cudaMemcpyAsync(y64.p, b64.p, n * 8, cudaMemcpyDeviceToDevice, s));
  HP_TRY(f64_trsv(l64.as<double>(), y64.as<double>(), n, false, s));
  HP_TRY(f64_trsv(l64.as<double>(), y64.as<double>(), n, true, s));
  HP_TRY(cond_estimate(l64.as<double>(), n, false, scal.as<double>(), s));
  double kappa;
  HP_TRY(d2h_double(&kappa, scal.as<double>(), s));
  DevBuf x128(n * 16, s), r(n * 16, s), dx(n * 16, s);
  if (!x128.p || !r.p || !dx.p) return HP_ERR_CUDA;
  HP_TRY(dd_vec(2, nullptr, nullptr, x128.as<double>(), y64.as<double>(), n, s));
  if (kappa < 1e10) {  // lib.rs:48-60
    double rn;
    HP_TRY(residual_norm_dev(a128.as<double>(), x128.as<double>(), b128.as<double>(), n, r.as<double>(),
                             scal.as<double>() + 1, &rn, s));
    HP_CUDA_TRY(cudaMemcpyAsync(x, x128.p, n * 16, cudaMemcpyDeviceToHost, s));
    if (x_f64) HP_CUDA_TRY(cudaMemcpyAsync(x_f64, y64.p, n * 8, cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    if (sol) *sol = hp_solution_t{kappa, rn, 0, 0};
    return HP_OK;
  }
  // iterative_refinement (lib.rs:75-125)
  DevBuf l128(2 * bytes, s);
  if (!l128.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(l128.p, a128.p, 2 * bytes, cudaMemcpyDeviceToDevice, s));
  rc = dd_cholesky(l128.as<double>(), n, 0, false, pivot, nullptr, s, true);
  if (rc != HP_OK) return rc;
  HP_TRY(cond_estimate(l128.as<double>(), n, true, scal.as<double>(), s));
  double kappa128;
  HP_TRY(d2h_double(&kappa128, scal.as<double>(), s));
  double bnorm;
  HP_TRY(dd_norm(b128.as<double>(), n, scal.as<double>() + 1, s));
  HP_TRY(d2h_double(&bnorm, scal.as<double>() + 1, s));
  double best = DBL_MAX;
  int iters = 0;
  for (int it = 0; it < 30; it++) {
    HP_TRY(dd_matvec(a128.as<double>(), x128.as<double>(), r.as<double>(), n, n, s));
    HP_TRY(dd_vec(0, b128.as<double>(), r.as<double>(), r.as<double>(), nullptr, n, s));
    double rnorm;
    HP_TRY(dd_norm(r.as<double>(), n, scal.as<double>() + 2, s));
    HP_TRY(d2h_double(&rnorm, scal.as<double>() + 2, s));
    iters++;
    if (rnorm < 1e-28 * bnorm) break;
    if (iters > 3 && rnorm > 0.5 * best) break;
    if (rnorm < best) best = rnorm;
    HP_TRY(solve_chol_dev(l128.as<double>(), r.as<double>(), dx.as<double>(), n, s));
    HP_TRY(dd_vec(1, x128.as<double>(), dx.as<double>(), x128.as<double>(), nullptr, n, s));
  }
  double rn;
  HP_TRY(residual_norm_dev(a128.as<double>(), x128.as<double>(), b128.as<double>(), n, r.as<double>(),
                           scal.as<double>() + 3, &rn, s));
  HP_CUDA_TRY(cudaMemcpyAsync(x, x128.p, n * 16, cudaMemcpyDeviceToHost, s));
  if (x_f64) {
    HP_TRY(dd_vec(3, x128.as<double>(), nullptr, r.as<double>(), nullptr, n, s));
    HP_CUDA_TRY(cudaMemcpyAsync(x_f64, r.p, n * 8, cudaMemcpyDeviceToHost, s));
  }
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (sol) *sol = hp_solution_t{kappa128, rn, 1, iters};
  return HP_OK;
}

}  // extern "C"
