// C ABI for the f128 / f256 GEMM entry points (include/hyperprec_gpu.h).
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
namespace {

int check_args(const void* a, const void* b, const void* c, size_t m, size_t n, size_t k,
               int mode, size_t limbs, size_t* bytes_a, size_t* bytes_b, size_t* bytes_c) {
  if (mode != HP_MODE_PLAIN && mode != HP_MODE_OZAKI) {
    set_error("unknown mode %d", mode);
    return HP_ERR_INVALID_ARG;
  }
  size_t t;
  if (mul_overflows(m, k, &t) || mul_overflows(t, 8 * limbs, bytes_a) || mul_overflows(k, n, &t) ||
      mul_overflows(t, 8 * limbs, bytes_b) || mul_overflows(m, n, &t) ||
      mul_overflows(t, 8 * limbs, bytes_c)) {
    set_error("matrix size overflows size_t");
    return HP_ERR_INVALID_ARG;
  }
  if ((*bytes_a && !a) || (*bytes_b && !b) || (*bytes_c && !c)) {
    set_error("null pointer with non-zero size");
    return HP_ERR_INVALID_ARG;
  }
  return HP_OK;
}

int gemm_dev(int limbs, const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
             bool atb, int mode, cudaStream_t s) {
  size_t ba, bb, bc;
  HP_TRY(check_args(a, b, c, m, n, k, mode, limbs, &ba, &bb, &bc));
  size_t align = limbs == 2 ? 16 : 32;
  if (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c) % align) {
    set_error("device pointers must be %zu-byte aligned", align);
    return HP_ERR_INVALID_ARG;
  }
  if (mode == HP_MODE_OZAKI) {
    if (limbs == 2) return ozaki_dd_gemm(a, b, c, m, n, k, atb, s);
    return ozaki_qd_gemm(a, b, c, m, n, k, atb, s);
  }
  return limbs == 2 ? dd_gemm_plain(a, b, c, m, n, k, atb, s) : qd_gemm_plain(a, b, c, m, n, k, atb, s);
}

int gemm_host(int limbs, const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
              bool atb, int mode) {
  size_t ba, bb, bc;
  HP_TRY(check_args(a, b, c, m, n, k, mode, limbs, &ba, &bb, &bc));
  if (bc == 0) return HP_OK;
  // chosen f128 op(A) B with enough rows to split: op(A) in row panels and B
  // in column panels, the blocks' kernels and copies back overlapping the
  // remaining copies
  if (limbs == 2 && mode == HP_MODE_OZAKI && m >= 512 && k > 0) return ozaki_dd_gemm_host(a, b, c, m, n, k, atb);
  if (limbs == 4 && mode == HP_MODE_OZAKI && m >= 512 && k > 0) return ozaki_qd_gemm_host(a, b, c, m, n, k, atb);
  cudaStream_t s = library_stream();
  DevBuf da(ba, s), db(bb, s), dc(bc, s);
  if ((ba && !da.p) || (bb && !db.p) || !dc.p) {
    set_error("device allocation of %zu bytes failed", ba + bb + bc);
    return HP_ERR_CUDA;
  }
  HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, ba, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(db.p, b, bb, cudaMemcpyHostToDevice, s));
  HP_TRY(gemm_dev(limbs, da.as<double>(), db.as<double>(), dc.as<double>(), m, n, k, atb, mode, s));
  HP_CUDA_TRY(cudaMemcpyAsync(c, dc.p, bc, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  // the tensor-core path's bounded waits report through the device status word
  if (mode == HP_MODE_OZAKI) HP_TRY(consume_device_status(s));
  return HP_OK;
}

}  // namespace
}  // namespace hp

extern "C" {

int hp_f128_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, int mode) {
  return hp::gemm_host(2, a, b, c, m, n, k, false, mode);
}
int hp_f128_gemm_atb(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                     int mode) {
  return hp::gemm_host(2, a, b, c, m, n, k, true, mode);
}
int hp_f128_gemm_dev(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                     int mode, void* stream) {
  return hp::gemm_dev(2, a, b, c, m, n, k, false, mode, (cudaStream_t)stream);
}
int hp_f128_gemm_atb_dev(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                         int mode, void* stream) {
  return hp::gemm_dev(2, a, b, c, m, n, k, true, mode, (cudaStream_t)stream);
}
int hp_f256_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, int mode) {
  return hp::gemm_host(4, a, b, c, m, n, k, false, mode);
}
int hp_f256_gemm_atb(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                     int mode) {
  return hp::gemm_host(4, a, b, c, m, n, k, true, mode);
}
int hp_f256_gemm_dev(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                     int mode, void* stream) {
  return hp::gemm_dev(4, a, b, c, m, n, k, false, mode, (cudaStream_t)stream);
}
int hp_f256_gemm_atb_dev(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                         int mode, void* stream) {
  return hp::gemm_dev(4, a, b, c, m, n, k, true, mode, (cudaStream_t)stream);
}

}  // extern "C"
