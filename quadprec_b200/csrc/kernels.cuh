// Internal launchers (device pointers, stream-ordered). Each returns HP_OK or
// an HP_ERR_* code and never synchronises unless stated.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace hp {

// gemm_plain.cu
int dd_gemm_plain(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                  bool atb, cudaStream_t s);
int qd_gemm_plain(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                  bool atb, cudaStream_t s);

}  // namespace hp

namespace hp {
// ozaki.cu: exact int8-residue (Ozaki scheme II, CRT) GEMM on tcgen05.
int ozaki_dd_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                  bool atb, cudaStream_t s);
int ozaki_qd_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                  bool atb, cudaStream_t s);
}  // namespace hp

namespace hp {
// cholesky.cu: bit-identical f128 / f64 Cholesky (see file comment).
int dd_cholesky(double* a, size_t n, size_t nb, bool blocked, int64_t* pivot, double* value, cudaStream_t s,
                bool sync_status);
int f64_cholesky(double* a, size_t n, int64_t* pivot, cudaStream_t s);
// solve.cu
int dd_trsv(const double* L, double* y, size_t n, bool upper_t, cudaStream_t s);
int f64_trsv(const double* L, double* y, size_t n, bool upper_t, cudaStream_t s);
int dd_matvec(const double* A, const double* x, double* y, size_t rows, size_t cols, cudaStream_t s);
int dd_norm(const double* v, size_t n, double* out_dev, cudaStream_t s);
int cond_estimate(const double* L, size_t n, bool is_dd, double* out_dev, cudaStream_t s);
// op: 0 out=a-b, 1 out=a+b, 2 out=promote(f), 3 out(f64)=to_f64(a)
int dd_vec(int op, const double* a, const double* b, double* out, const double* f, size_t n, cudaStream_t s);
}  // namespace hp
