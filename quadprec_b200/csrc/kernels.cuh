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
