// Internal launchers (device pointers, stream-ordered). Each returns HP_OK or
// an HP_ERR_* code and never synchronises unless stated.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

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
// Host pointers, C = A B: copies overlapped with the panels' kernels (bit-
// identical to ozaki_dd_gemm); synchronous.
int ozaki_dd_gemm_host(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, bool atb);
int ozaki_qd_gemm_host(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, bool atb);
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
// part: ceil(len / 1024) f128 of workspace; out: one f128 (device).
int dd_dot(const double* a, const double* b, size_t len, double* part, double* out, cudaStream_t s);
int dd_norm(const double* v, size_t n, double* out_dev, cudaStream_t s);
int cond_estimate(const double* L, size_t n, bool is_dd, double* out_dev, cudaStream_t s);
// op: 0 out=a-b, 1 out=a+b, 2 out=promote(f), 3 out(f64)=to_f64(a)
int dd_vec(int op, const double* a, const double* b, double* out, const double* f, size_t n, cudaStream_t s);
}  // namespace hp

namespace hp {
// overlap.cu
int overlap_norm_dd(size_t n, const double* centers, const double* alpha, double* S, cudaStream_t s);
}  // namespace hp

namespace hp {
// ozaki.cu: int8 residue GEMM core. cres[l][c_row0 + i][c_col0 + j] is set /
// incremented / decremented (acc_mode 0 / 1 / 2) by (A_l B_l^T)_ij mod m_l
// for i < Mp, j < Np (tile extents, multiples of 128 / 256). ares / bres hold
// ra_rows / rb_rows rows of Kp bytes per modulus.
int ozaki_residue_gemm(const int8_t* ares, const int8_t* bres, uint8_t* cres, int L, size_t Mp, size_t Np,
                       size_t Kp, cudaStream_t s);
int ozaki_residue_gemm_ex(const int8_t* ares, const int8_t* bres, uint8_t* cres, int L, size_t Mp, size_t Np,
                          size_t Kp, size_t ldc, size_t plane, size_t c_row0, size_t c_col0, int acc_mode,
                          cudaStream_t s, size_t ra_rows, size_t rb_rows);
// pdl: launch the GEMM as a programmatic dependent launch of the preceding
// kernel in s (which it waits for before reading the residues). u8: the
// residues are unsigned bytes in [0, m) (else balanced signed bytes).
int ozaki_residue_gemm_k(const int8_t* ares, const int8_t* bres, uint8_t* cres, int L, size_t Mp, size_t Np,
                         size_t ka, size_t kb_len_b, size_t a_k0, size_t k_len, size_t b_k0, size_t ldc,
                         size_t plane, size_t c_row0, size_t c_col0, int acc_mode, cudaStream_t s, size_t ra_rows,
                         size_t rb_rows, bool pdl = false, bool u8 = false);
int ozaki_moduli_for(size_t k, int beta);
// refine.cu
int dd_residual(const double* S, const double* x, const double* b, double* r, size_t n, bool accurate_qd,
                cudaStream_t s);
int dd_maxabs(const double* v, size_t n, double* out_dev, cudaStream_t s);
// x += dx; out_dev[0] = max |dx.hi|, out_dev[1] = max |x.hi| (updated x).
int dd_update_norms(double* x, const double* dx, size_t n, double* out_dev, cudaStream_t s);
// Outcome of a device-side factorisation: flag != 0 when a pivot was not
// positive, pivot = the first such index.
struct FactorErr {
  int flag;
  int pad;
  long long pivot;
};
// ozaki.cu: Cholesky with the trailing matrix kept in the residue domain.
// Writes the lower triangle of L (the strict upper triangle is not touched).
// With err_out == nullptr it synchronises s and returns HP_ERR_NOT_SPD with
// *pivot on failure; otherwise it copies the outcome to the device word
// err_out on s and returns without synchronising.
int rns_cholesky(const double* S, double* L, size_t n, int64_t* pivot, cudaStream_t s,
                 FactorErr* err_out = nullptr);
}  // namespace hp

namespace hp {
// trsv_blocked.cu: solves with precomputed inverses of the 64 x 64 diagonal blocks.
int dd_block_inverses(const double* L, size_t n, double* Xall, cudaStream_t s);
size_t dd_block_inverses_bytes(size_t n);
// Every wait of the solve gives up after wait_ns of global time (then the
// launch records DEV_STATUS_TIMEOUT); withheld >= 0 is the diagnostic hook of
// hp_debug_trsv_wavefront (that ticket's block is solved but not published).
constexpr uint64_t TRSV_WAIT_NS = 2000000000ull;
int dd_trsv_blocked(const double* L, const double* Xall, double* v, size_t n, bool upper_t, cudaStream_t s,
                    uint64_t wait_ns = TRSV_WAIT_NS, int withheld = -1);
// Device address of the status word of the solves on Xall (DEV_STATUS_TIMEOUT
// once a wavefront wait gave up).
const unsigned* dd_trsv_status_word(const double* Xall, size_t n);
}  // namespace hp

namespace hp {
// batched.cu: the persistent batched solver and its launch configurations
// (threads per CTA, CTAs per SM); all configurations give the same bits.
struct BatchedConfig {
  int threads;
  int ctas_per_sm;
};
std::vector<BatchedConfig> batched_spd_candidates(int nmax);  // launch shapes that fit with n <= nmax
int batched_spd_prepare(int nmax);  // shared-memory limit for systems up to nmax (call outside a capture)
int batched_spd_grid(const BatchedConfig& cfg);
size_t batched_spd_work_bytes(int grid, int nmax);
int batched_spd(int count, const int* order, const int64_t* off, const double* centers, const double* alpha,
                const double* b, double* x, int* status, int* iters, int nmax, double tol, int max_iter,
                cudaStream_t s, const BatchedConfig& cfg);
int batched_spd_launch(int count, const int* order, const int64_t* off, const double* centers, const double* alpha,
                       const double* b, double* x, int* status, int* iters, int nmax, double tol, int max_iter,
                       void* work, int* queue, const BatchedConfig& cfg, cudaStream_t s);
// order (device, optional): matrices largest first; the first count_big
// (n > JACOBI_SMALL_N) run in one launch, the rest (n <= nmax_small) in a
// second one with less shared memory per CTA.
constexpr int JACOBI_SMALL_N = 80;
int batched_jacobi(int count, const int64_t* n_off, const int64_t* mat_off, const double* A, double* evals,
                   double* evecs, int* sweeps, int* status, int nmax, int max_sweeps, cudaStream_t s,
                   const int* order = nullptr, int count_big = -1, int nmax_small = 0);
int batched_assemble(int count, const int64_t* off, const double* centers, const double* alpha,
                     const int64_t* mat_off, double* S, cudaStream_t s);
}  // namespace hp
