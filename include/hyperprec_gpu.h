/*
 * hyperprec_gpu.h -- C ABI of the B200 (sm_100a) extended-precision
 * linear-algebra library (quadprec_b200/libhyperprec_gpu.so).
 *
 * Each entry point replaces one public function of hyperprec (m0at/quadprec)
 * and keeps its argument meaning; the Rust signature it replaces is cited at
 * each declaration (paths relative to the hyperprec repository).
 *
 * Data layout is the reference's in-memory layout, so a Rust caller passes
 * `slice.as_ptr() as *const f64` without conversion:
 *   f128            = { double hi; double lo; }            (16 bytes)
 *   MultiFloat<N>   = { double limbs[N]; } most significant first
 *   matrices        = row-major, dense, no leading dimension.
 *
 * Conventions
 *   - Return value: HP_OK (0) or a negative HP_ERR_* code; nothing aborts.
 *     hp_last_error() returns a thread-local message for the last failure.
 *   - Plain entry points take HOST pointers: they copy inputs to the GPU,
 *     compute on the library's stream, copy results back and return when the
 *     results are in host memory (synchronous, like the Rust functions).
 *   - *_dev entry points take DEVICE pointers and a cudaStream_t (passed as
 *     void*; NULL = legacy default stream). They are stream-ordered and
 *     return after enqueueing; status codes that depend on data (e.g. a
 *     failed Cholesky pivot) are only available from the host-pointer form,
 *     and a device-side wait that gave up is reported by hp_device_status.
 *   - Sizes of zero are valid and do nothing. NULL pointers with non-zero
 *     sizes return HP_ERR_INVALID_ARG. The Rust wrapper keeps the
 *     reference's assert_eq! length checks before calling (slices carry
 *     lengths; raw pointers do not).
 *   - No CPU fallback exists: without a usable CUDA device every compute
 *     entry point returns HP_ERR_CUDA.
 */
#ifndef HYPERPREC_GPU_H
#define HYPERPREC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define HP_OK 0
#define HP_ERR_INVALID_ARG (-1)  /* null pointer, overflow, bad mode, size limit */
#define HP_ERR_NOT_SPD (-2)      /* Cholesky pivot <= 0 (linalg.rs:54-57)          */
#define HP_ERR_NO_CONVERGE (-3)  /* iteration limit reached (linalg.rs:361)         */
#define HP_ERR_CUDA (-4)         /* CUDA runtime / launch failure, or no device    */
#define HP_ERR_TIMEOUT (-5)      /* a bounded device-side wait gave up              */
#define HP_ERR_UNSUPPORTED (-6)  /* valid request this build does not support      */

/* ---- GEMM modes ---- */
#define HP_MODE_PLAIN 0 /* CUDA-core dd/qd FMA; bit-identical to the reference */
#define HP_MODE_OZAKI 1 /* exact int8 residue split on tcgen05 tensor cores     */

/* Library / device information. */
const char* hp_last_error(void);
const char* hp_version(void);
/* 1 if a CUDA device of compute capability 10.0 is visible, else 0. */
int hp_device_ok(void);

/* Status of the stream-ordered *_dev calls (no counterpart in the
 * reference: its calls are synchronous). The tensor-core kernels behind
 * hp_f128_gemm_dev, hp_f128_gemm_atb_dev, hp_f256_gemm_dev and
 * hp_f256_gemm_atb_dev (HP_MODE_OZAKI) bound every wait and, when one gives
 * up, OR a bit into one sticky status word of the current device instead of
 * trapping. This call synchronises `stream`, stores the word in *bits (may be
 * NULL), clears it if `clear` is non-zero, and returns HP_ERR_TIMEOUT if the
 * timeout bit is set (HP_ERR_NOT_SPD / HP_ERR_CUDA for the other bits), else
 * HP_OK. Call it after a sequence of *_dev calls to learn whether any of them
 * gave up; the host-pointer entry points read and clear the word themselves. */
int hp_device_status(void* stream, uint32_t* bits, int clear);

/* Diagnostic form of the blocked wavefront triangular solve that the refined
 * SPD solvers run (no counterpart in the reference; the reference-order
 * solves are hp_f128_forward_solve / hp_f128_backward_solve). Host pointers:
 * l is n x n f128 lower triangular, b n f128, x receives L^-1 b (upper_t = 0)
 * or L^-T b (upper_t != 0) to f128 accuracy. wait_ns bounds every wait of
 * the launch (0 = the solver's 2 s). withheld_block >= 0 makes that 64-row
 * block row solve without publishing its result, so that the waits of the
 * rows after it run out: the call then returns HP_ERR_TIMEOUT with the
 * device still usable (x unspecified). -1 = normal solve. */
int hp_debug_trsv_wavefront(const double* l, const double* b, double* x, size_t n, int upper_t,
                            uint64_t wait_ns, int withheld_block);

/* Roofline denominators measured on the current device (no counterpart in
 * the reference): a DFMA loop at full occupancy (FP64 pipe, 2 flops per DFMA)
 * and a tcgen05.mma kind::i8 loop (one CTA per SM, M = 128, N = 256, K = 32
 * unsigned MMAs from shared memory into TMEM). Each runs reps + 1 times; the
 * best of the last reps is returned as fp64_tflops / i8_tops (TFLOP/s, TOP/s)
 * and its duration in ms. Any output pointer may be NULL. */
int hp_measure_peaks(int reps, double* fp64_tflops, double* i8_tops, double* fp64_ms, double* i8_ms);

/* Phase timing for benchmarks (no counterpart in the reference). While
 * enabled, the multi-kernel drivers record a CUDA event at each phase
 * boundary on their stream; hp_profile_read() waits for the last one and
 * returns up to max_phases durations in ms (phase i ends at mark i+1) and a
 * comma-separated list of phase names. Not thread-safe; off by default. */
void hp_profile_enable(int on);
int hp_profile_read(double* ms, int max_phases, char* names, size_t names_len);

/* ------------------------------------------------------------------------
 * f128 GEMM
 * replaces: pub fn gemm(a: &[f128], b: &[f128], c: &mut [f128],
 *                       m: usize, n: usize, k: usize)
 *           crates/quad/src/linalg.rs:150-165
 * C (m x n) = A (m x k) * B (k x n).
 * HP_MODE_PLAIN: each C entry is accumulated s += a*b in k order with the
 * reference's f128 Mul and Add, so C is bit-identical to the reference.
 * HP_MODE_OZAKI: normwise relative error <= 4*k*2^-104 against the same.
 * ---------------------------------------------------------------------- */
int hp_f128_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                 int mode);
/* replaces: pub fn gemm_atb(...)  crates/quad/src/linalg.rs:168-182
 * C (m x n) = A^T * B with A stored k x m. */
int hp_f128_gemm_atb(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                     int mode);
/* Device-pointer forms of the two calls above. */
int hp_f128_gemm_dev(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                     int mode, void* stream);
int hp_f128_gemm_atb_dev(const double* a, const double* b, double* c, size_t m, size_t n,
                         size_t k, int mode, void* stream);
/* Allocation-free form of hp_f128_gemm_dev in HP_MODE_OZAKI (no counterpart
 * in the reference): C = A * B on device pointers, with the whole workspace in
 * a static 64 MiB device array (about m = n = k = 768 at most; larger sizes
 * return HP_ERR_INVALID_ARG naming the bytes needed). It calls no device
 * allocator. The first call on each device does a blocking set-up, so make
 * it before any stream capture; calls that overlap in time share the scratch
 * and race, so the caller must order them. Each call waits for its stream to
 * finish the call and reads its own status word back: HP_ERR_TIMEOUT if a
 * bounded device-side wait gave up (C is then unspecified). */
int hp_f128_gemm_noalloc_dev(const double* a, const double* b, double* c, size_t m, size_t n,
                             size_t k, void* stream);

/* ------------------------------------------------------------------------
 * f256 (MultiFloat<4>) GEMM
 * replaces: pub fn mf_gemm<const N: usize>(a, b, c, m, n, k)   (N = 4)
 *           crates/quad/src/multifloat/linalg.rs:39-61
 *           pub fn mf_gemm_atb<const N: usize>(...)            (N = 4)
 *           crates/quad/src/multifloat/linalg.rs:64-85
 * HP_MODE_PLAIN is bit-identical to the reference.
 * ---------------------------------------------------------------------- */
int hp_f256_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                 int mode);
int hp_f256_gemm_atb(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                     int mode);
int hp_f256_gemm_dev(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                     int mode, void* stream);
int hp_f256_gemm_atb_dev(const double* a, const double* b, double* c, size_t m, size_t n,
                         size_t k, int mode, void* stream);

/* ------------------------------------------------------------------------
 * f512 (MultiFloat<8>) GEMM, Cholesky and solve (plain CUDA-core kernels)
 * replaces: pub fn mf_gemm<const N: usize>(a, b, c, m, n, k)      (N = 8)
 *           pub fn mf_gemm_atb<const N: usize>(a, b, c, m, n, k)  (N = 8)
 *           crates/quad/src/multifloat/linalg.rs:39-85
 * AoS f512 (8 limbs per entry); each C entry summed s = s + a b in k order
 * with the reference's MultiFloat<8> Add and Mul: bit-identical.
 * _dev: device pointers (32-byte aligned), atb != 0 for A^T B.
 * ---------------------------------------------------------------------- */
int hp_f512_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k);
int hp_f512_gemm_atb(const double* a, const double* b, double* c, size_t m, size_t n, size_t k);
int hp_f512_gemm_dev(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, int atb,
                     void* stream);
/* replaces: pub fn mf_cholesky<const N: usize>(a, n) -> Result<(), &str>  (N = 8)
 *           crates/quad/src/multifloat/linalg.rs:88-139
 * In place; the lower triangle becomes L, bit-identical; a first limb <= 0 on
 * the diagonal returns HP_ERR_NOT_SPD with *pivot (may be NULL). */
int hp_f512_cholesky(double* a, size_t n, int64_t* pivot);
/* replaces: pub fn mf_cholesky_solve<const N: usize>(l, b, x, n)  (N = 8)
 *           crates/quad/src/multifloat/linalg.rs:141-172
 * L L^T x = b; forward sweep bit-identical, backward sweep with each row's
 * subtractions in descending order (f512-level accuracy). */
int hp_f512_cholesky_solve(const double* l, const double* b, double* x, size_t n);

/* ------------------------------------------------------------------------
 * f128 Cholesky and triangular solves
 * ---------------------------------------------------------------------- */
/* replaces: pub fn cholesky(a: &mut [f128], n: usize) -> Result<(), CholeskyError>
 *           crates/quad/src/linalg.rs:42-96
 * In place: the lower triangle of a becomes L (bit-identical to the
 * reference); the strict upper triangle is left untouched. On a pivot <= 0
 * returns HP_ERR_NOT_SPD with *pivot and *value (CholeskyError{pivot,value},
 * linalg.rs:197-200; either pointer may be NULL) and a is unspecified. */
int hp_f128_cholesky(double* a, size_t n, int64_t* pivot, double* value);
/* replaces: pub fn cholesky_blocked(a: &mut [f128], n: usize, nb: usize)
 *           crates/quad/src/linalg.rs:238-293  (nb = 0 means 64; nb <= 64)
 * Bit-identical to the reference's blocked arithmetic for the same nb. */
int hp_f128_cholesky_blocked(double* a, size_t n, size_t nb, int64_t* pivot, double* value);
/* Device-pointer form of hp_f128_cholesky; synchronises `stream` to report
 * HP_ERR_NOT_SPD. */
int hp_f128_cholesky_dev(double* a, size_t n, int64_t* pivot, double* value, void* stream);
/* replaces: pub fn forward_solve(l, b, n) -> Vec<f128>   linalg.rs:99-108
 * L y = b; bit-identical. */
int hp_f128_forward_solve(const double* l, const double* b, double* y, size_t n);
/* replaces: pub fn backward_solve(l, y, n) -> Vec<f128>  linalg.rs:111-120
 * L^T x = y; normwise error within the reference's bound (summation order
 * differs, see quadprec_b200/csrc/solve.cu). */
int hp_f128_backward_solve(const double* l, const double* y, double* x, size_t n);
/* replaces: pub fn solve_cholesky(l, b, n) -> Vec<f128>  linalg.rs:123-126 */
int hp_f128_solve_cholesky(const double* l, const double* b, double* x, size_t n);
/* Device-pointer form of hp_f128_solve_cholesky: x holds b on entry and
 * L^-T L^-1 b on return (stream-ordered, the same kernels). */
int hp_f128_solve_cholesky_dev(const double* l, double* x, size_t n, void* stream);
/* replaces: pub fn matvec(a, x, n) -> Vec<f128>          linalg.rs:129-147
 * bit-identical. */
int hp_f128_matvec(const double* a, const double* x, double* y, size_t n);
/* replaces: pub fn dot(a: &[f128], b: &[f128]) -> f128   linalg.rs:7-26
 * Below 1024 entries the serial sum (bit-identical); otherwise the serial
 * sums of the 1024-entry chunks are folded left to right from zero (one
 * order of the reference's rayon reduce, bit-identical to it). out: 1 f128. */
int hp_f128_dot(const double* a, const double* b, size_t len, double* out);
/* replaces: pub fn gemv(a: &[f128], rows, cols, x: &[f128], y: &mut [f128])
 *           linalg.rs:29-38
 * y (rows) = A (rows x cols) x; each row summed in column order
 * (bit-identical). */
int hp_f128_gemv(const double* a, size_t rows, size_t cols, const double* x, double* y);
/* replaces: pub fn cond_estimate(l, n) -> f64            linalg.rs:185-194 */
int hp_f128_cond_estimate(const double* l, size_t n, double* kappa);

/* ------------------------------------------------------------------------
 * f256 (MultiFloat<4>) Cholesky and solve
 * ---------------------------------------------------------------------- */
/* replaces: pub fn mf_cholesky<const N: usize>(a, n) -> Result<(), &str>  (N = 4)
 *           crates/quad/src/multifloat/linalg.rs:88-139
 * In place on AoS f256 (4 limbs per entry): the lower triangle becomes L,
 * bit-identical to the reference; the strict upper triangle is untouched.
 * A first limb <= 0 on the diagonal returns HP_ERR_NOT_SPD with *pivot
 * (may be NULL). */
int hp_f256_cholesky(double* a, size_t n, int64_t* pivot);
/* Device-pointer form (32-byte aligned); synchronises `stream`. */
int hp_f256_cholesky_dev(double* a, size_t n, int64_t* pivot, void* stream);
/* replaces: pub fn mf_cholesky_solve<const N: usize>(l, b, x, n)  (N = 4)
 *           crates/quad/src/multifloat/linalg.rs:141-172
 * L L^T x = b. The forward sweep is bit-identical; the backward sweep
 * applies each row's subtractions in descending instead of ascending order
 * (f256-level accuracy). */
int hp_f256_cholesky_solve(const double* l, const double* b, double* x, size_t n);
/* replaces: pub fn mf_gemv<const N: usize>(a, x, y, n, m)  (N = 4)
 *           crates/quad/src/multifloat/linalg.rs:17-37
 * y (n) = A (n x m, AoS f256) x (m); bit-identical (each row summed in
 * column order). */
int hp_f256_gemv(const double* a, const double* x, double* y, size_t n, size_t m);
/* replaces: pub fn mf_dot<const N: usize>(a, b) -> MultiFloat<N>  (N = 4)
 *           crates/quad/src/multifloat/linalg.rs:7-14; bit-identical. */
int hp_f256_dot(const double* a, const double* b, size_t len, double* out);

/* ------------------------------------------------------------------------
 * SPD solver (crates/solver/src/lib.rs)
 * ---------------------------------------------------------------------- */
typedef struct {
  double kappa;          /* Solution.kappa            (lib.rs:16) */
  double residual_norm;  /* Solution.residual_norm    (lib.rs:18) */
  int32_t strategy;      /* 0 Float64, 1 MixedPrecision, 2 Float128 (lib.rs:26-30) */
  int32_t refinement_iters;
} hp_solution_t;
/* replaces: pub fn solve_spd(a_f64: &[f64], b_f64: &[f64], n) -> Result<Solution, SolveError>
 *           crates/solver/src/lib.rs:38-68
 * Same strategy selection (f64 Cholesky, kappa < 1e10, f128 refinement up
 * to 30 steps, f128 fallback). x: n f128 (Solution.x), x_f64: n doubles
 * (may be NULL). HP_ERR_NOT_SPD sets *pivot (SolveError::NotPositiveDefinite). */
int hp_solve_spd(const double* a_f64, const double* b_f64, size_t n, double* x, double* x_f64,
                 hp_solution_t* sol, int64_t* pivot);
/* replaces: pub fn solve_spd_f128(a: &[f128], b: &[f128], n)  lib.rs:71-73 */
int hp_solve_spd_f128(const double* a, const double* b, size_t n, double* x, double* x_f64,
                      hp_solution_t* sol, int64_t* pivot);

/* ------------------------------------------------------------------------
 * SPD solve to 1e-25 for ill-conditioned f128 matrices (kappa up to ~1e28)
 * extends: crates/solver/src/lib.rs:75-125 iterative_refinement. Same
 * scheme (f128 Cholesky factor, refine x += L^-T L^-1 (b - S x)), with the
 * residual evaluated to ~2^-159 instead of f128, so the attainable error is
 * kappa * 2^-159 rather than kappa * 2^-104 (the reference solver stalls at
 * ~1e-14 for kappa ~ 1e18).
 *   HP_MODE_PLAIN: the reference's f128 cholesky (bit-identical) + residual
 *                  in MultiFloat<4> arithmetic (mf_gemv semantics).
 *   HP_MODE_OZAKI: Cholesky whose trailing matrix lives in the int8 residue
 *                  domain (exact Schur updates on tcgen05), residual by
 *                  error-free products with a 3-level TwoSum cascade.
 * S: n x n f128 (symmetric, SPD; lower triangle and diagonal are read);
 * b, x: n f128. Stops when max|dx| <= tol * max|x| or after max_iter steps.
 * ---------------------------------------------------------------------- */
typedef struct {
  int32_t iterations;      /* refinement steps taken */
  int32_t converged;       /* 1 if the tol criterion was met */
  double last_correction;  /* max|dx| / max|x| of the last step */
  double factor_ms;        /* device time of the factorisation */
  double total_ms;         /* device time of factor + solves + refinement */
} hp_refine_info_t;
int hp_spd_solve_refined(const double* S, const double* b, size_t n, int mode, double tol,
                         int max_iter, double* x, hp_refine_info_t* info, int64_t* pivot);
int hp_spd_solve_refined_dev(const double* S, const double* b, size_t n, int mode, double tol,
                             int max_iter, double* x, hp_refine_info_t* info, int64_t* pivot,
                             void* stream);

/* ------------------------------------------------------------------------
 * Gaussian overlap assembly (crates/overlap)
 * ---------------------------------------------------------------------- */
/* replaces: pub fn assemble_overlap_mixed(basis: &BasisSet, params: &ScreenParams)
 *           -> OverlapResult      crates/overlap/src/assemble.rs:35-85
 * for bases of s shells (ShellKind::S, basis.rs:10-12). Shell s has centre
 * centers[3s..3s+2] and primitives prim_off[s] .. prim_off[s+1]-1 of
 * (alpha, coeff) (Primitive, basis.rs:2-6). params = {diffuse_threshold,
 * ratio_threshold, eps_skip, safe_distance} (ScreenParams, screen.rs:16-45).
 * matrix: n_shells x n_shells f64 (OverlapResult.matrix); tier_counts =
 * {f64_pairs, f128_pairs, skipped_pairs} (TierCounts, assemble.rs:16-21). */
int hp_assemble_overlap_s(size_t n_shells, const double* centers, const int64_t* prim_off,
                          const double* alpha, const double* coeff, const double* params,
                          double* matrix, int64_t* tier_counts);
/* replaces: pub fn assemble_overlap_mixed(basis: &BasisSet, params: &ScreenParams)
 *           -> OverlapResult      crates/overlap/src/assemble.rs:35-85
 * for shells of any kind: shell_l[s] = 0, 1, 2, 3 for ShellKind S, P, D, F
 * (basis.rs:9-28). Shell s contributes (l+1)(l+2)/2 Cartesian AOs in the
 * reference's order (integral.rs:223-233: lx descending, then ly
 * descending); s-s pairs as in hp_assemble_overlap_s, other pairs by the
 * contracted Obara-Saika recurrence (integral.rs:144-352) in f64 or f128 by
 * the same screening tiers. matrix: n_ao x n_ao f64 (OverlapResult.matrix);
 * *n_ao_out (may be NULL) = the AO count. Values agree with the reference to
 * the last ulps of f64 (CUDA's exp is not the host libm's). */
int hp_assemble_overlap(size_t n_shells, const int32_t* shell_l, const double* centers, const int64_t* prim_off,
                        const double* alpha, const double* coeff, const double* params, double* matrix,
                        int64_t* tier_counts, size_t* n_ao_out);
/* f128 overlap matrix of normalised s Gaussians (one primitive per basis
 * function): S_ij = (4 a b/(a+b)^2)^{3/4} exp(-a b/(a+b) |R_i - R_j|^2),
 * evaluated with the reference's f128 operations (dd.rs:61-121) so it is
 * bit-identical to the CPU evaluation; exponents below -700 give 0. This is
 * the problem matrix of the overlap SPD workloads (the reference's own
 * assembly stores f64, assemble.rs:57-58). s_out: n x n f128. */
int hp_overlap_norm_dd(size_t n, const double* centers, const double* alpha, double* s_out);
int hp_overlap_norm_dd_dev(size_t n, const double* centers, const double* alpha, double* s_out,
                           void* stream);

/* ------------------------------------------------------------------------
 * Batched uneven overlap SPD solves (no single reference counterpart: a
 * batch of the reference's assemble -> solve_spd chains, each solved to
 * 1e-25 as hp_spd_solve_refined does).
 * System s owns basis functions offsets[s] .. offsets[s+1]-1 (centres
 * 3 doubles each, exponents alpha, one normalised s Gaussian per function)
 * and b[offsets[s] ..] (f128). All systems run in ONE persistent launch: CTAs
 * pull systems from a queue ordered largest first; per system, in one CTA:
 * f128 assembly, Cholesky, solve, refinement with ~2^-159 residuals until
 * max|dx| <= tol max|x| (at most max_iter steps).
 * status[s] = HP_OK, HP_ERR_NOT_SPD or HP_ERR_NO_CONVERGE; iters[s] = steps.
 * Systems up to n = 1163 (a CTA keeps its system's Cholesky panel and
 * vectors in shared memory); a larger one returns HP_ERR_UNSUPPORTED.
 * _dev: offsets is a HOST array (count+1), everything else device memory;
 * the launch is captured in a CUDA graph on first use and replayed for
 * identical arguments. The plain form takes host arrays (b as f128).
 * Launch shape: the first call for a batch class (count rounded up to a
 * power of two, largest n rounded up to 32, per device) times every
 * candidate CTA size (256 / 512 / 1024 threads) x CTAs per SM (1..4, as
 * occupancy allows) on the batch itself and keeps the fastest for the
 * process; that call blocks until the search is done. All candidates
 * compute the same bits. HP_AUTOTUNE=0 in the environment skips the search
 * (512 threads, one CTA per SM). */
int hp_spd_solve_batched(int count, const int64_t* offsets, const double* centers,
                         const double* alpha, const double* b, double* x, int32_t* status,
                         int32_t* iters, double tol, int max_iter);
int hp_spd_solve_batched_dev(int count, const int64_t* offsets, const double* centers,
                             const double* alpha, const double* b, double* x, int32_t* status,
                             int32_t* iters, double tol, int max_iter, void* stream);
/* Launch shape (threads per CTA, CTAs per SM) of the latest batched solve in
 * this process (no reference counterpart: a report of the autotuner). */
int hp_batched_config(int32_t* threads, int32_t* ctas_per_sm);
/* Packed f128 overlap matrices of a batch (S_s at the running sum of n_t^2
 * entries, t < s); same evaluation as hp_overlap_norm_dd. offsets: host. */
int hp_overlap_norm_dd_batched_dev(int count, const int64_t* offsets, const double* centers,
                                   const double* alpha, double* S, void* stream);

/* ------------------------------------------------------------------------
 * Adjoint of overlap assembly + SPD solve (no reference counterpart: the
 * reference has no derivatives; this differentiates its assemble -> solve
 * chain). L = b^T S^-1 b with S the normalised s-Gaussian overlap matrix
 * (hp_overlap_norm_dd) of n basis functions; basis function u sits on
 * centre center_of[u] < n_centers. Returns loss (f128), grad_R
 * (n_centers x 3 f128: dL/d coordinates of each centre) and grad_lnalpha
 * (n f128: dL/d ln alpha_u). lambda = S^-1 b comes from the refined solve
 * (mode as hp_spd_solve_refined, tol 1e-28); dS is never stored: the
 * contraction sweeps the stored S and forms dS/dtheta = S dlnS/dtheta on
 * the fly. b is f64 (host form) / f128 (_dev form). */
int hp_overlap_adjoint(size_t n, const double* centers, const double* alpha, const double* b,
                       const int32_t* center_of, size_t n_centers, int mode, double* loss,
                       double* grad_R, double* grad_lnalpha, hp_refine_info_t* info);
int hp_overlap_adjoint_dev(size_t n, const double* centers, const double* alpha, const double* b,
                           const int32_t* center_of, size_t n_centers, int mode, double* loss,
                           double* grad_R, double* grad_lnalpha, hp_refine_info_t* info,
                           void* stream);

/* ------------------------------------------------------------------------
 * Jacobi eigensolver
 * replaces: pub fn jacobi_eigen(a: &[f128], n: usize, max_iter: usize)
 *           -> Result<(Vec<f128>, Vec<f128>), &'static str>
 *           crates/quad/src/linalg.rs:299-362
 * Same rotation formulas, skip and stopping rules; rotations are applied in
 * the parallel round-robin order (n/2 disjoint rotations per round) instead
 * of the sequential cyclic order, so results agree to rounding, not bits.
 * evals: n f128; evecs: n x n f128, eigenvectors as ROWS (as the reference
 * returns them). n <= 128. HP_ERR_NO_CONVERGE after max_iter sweeps. */
int hp_f128_jacobi_eigen(const double* a, size_t n, size_t max_iter, double* evals,
                         double* evecs, size_t* sweeps);
/* Batch of matrices packed back to back (matrix s is n_s x n_s with
 * n_s = n_off[s+1] - n_off[s]; n_off is a HOST array); evals packed by
 * n_off, evecs packed like A. One CTA per matrix. */
int hp_f128_jacobi_eigen_batched_dev(int count, const int64_t* n_off, const double* A,
                                     size_t max_iter, double* evals, double* evecs,
                                     int32_t* sweeps, int32_t* status, void* stream);

/* replaces: pub fn canonical_orthogonalize(s: &[f128], n: usize, threshold: f64) -> OrthoBasis
 *           crates/solver/src/ortho.rs:147-183
 * X = U diag(1 / sqrt(lambda)) over the eigenvalues with (hi + lo) > threshold,
 * ascending; x receives n x m f128 row-major (capacity n x n), *n_orth = m.
 * Eigenpairs from the GPU Jacobi solver above (the reference uses a private
 * max-pivot Jacobi): eigenvalues to f128 rounding, each column of X to
 * rounding and sign. n <= 128. */
int hp_canonical_orthogonalize(const double* s, size_t n, double threshold, double* x,
                               size_t* n_orth);
/* replaces: pub fn solve_gen_eigen(f: &[f128], s: &[f128], n: usize, threshold: f64)
 *           -> GenEigenResult          crates/solver/src/ortho.rs:185-239
 * F C = S C diag(eps) by canonical orthogonalisation: X from S as above,
 * F' = X^T F X (the reference's f128 gemm_rect / gemm_atb order, bit for bit),
 * symmetrised, diagonalised on the GPU, eigenpairs ascending. eigenvalues:
 * capacity n f128 (m used); eigenvectors: capacity n x n f128, receives C as
 * n x m row-major (column k = eigenvector k); *n_basis = m. n <= 128;
 * HP_ERR_NO_CONVERGE if a Jacobi sweep limit is reached. */
int hp_solve_gen_eigen(const double* f, const double* s, size_t n, double threshold,
                       double* eigenvalues, double* eigenvectors, size_t* n_basis);

/* ------------------------------------------------------------------------
 * Text exchange in the reference's serde formats (host only, no device)
 * replaces: impl Serialize / Deserialize for f128   crates/quad/src/dd.rs:441-514
 *           impl Serialize / Deserialize for MultiFloat<N>
 *           crates/quad/src/multifloat/traits.rs:7-155
 * Human-readable forms: f128 as format!("{:+.18e}+{:+.18e}", hi, lo), a
 * MultiFloat<N> as its limbs in "{:+.14e}" joined by '+' (Rust's exponent
 * style: "e-5", "e0"; NaN as "NaN"). The parsers split at the reference's
 * separator (a '+' followed by a sign and not preceded by 'e'/'E') and read
 * each part as Rust's f64::from_str does; anything Rust rejects returns
 * HP_ERR_INVALID_ARG. The compact forms ({hi, lo}, {limbs: [..]}) are the
 * in-memory limb layout. *_to_string write a NUL-terminated string of at
 * most cap bytes (HP_ERR_INVALID_ARG if it does not fit: 54 bytes hold any
 * f128, 24 N bytes any MultiFloat<N>).
 * ---------------------------------------------------------------------- */
int hp_f128_to_string(const double* v, char* out, size_t cap);
int hp_f128_from_string(const char* s, double* out);
int hp_mf_to_string(int n_limbs, const double* v, char* out, size_t cap);
int hp_mf_from_string(int n_limbs, const char* s, double* out);

#ifdef __cplusplus
}
#endif
#endif /* HYPERPREC_GPU_H */
