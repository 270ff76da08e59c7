// Blocked right-looking Cholesky on the GPU that reproduces the reference's
// factorisations bit-for-bit.
//
// reference `cholesky` (crates/quad/src/linalg.rs:42-96) and `cholesky_f64`
// (crates/solver/src/lib.rs:169-195): for each column j,
//     s_ij = sum_{k<j} L_ik L_jk  (accumulated in k order from zero),
//     L_jj = sqrt(A_jj - s_jj),  L_ij = (A_ij - s_ij) * recip(L_jj).
// Here the sums s_ij live in a separate accumulator S. Processing columns in
// blocks of nb, the trailing update adds the block's products to S in k
// order, so every s_ij sees exactly the reference's sequence of additions:
// the result does not depend on nb and equals the reference bit-for-bit.
//
// reference `cholesky_blocked` (linalg.rs:238-293, with trsm_right_lt
// :224-235): the diagonal block is factored from zero sums, the panel is
// solved by subtracting products one at a time, and the trailing block
// subtracts each block-sum from A. The BLOCKED template flag reproduces that
// arithmetic (nb is then part of the definition, as in the reference).
//
// Three kernels per block column: diag (one CTA), panel (one thread per row),
// syrk (64 x 64 lower-triangular tiles of the trailing matrix, CUDA cores).
#include <algorithm>
#include <type_traits>

#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"
#include "sm100_ptx.cuh"

namespace hp {

// Scalar traits: the same kernels run in f64 (cholesky_f64) and f128.
struct OpsF64 {
  using T = double;
  __device__ static T zero() { return 0.0; }
  __device__ static T add(T a, T b) { return __dadd_rn(a, b); }
  __device__ static T sub(T a, T b) { return __dsub_rn(a, b); }
  __device__ static T mul(T a, T b) { return __dmul_rn(a, b); }
  __device__ static T sqrt_(T a) { return __dsqrt_rn(a); }
  __device__ static T inv(T a) { return __ddiv_rn(1.0, a); }  // lib.rs:182: 1.0 / ljj
  __device__ static double hi(T a) { return a; }
  __device__ static double to_f64(T a) { return a; }
};
struct OpsDD {
  using T = dd;
  __device__ static T zero() { return dd{0.0, 0.0}; }
  __device__ static T add(T a, T b) { return dd_add(a, b); }
  __device__ static T sub(T a, T b) { return dd_sub(a, b); }
  __device__ static T mul(T a, T b) { return dd_mul(a, b); }
  __device__ static T sqrt_(T a) { return dd_sqrt(a); }
  __device__ static T inv(T a) { return dd_recip(a); }  // linalg.rs:60: ljj.recip()
  __device__ static double hi(T a) { return a.hi; }
  __device__ static double to_f64(T a) { return __dadd_rn(a.hi, a.lo); }
};

// MultiFloat<4> (f256): mf_cholesky (crates/quad/src/multifloat/linalg.rs:88-139)
// has the same per-column structure, sum = sum + l_jk l_jk,
// diag = a_jj - sum, l_jj = diag.sqrt(), l_ij = (a_ij - s) * l_jj.recip(),
// with the MultiFloat Add/Mul/sqrt/recip restated in hp_arith.cuh.
struct OpsQD {
  using T = qd;
  __device__ static T zero() { return qd_zero(); }
  __device__ static T add(T a, T b) { return qd_add(a, b); }
  __device__ static T sub(T a, T b) { return qd_sub(a, b); }
  __device__ static T mul(T a, T b) { return qd_mul(a, b); }
  __device__ static T sqrt_(T a) { return qd_sqrt(a); }
  __device__ static T inv(T a) { return qd_recip(a); }
  __device__ static double hi(T a) { return a.l[0]; }
  __device__ static double to_f64(T a) { return a.l[0]; }
};

struct CholErr {
  int flag;
  int pad;
  int64_t pivot;
  double value;
};

namespace {

constexpr int CH_MAXNB = 64;

// Diagonal block [kb, kb+jb): one CTA of 64 threads, thread t owns row kb+t.
template <class O, bool BLOCKED>
__global__ void __launch_bounds__(CH_MAXNB) chol_diag_kernel(typename O::T* A, const typename O::T* S, int64_t n,
                                                             int64_t kb, int jb, typename O::T* invd, CholErr* err) {
  using T = typename O::T;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Ls = reinterpret_cast<T*>(sm_raw);  // [64][65]
  __shared__ T inv_s[CH_MAXNB];
  __shared__ int fail;
  const int t = threadIdx.x;
  if (err->flag) return;
  if (t == 0) fail = 0;
  if (t < jb)
    for (int c = 0; c <= t; c++) Ls[t * 65 + c] = A[(kb + t) * n + kb + c];
  __syncthreads();
  for (int j = 0; j < jb; j++) {
    if (t == j) {
      T s = BLOCKED ? O::zero() : S[(kb + j) * n + kb + j];
      for (int k = 0; k < j; k++) {
        T l = Ls[j * 65 + k];
        s = O::add(s, O::mul(l, l));
      }
      T d = O::sub(Ls[j * 65 + j], s);
      if (!(O::hi(d) > 0.0) && !(O::hi(d) != O::hi(d))) {  // diag <= 0 (NaN passes, as in Rust)
        fail = 1;
        err->flag = 1;
        err->pivot = kb + j;
        err->value = O::to_f64(d);
      } else {
        T l = O::sqrt_(d);
        Ls[j * 65 + j] = l;
        inv_s[j] = O::inv(l);
      }
    }
    __syncthreads();
    if (fail) return;
    if (t > j && t < jb) {
      T s = BLOCKED ? O::zero() : S[(kb + t) * n + kb + j];
      for (int k = 0; k < j; k++) s = O::add(s, O::mul(Ls[t * 65 + k], Ls[j * 65 + k]));
      Ls[t * 65 + j] = O::mul(O::sub(Ls[t * 65 + j], s), inv_s[j]);
    }
    __syncthreads();
  }
  if (t < jb) {
    for (int c = 0; c <= t; c++) A[(kb + t) * n + kb + c] = Ls[t * 65 + c];
    invd[kb + t] = inv_s[t];
  }
}

// Panel rows i >= kb+jb, columns [kb, kb+jb): one thread per row.
template <class O, bool BLOCKED>
__global__ void __launch_bounds__(64) chol_panel_kernel(typename O::T* A, const typename O::T* S, int64_t n,
                                                        int64_t kb, int jb, const typename O::T* invd,
                                                        const CholErr* err) {
  using T = typename O::T;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Ld = reinterpret_cast<T*>(sm_raw);  // [jb][jb]
  T* Lr = Ld + jb * jb;                   // [jb][64]: this block's rows, column-major
  if (err->flag) return;
  const int t = threadIdx.x;
  for (int e = t; e < jb * jb; e += 64) {
    int r = e / jb, c = e % jb;
    Ld[e] = (c <= r) ? A[(kb + r) * n + kb + c] : O::zero();
  }
  __syncthreads();
  const int64_t i = kb + jb + (int64_t)blockIdx.x * 64 + t;
  if (i >= n) return;
  T* arow = A + i * n + kb;
  for (int j = 0; j < jb; j++) {
    T v;
    if (BLOCKED) {  // trsm_right_lt: s = b_ij; s -= b_ik l_jk; b_ij = s * recip(l_jj)
      T s = arow[j];
      for (int k = 0; k < j; k++) s = O::sub(s, O::mul(Lr[k * 64 + t], Ld[j * jb + k]));
      v = O::mul(s, invd[kb + j]);
    } else {
      T s = S[i * n + kb + j];
      for (int k = 0; k < j; k++) s = O::add(s, O::mul(Lr[k * 64 + t], Ld[j * jb + k]));
      v = O::mul(O::sub(arow[j], s), invd[kb + j]);
    }
    Lr[j * 64 + t] = v;
  }
  for (int j = 0; j < jb; j++) arow[j] = Lr[j * 64 + t];
}

// Right-looking forms of the two kernels above for the unblocked f128
// factorisation (the reference's `cholesky`). Every sum s_ij still receives
// the products L_ik L_jk one at a time in k order, starting from the value
// the trailing updates of earlier blocks left in S, so the factor is the
// same bit for bit; what changes is only when each product is added: as
// soon as column k is final, all sums of the block take their k-th product
// at once (independent operations), instead of each sum walking its k loop
// after the column it waits for.
//
// Diagonal block: one CTA, pivots on a critical warp. At step j warp 0's
// lane 0 forms L_{j+1,j} = (A - s) recip(L_jj), adds its square to the sum of
// the next diagonal entry (the k = j product, after the bulk's earlier ones),
// and forms pivot j + 1 (sqrt, recip); the bulk warps meanwhile scale the
// rest of column j and add its products to every other sum of the remaining
// lower triangle. L_{j+1,j} reaches the bulk through a named barrier that the
// critical warp passes without waiting, so the pivot chain runs while the
// bulk's updates of step j run, with one block barrier per step. Each sum
// still takes its products one at a time in k order, by the same formulas,
// so the factor is the reference's bit for bit.
constexpr int RL_THREADS = 512, RL_BULK = RL_THREADS - 32;
template <class O>
__global__ void __launch_bounds__(RL_THREADS) chol_diag_rl_kernel(typename O::T* A, const typename O::T* S, int64_t n,
                                                                  int64_t kb, int jb, typename O::T* invd,
                                                                  CholErr* err) {
  using T = typename O::T;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Ls = reinterpret_cast<T*>(sm_raw);  // [64][65]: the block, then L
  T* Ss = Ls + 64 * 65;                  // [64][65]: running sums
  __shared__ T inv_s[CH_MAXNB];
  __shared__ int fail;
  const int t = threadIdx.x, warp = t / 32, bt = t - 32;  // bt: bulk thread index (warps 1..)
  if (err->flag) return;
  if (t == 0) fail = 0;
  for (int e = t; e < jb * jb; e += RL_THREADS) {
    const int r = e / jb, c = e % jb;
    if (c <= r) {
      Ls[r * 65 + c] = A[(kb + r) * n + kb + c];
      Ss[r * 65 + c] = S[(kb + r) * n + kb + c];
    }
  }
  __syncthreads();
  // pivot p from its finished sum; false (and the error recorded) if not positive
  auto pivot = [&](int p) -> bool {
    const T d = O::sub(Ls[p * 65 + p], Ss[p * 65 + p]);
    if (!(O::hi(d) > 0.0) && !(O::hi(d) != O::hi(d))) {  // diag <= 0 (NaN passes, as in Rust)
      fail = 1;
      err->flag = 1;
      err->pivot = kb + p;
      err->value = O::to_f64(d);
      return false;
    }
    const T l = O::sqrt_(d);
    Ls[p * 65 + p] = l;
    inv_s[p] = O::inv(l);
    return true;
  };
  if (t == 0) pivot(0);
  __syncthreads();
  for (int j = 0; j < jb; j++) {
    if (fail) return;
    if (warp == 0) {
      if (t == 0 && j + 1 < jb) {
        const T l1 = O::mul(O::sub(Ls[(j + 1) * 65 + j], Ss[(j + 1) * 65 + j]), inv_s[j]);
        Ls[(j + 1) * 65 + j] = l1;
        __threadfence_block();
      }
      __syncwarp();
      sm100::named_arrive(1, RL_THREADS);  // L_{j+1,j} is in place
      if (t == 0 && j + 1 < jb) {
        const T l1 = Ls[(j + 1) * 65 + j];
        Ss[(j + 1) * 65 + j + 1] = O::add(Ss[(j + 1) * 65 + j + 1], O::mul(l1, l1));
        pivot(j + 1);
      }
    } else {
      for (int r = j + 2 + bt; r < jb; r += RL_BULK)
        Ls[r * 65 + j] = O::mul(O::sub(Ls[r * 65 + j], Ss[r * 65 + j]), inv_s[j]);
      sm100::named_sync(1, RL_THREADS);  // column j scaled (L_{j+1,j} by the critical warp)
      // sums (r, c), j < c <= r < jb, take the product L_rj L_cj, except
      // (j + 1, j + 1), which the critical warp has taken
      const int m = jb - j - 1;
      for (int e = bt + 1; e < m * (m + 1) / 2; e += RL_BULK) {
        int r = (int)((sqrtf(8.0f * e + 1.0f) - 1.0f) * 0.5f);
        while (r * (r + 1) / 2 > e) r--;
        while ((r + 1) * (r + 2) / 2 <= e) r++;
        const int c = e - r * (r + 1) / 2;
        const int rr = j + 1 + r, cc = j + 1 + c;
        Ss[rr * 65 + cc] = O::add(Ss[rr * 65 + cc],
                                  rr == cc ? O::mul(Ls[rr * 65 + j], Ls[rr * 65 + j]) : O::mul(Ls[rr * 65 + j], Ls[cc * 65 + j]));
      }
    }
    __syncthreads();
  }
  for (int e = t; e < jb * jb; e += RL_THREADS) {
    const int r = e / jb, c = e % jb;
    if (c <= r) A[(kb + r) * n + kb + c] = Ls[r * 65 + c];
  }
  if (t < jb) invd[kb + t] = inv_s[t];
}

// Panel rows i >= kb + 32 below a full 32-column diagonal block: one warp
// per row, lane q keeping the row's running sum s_iq. At step j lane j
// forms L_ij = (A_ij - s_ij) recip(L_jj) and broadcasts it; every lane
// q > j adds L_ij L_qj to its sum (the reference's product for k = j, in k
// order). A step costs one scaling and one multiply-add of latency, and
// the rows' warps fill the GPU.
constexpr int PW_ROWS = 4;  // rows (warps) per CTA
template <class O>
__global__ void __launch_bounds__(PW_ROWS * 32) chol_panel_warp_kernel(typename O::T* A, const typename O::T* S,
                                                                       int64_t n, int64_t kb,
                                                                       const typename O::T* invd,
                                                                       const CholErr* err) {
  using T = typename O::T;
  __shared__ T Ld[32][33];  // [q][j]: L_qj of the diagonal block
  __shared__ T inv_s[32];
  if (err->flag) return;
  const int t = threadIdx.x, lane = t % 32;
  for (int e = t; e < 32 * 32; e += PW_ROWS * 32) {
    const int q = e / 32, j = e % 32;
    Ld[q][j] = (j < q) ? A[(kb + q) * n + kb + j] : O::zero();
  }
  if (t < 32) inv_s[t] = invd[kb + t];
  __syncthreads();
  const int64_t i = kb + 32 + (int64_t)blockIdx.x * PW_ROWS + t / 32;
  if (i >= n) return;
  T* arow = A + i * n + kb;
  const T a = arow[lane];
  T sum = S[i * n + kb + lane], out = O::zero();
#pragma unroll 4
  for (int j = 0; j < 32; j++) {
    T v = O::zero();
    if (lane == j) {
      v = O::mul(O::sub(a, sum), inv_s[j]);
      out = v;
    }
    v.hi = __shfl_sync(0xffffffffu, v.hi, j);
    v.lo = __shfl_sync(0xffffffffu, v.lo, j);
    if (lane > j) sum = O::add(sum, O::mul(v, Ld[lane][j]));
  }
  arow[lane] = out;
}

// Trailing update on the lower triangle of rows/cols >= t0 = kb + jb:
//   unblocked semantics: S_ij = S_ij + sum_{k in block} L_ik L_jk  (k order)
//   BLOCKED:             A_ij = A_ij - (sum_{k in block} L_ik L_jk)
// (16 TT) x (16 TT) tiles, 256 threads, TT x TT entries per thread (TT = 4 for
// f64/f128, 2 for f256); the block's jb columns are staged through shared
// memory in k-slices of 16.
template <class O, bool BLOCKED, int TT>
__global__ void __launch_bounds__(256) chol_syrk_kernel(typename O::T* A, typename O::T* S, int64_t n, int64_t kb,
                                                        int jb, const CholErr* err) {
  using T = typename O::T;
  constexpr int TL = 16 * TT;
  __shared__ T Ps[16][TL + 1], Qs[16][TL + 1];
  if (err->flag) return;
  const int64_t t0 = kb + jb;
  // lower-triangular tile index -> (bi, bj), bi >= bj
  int64_t idx = blockIdx.x;
  int64_t bi = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
  while (bi * (bi + 1) / 2 > idx) bi--;
  while ((bi + 1) * (bi + 2) / 2 <= idx) bi++;
  const int64_t bj = idx - bi * (bi + 1) / 2;
  const int64_t i0 = t0 + bi * TL, j0 = t0 + bj * TL;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16, tid = threadIdx.x;
  T acc[TT][TT];
#pragma unroll
  for (int a = 0; a < TT; a++)
#pragma unroll
    for (int b = 0; b < TT; b++) {
      int64_t i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      acc[a][b] = (!BLOCKED && i < n && j < n && j <= i) ? S[i * n + j] : O::zero();
    }
  for (int k0 = 0; k0 < jb; k0 += 16) {
    __syncthreads();
    for (int e = tid; e < 16 * TL; e += 256) {
      int r = e / 16, c = e % 16;  // row r of the tile, k offset c
      int64_t gi = i0 + r, gj = j0 + r;
      bool kin = k0 + c < jb;
      Ps[c][r] = (gi < n && kin) ? A[gi * n + kb + k0 + c] : O::zero();
      Qs[c][r] = (gj < n && kin) ? A[gj * n + kb + k0 + c] : O::zero();
    }
    __syncthreads();
    const int kmax = min(16, jb - k0);
    for (int kk = 0; kk < kmax; kk++) {
      T p[TT], q[TT];
#pragma unroll
      for (int a = 0; a < TT; a++) p[a] = Ps[kk][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < TT; b++) q[b] = Qs[kk][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < TT; a++)
#pragma unroll
        for (int b = 0; b < TT; b++) acc[a][b] = O::add(acc[a][b], O::mul(p[a], q[b]));
    }
  }
#pragma unroll
  for (int a = 0; a < TT; a++)
#pragma unroll
    for (int b = 0; b < TT; b++) {
      int64_t i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      if (i < n && j < n && j <= i) {
        if (BLOCKED)
          A[i * n + j] = O::sub(A[i * n + j], acc[a][b]);
        else
          S[i * n + j] = acc[a][b];
      }
    }
}

// cholesky_f64 zeroes the strict upper triangle (lib.rs:190-192).
__global__ void zero_upper_kernel(double* L, int64_t n) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  int64_t i = idx / n, j = idx % n;
  if (j > i) L[idx] = 0.0;
}

template <class O, bool BLOCKED>
int cholesky_run(typename O::T* A, size_t n, size_t nb, CholErr* derr, cudaStream_t s) {
  using T = typename O::T;
  DevBuf Sbuf(BLOCKED ? 0 : n * n * sizeof(T), s), invd(n * sizeof(T), s);
  if ((!BLOCKED && !Sbuf.p) || !invd.p) {
    set_error("cholesky: workspace allocation failed");
    return HP_ERR_CUDA;
  }
  T* S = Sbuf.as<T>();
  if (!BLOCKED) HP_CUDA_TRY(cudaMemsetAsync(S, 0, n * n * sizeof(T), s));
  constexpr int TT = sizeof(T) > 16 ? 2 : 4;  // per-thread tile of the trailing update
  constexpr int TL = 16 * TT;
  const size_t diag_smem = 64 * 65 * sizeof(T);
  const size_t panel_max = (size_t)(nb * nb + nb * 64) * sizeof(T);
  static bool attr[64] = {}, attr_rl[64] = {};
  int dev = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 64 && !attr[dev]) {
    HP_CUDA_TRY(cudaFuncSetAttribute(chol_diag_kernel<O, BLOCKED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)diag_smem));
    HP_CUDA_TRY(cudaFuncSetAttribute(chol_panel_kernel<O, BLOCKED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)((64 * 64 + 64 * 64) * std::min(sizeof(T), (size_t)16))));
    attr[dev] = true;
  }
  if (panel_max > (64 * 64 + 64 * 64) * std::min(sizeof(T), (size_t)16)) {
    set_error("cholesky: block size %zu too large for this element type", nb);
    return HP_ERR_UNSUPPORTED;
  }
  // the right-looking kernels serve the unblocked f128 factorisation at
  // nb = RL_NB (its result does not depend on nb)
  constexpr bool RL = !BLOCKED && std::is_same<T, dd>::value;
  constexpr int RL_NB = 32;
  if constexpr (RL) nb = RL_NB;
  const size_t rl_smem = 2 * 64 * 65 * sizeof(T);
  if constexpr (RL) {
    if (dev < 64 && !attr_rl[dev]) {
      HP_CUDA_TRY(cudaFuncSetAttribute(chol_diag_rl_kernel<O>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)rl_smem));
      attr_rl[dev] = true;
    }
  }
  for (size_t kb = 0; kb < n; kb += nb) {
    const int jb = (int)std::min(nb, n - kb);
    if constexpr (RL)
      chol_diag_rl_kernel<O><<<1, RL_THREADS, rl_smem, s>>>(A, S, n, kb, jb, invd.as<T>(), derr);
    else
      chol_diag_kernel<O, BLOCKED><<<1, CH_MAXNB, diag_smem, s>>>(A, S, n, kb, jb, invd.as<T>(), derr);
    HP_LAUNCH_CHECK();
    const size_t rest = n - kb - jb;
    if (rest == 0) break;
    if constexpr (RL) {
      static_assert(RL_NB == 32, "one lane per column of the panel");
      chol_panel_warp_kernel<O><<<(unsigned)((rest + PW_ROWS - 1) / PW_ROWS), PW_ROWS * 32, 0, s>>>(A, S, n, kb,
                                                                                                  invd.as<T>(), derr);
    } else {
      const size_t panel_smem = (size_t)(jb * jb + jb * 64) * sizeof(T);
      chol_panel_kernel<O, BLOCKED><<<(unsigned)((rest + 63) / 64), 64, panel_smem, s>>>(A, S, n, kb, jb,
                                                                                        invd.as<T>(), derr);
    }
    HP_LAUNCH_CHECK();
    const size_t tiles = (rest + TL - 1) / TL;
    // small trailing matrices: half-size tiles, so that more SMs take part
    // (same per-entry operations and order, hence the same bits)
    constexpr int TTS = TT > 2 ? TT / 2 : TT;
    const size_t tiles_s = (rest + 16 * TTS - 1) / (16 * TTS);
    if (TTS != TT && tiles * (tiles + 1) / 2 < 2 * 148)
      chol_syrk_kernel<O, BLOCKED, TTS><<<(unsigned)(tiles_s * (tiles_s + 1) / 2), 256, 0, s>>>(A, S, n, kb, jb,
                                                                                                 derr);
    else
      chol_syrk_kernel<O, BLOCKED, TT><<<(unsigned)(tiles * (tiles + 1) / 2), 256, 0, s>>>(A, S, n, kb, jb, derr);
    HP_LAUNCH_CHECK();
  }
  return HP_OK;
}

}  // namespace

int dd_cholesky(double* a, size_t n, size_t nb, bool blocked, int64_t* pivot, double* value, cudaStream_t s,
                bool sync_status) {
  if (n == 0) return HP_OK;
  if (nb == 0) nb = blocked ? 64 : 32;
  if (nb > (size_t)CH_MAXNB) {
    set_error("cholesky: block size %zu exceeds %d", nb, CH_MAXNB);
    return HP_ERR_UNSUPPORTED;
  }
  DevBuf err(sizeof(CholErr), s);
  if (!err.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(CholErr), s));
  int rc = blocked ? cholesky_run<OpsDD, true>(reinterpret_cast<dd*>(a), n, nb, err.as<CholErr>(), s)
                   : cholesky_run<OpsDD, false>(reinterpret_cast<dd*>(a), n, nb, err.as<CholErr>(), s);
  if (rc != HP_OK) return rc;
  if (sync_status) {
    CholErr h;
    HP_CUDA_TRY(cudaMemcpyAsync(&h, err.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    if (h.flag) {
      if (pivot) *pivot = h.pivot;
      if (value) *value = h.value;
      set_error("Cholesky failed at pivot %lld (value=%.4e)", (long long)h.pivot, h.value);
      return HP_ERR_NOT_SPD;
    }
  }
  return HP_OK;
}

int qd_cholesky(double* a, size_t n, int64_t* pivot, cudaStream_t s) {
  if (n == 0) return HP_OK;
  DevBuf err(sizeof(CholErr), s);
  if (!err.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(CholErr), s));
  HP_TRY((cholesky_run<OpsQD, false>(reinterpret_cast<qd*>(a), n, 32, err.as<CholErr>(), s)));
  CholErr h;
  HP_CUDA_TRY(cudaMemcpyAsync(&h, err.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (h.flag) {
    if (pivot) *pivot = h.pivot;
    set_error("Cholesky failed: matrix is not positive definite (pivot %lld)", (long long)h.pivot);
    return HP_ERR_NOT_SPD;
  }
  return HP_OK;
}

int f64_cholesky(double* a, size_t n, int64_t* pivot, cudaStream_t s) {
  if (n == 0) return HP_OK;
  DevBuf err(sizeof(CholErr), s);
  if (!err.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(CholErr), s));
  HP_TRY((cholesky_run<OpsF64, false>(a, n, 32, err.as<CholErr>(), s)));
  CholErr h;
  HP_CUDA_TRY(cudaMemcpyAsync(&h, err.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (h.flag) {
    if (pivot) *pivot = h.pivot;
    set_error("f64 Cholesky failed at pivot %lld", (long long)h.pivot);
    return HP_ERR_NOT_SPD;
  }
  zero_upper_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>(a, n);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace hp
