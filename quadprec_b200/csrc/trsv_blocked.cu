// Blocked f128 triangular solves for refinement loops: L y = b and L^T x = y
// with the inverses X_k = L_kk^-1 of the 64 x 64 diagonal blocks of L
// precomputed once per factorisation:
//   forward:  y_k = X_k (b_k - sum_{j<k} L_kj y_j)
//   backward: x_k = X_k^T (y_k - sum_{j>k} L_jk^T x_j)
// One launch, one CTA per block row, no grid-wide barrier: CTAs take block
// rows in dependency order from a ticket counter; each accumulates the
// products with the solved blocks as their ready flags appear (its L tile is
// loaded before the wait), then applies X_k, stores its block and raises its
// own flag. A CTA only ever waits for CTAs that took earlier tickets, so the
// wavefront makes progress whatever the residency. Every wait is bounded
// (2 s of global time, or an abort raised by another CTA) and a CTA that
// gives up records DEV_STATUS_TIMEOUT in the status word the host reads.
// Same operations as the reference's substitutions (crates/quad/src/
// linalg.rs:99-120) grouped by blocks, in another order: f128-level accuracy,
// not bit-identical. Used where a solve is repeated (refinement), with the
// reference-order kernels in solve.cu kept for the single-solve entry points.
#include <atomic>

#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"
#include "sm100_ptx.cuh"

namespace hp {
namespace {

constexpr int TB = 64;  // block size

// X_k = L_kk^-1 for every diagonal block, one CTA (256 threads) per block.
// Xall[k] is stored row-major 64 x 64 (rows/cols beyond the last block's
// size are zero).
__global__ void __launch_bounds__(256) block_inverse_kernel(const dd* __restrict__ L, int64_t n,
                                                            dd* __restrict__ Xall) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  dd(*A)[TB + 1] = reinterpret_cast<dd(*)[TB + 1]>(sm_raw);  // [TB][TB + 1]
  dd(*X)[TB + 1] = A + TB;                                   // [TB][TB + 1]
  __shared__ dd inv[TB];
  const int t = threadIdx.x;
  const int64_t k0 = (int64_t)blockIdx.x * TB;
  const int jb = (int)min((int64_t)TB, n - k0);
  for (int q = t; q < TB * TB; q += 256) {
    const int r = q / TB, c = q % TB;
    A[r][c] = (r < jb && c <= r) ? L[(k0 + r) * n + k0 + c] : dd{0.0, 0.0};
    X[r][c] = dd_from(r == c && r < jb ? 1.0 : 0.0);
  }
  __syncthreads();
  if (t < jb) inv[t] = dd_recip(A[t][t]);
  __syncthreads();
  for (int k = 0; k < jb; k++) {  // row-oriented forward substitution, all columns at once
    for (int c = t; c <= k; c += 256) X[k][c] = dd_mul(X[k][c], inv[k]);
    __syncthreads();
    const int rows = jb - k - 1;
    for (int q = t; q < rows * (k + 1); q += 256) {
      const int i = k + 1 + q / (k + 1), c = q % (k + 1);
      X[i][c] = dd_sub(X[i][c], dd_mul(A[i][k], X[k][c]));
    }
    __syncthreads();
  }
  dd* out = Xall + (size_t)blockIdx.x * TB * TB;
  for (int q = t; q < TB * TB; q += 256) out[q] = X[q / TB][q % TB];
}

// Wavefront bookkeeping behind the inverses in the same workspace.
struct TrsvSync {
  unsigned ticket;  // next block row to hand out (reset before each launch)
  unsigned abort;   // a CTA gave up: the others stop waiting
  unsigned status;  // DEV_STATUS_* bits, read by the host
  unsigned pad;
};
inline size_t nblocks(size_t n) { return (n + TB - 1) / TB; }
inline size_t inverses_bytes(size_t n) { return nblocks(n) * TB * TB * 16; }

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ dd ld_dd_cg(const dd* p) {
  const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
  return dd{v.x, v.y};
}

// Block row k: thread (r, q) = (t / 4, t % 4) owns row r of the block and
// the columns c = q (mod 4) of each 64 x 64 tile it multiplies.
constexpr uint64_t TRSV_WAIT_NS = 2000000000ull;
template <bool UPPER_T>
__global__ void __launch_bounds__(256) trsv_wave_kernel(const dd* __restrict__ L, const dd* __restrict__ Xall,
                                                        dd* v, int64_t n, int nblk, TrsvSync* sync,
                                                        unsigned* flags, unsigned epoch) {
  __shared__ unsigned my;
  __shared__ int bad;
  __shared__ dd vj[TB], sv[TB];
  __shared__ dd part[TB][4];
  const int t = threadIdx.x, r = t / 4, q = t % 4;
  if (t == 0) {
    my = atomicAdd(&sync->ticket, 1u);
    bad = 0;
  }
  __syncthreads();
  const int s = (int)my;
  if (s >= nblk) return;
  const int k = UPPER_T ? nblk - 1 - s : s;
  const int64_t k0 = (int64_t)k * TB;
  const int jb = (int)min((int64_t)TB, n - k0);
  // X_k row r (forward) or column r (backward), loaded before any wait
  const dd* X = Xall + (size_t)k * TB * TB;
  dd xr[TB / 4];
#pragma unroll
  for (int m = 0; m < TB / 4; m++) {
    const int c = q + 4 * m;
    xr[m] = UPPER_T ? X[c * TB + r] : X[r * TB + c];
  }
  dd acc0 = {0.0, 0.0}, acc1 = {0.0, 0.0};
  for (int d = 0; d < s; d++) {
    const int j = UPPER_T ? nblk - 1 - d : d;
    const int64_t j0 = (int64_t)j * TB;
    const int jbj = (int)min((int64_t)TB, n - j0);
    dd lv[TB / 4];
#pragma unroll
    for (int m = 0; m < TB / 4; m++) {
      const int c = q + 4 * m;
      const bool in = r < jb && c < jbj;
      lv[m] = in ? (UPPER_T ? L[(j0 + c) * n + k0 + r] : L[(k0 + r) * n + j0 + c]) : dd{0.0, 0.0};
    }
    if (t == 0) {
      const uint64_t t0 = sm100::globaltimer_ns();
      while (ld_acquire_gpu(flags + j) != epoch) {
        if (ld_acquire_gpu(&sync->abort) || sm100::globaltimer_ns() - t0 > TRSV_WAIT_NS) {
          atomicOr(&sync->status, (unsigned)DEV_STATUS_TIMEOUT);
          atomicExch(&sync->abort, 1u);
          bad = 1;
          break;
        }
      }
    }
    __syncthreads();
    if (bad) return;
    if (t < TB) vj[t] = t < jbj ? ld_dd_cg(v + j0 + t) : dd{0.0, 0.0};
    __syncthreads();
#pragma unroll
    for (int m = 0; m < TB / 4; m += 2) {
      acc0 = dd_fms_fast(acc0, dd{-lv[m].hi, -lv[m].lo}, vj[q + 4 * m]);
      acc1 = dd_fms_fast(acc1, dd{-lv[m + 1].hi, -lv[m + 1].lo}, vj[q + 4 * m + 4]);
    }
    __syncthreads();  // vj is rewritten by the next dependency
  }
  part[r][q] = dd_add(acc0, acc1);
  __syncthreads();
  if (q == 0)
    sv[r] = r < jb ? dd_sub(ld_dd_cg(v + k0 + r), dd_add(dd_add(part[r][0], part[r][1]), dd_add(part[r][2], part[r][3])))
                   : dd{0.0, 0.0};
  __syncthreads();
  acc0 = acc1 = dd{0.0, 0.0};
#pragma unroll
  for (int m = 0; m < TB / 4; m += 2) {
    acc0 = dd_fms_fast(acc0, dd{-xr[m].hi, -xr[m].lo}, sv[q + 4 * m]);
    acc1 = dd_fms_fast(acc1, dd{-xr[m + 1].hi, -xr[m + 1].lo}, sv[q + 4 * m + 4]);
  }
  part[r][q] = dd_add(acc0, acc1);
  __syncthreads();
  if (q == 0 && r < jb) v[k0 + r] = dd_add(dd_add(part[r][0], part[r][1]), dd_add(part[r][2], part[r][3]));
  // the barrier orders the block's stores before thread 0's release store
  __syncthreads();
  if (t == 0) st_release_gpu(flags + k, epoch);
}

}  // namespace

int dd_block_inverses(const double* L, size_t n, double* Xall, cudaStream_t s) {
  if (n == 0) return HP_OK;
  const int smem = 2 * TB * (TB + 1) * 16;
  HP_CUDA_TRY(cudaFuncSetAttribute(block_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  block_inverse_kernel<<<(unsigned)nblocks(n), 256, smem, s>>>(reinterpret_cast<const dd*>(L), n,
                                                              reinterpret_cast<dd*>(Xall));
  HP_LAUNCH_CHECK();
  // wavefront bookkeeping: ticket, abort, status and the ready flags start at 0
  HP_CUDA_TRY(cudaMemsetAsync(reinterpret_cast<char*>(Xall) + inverses_bytes(n), 0,
                              sizeof(TrsvSync) + nblocks(n) * sizeof(unsigned), s));
  return HP_OK;
}

size_t dd_block_inverses_bytes(size_t n) {
  return inverses_bytes(n) + sizeof(TrsvSync) + (nblocks(n) * sizeof(unsigned) + 15) / 16 * 16;
}

int dd_trsv_blocked(const double* L, const double* Xall, double* v, size_t n, bool upper_t, cudaStream_t s) {
  if (n == 0) return HP_OK;
  static std::atomic<unsigned> epochs{0};
  unsigned epoch = ++epochs;
  if (epoch == 0) epoch = ++epochs;  // 0 is the flags' initial value
  char* tail = const_cast<char*>(reinterpret_cast<const char*>(Xall)) + inverses_bytes(n);
  TrsvSync* sync = reinterpret_cast<TrsvSync*>(tail);
  unsigned* flags = reinterpret_cast<unsigned*>(tail + sizeof(TrsvSync));
  HP_CUDA_TRY(cudaMemsetAsync(&sync->ticket, 0, sizeof(unsigned), s));
  const int nblk = (int)nblocks(n);
  const dd* Lp = reinterpret_cast<const dd*>(L);
  const dd* Xp = reinterpret_cast<const dd*>(Xall);
  dd* vp = reinterpret_cast<dd*>(v);
  if (upper_t)
    trsv_wave_kernel<true><<<nblk, 256, 0, s>>>(Lp, Xp, vp, (int64_t)n, nblk, sync, flags, epoch);
  else
    trsv_wave_kernel<false><<<nblk, 256, 0, s>>>(Lp, Xp, vp, (int64_t)n, nblk, sync, flags, epoch);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

int dd_trsv_status(const double* Xall, size_t n, cudaStream_t s) {
  if (n == 0) return HP_OK;
  const TrsvSync* sync = reinterpret_cast<const TrsvSync*>(reinterpret_cast<const char*>(Xall) + inverses_bytes(n));
  unsigned h = 0;
  HP_CUDA_TRY(cudaMemcpyAsync(&h, &sync->status, sizeof(h), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (h & DEV_STATUS_TIMEOUT) {
    set_error("triangular solve: a block wait timed out");
    return HP_ERR_TIMEOUT;
  }
  return HP_OK;
}

}  // namespace hp
