// Blocked f128 triangular solves for refinement loops: L y = b and L^T x = y
// with the inverses of the 64 x 64 diagonal blocks of L precomputed once per
// factorisation. One cooperative launch sweeps the block columns:
//   forward:  y_k = X_k (b_k - sum_{j<k} L_kj y_j)     (X_k = L_kk^-1)
//   backward: x_k = X_k^T (y_k - sum_{j>k} L_jk^T x_j)
// Step k: CTA 0 applies X_k to block k (4 threads per output, partial dd
// sums combined in order); grid sync; every warp updates its rows of the
// remaining right-hand side with block column k; grid sync.
// Same operations as the reference's substitutions (crates/quad/src/
// linalg.rs:99-120) grouped by blocks, in another order: f128-level accuracy,
// not bit-identical. Used where a solve is repeated (refinement), with the
// reference-order kernels in solve.cu kept for the single-solve entry points.
#include <cooperative_groups.h>

#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace cg = cooperative_groups;

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

template <bool UPPER_T>
__global__ void __launch_bounds__(256) trsv_blocked_kernel(const dd* __restrict__ L, const dd* __restrict__ Xall,
                                                           dd* __restrict__ v, int64_t n) {
  cg::grid_group grid = cg::this_grid();
  __shared__ dd part[TB][4];
  __shared__ dd vk[TB];
  const int t = threadIdx.x, lane = t % 32;
  const int nblk = (int)((n + TB - 1) / TB);
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + t) / 32;
  const int64_t nwarps = (int64_t)gridDim.x * blockDim.x / 32;
  for (int s = 0; s < nblk; s++) {
    const int k = UPPER_T ? nblk - 1 - s : s;
    const int64_t k0 = (int64_t)k * TB;
    const int jb = (int)min((int64_t)TB, n - k0);
    if (blockIdx.x == 0) {
      // block k of v <- X_k v_k (forward) or X_k^T v_k (backward)
      const dd* X = Xall + (size_t)k * TB * TB;
      const int r = t / 4, q = t % 4;
      dd acc = dd{0.0, 0.0};
      if (r < jb)
        for (int c = q; c < jb; c += 4) {
          const dd xv = UPPER_T ? X[c * TB + r] : X[r * TB + c];
          acc = dd_add(acc, dd_mul(xv, v[k0 + c]));
        }
      part[r][q] = acc;
      __syncthreads();
      if (q == 0 && r < jb) vk[r] = dd_add(dd_add(part[r][0], part[r][1]), dd_add(part[r][2], part[r][3]));
      __syncthreads();
      if (t < jb) v[k0 + t] = vk[t];
    }
    grid.sync();
    // update the remaining rows with block column k
    const int64_t lo = UPPER_T ? 0 : k0 + jb, hi = UPPER_T ? k0 : n;
    for (int64_t i = lo + gwarp; i < hi; i += nwarps) {
      dd acc = dd{0.0, 0.0};
      for (int c = lane; c < jb; c += 32) {
        const dd lv = UPPER_T ? L[(k0 + c) * n + i] : L[i * n + k0 + c];
        acc = dd_add(acc, dd_mul(lv, v[k0 + c]));
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        dd other;
        other.hi = __shfl_down_sync(0xffffffffu, acc.hi, o);
        other.lo = __shfl_down_sync(0xffffffffu, acc.lo, o);
        if (lane < o) acc = dd_add(acc, other);
      }
      if (lane == 0) v[i] = dd_sub(v[i], acc);
    }
    grid.sync();
  }
}

int coop_grid(const void* fn, int threads) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0);
  return sms * (per_sm > 0 ? (per_sm > 2 ? 2 : per_sm) : 1);
}

}  // namespace

int dd_block_inverses(const double* L, size_t n, double* Xall, cudaStream_t s) {
  if (n == 0) return HP_OK;
  const int smem = 2 * TB * (TB + 1) * 16;
  HP_CUDA_TRY(cudaFuncSetAttribute(block_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  block_inverse_kernel<<<(unsigned)((n + TB - 1) / TB), 256, smem, s>>>(reinterpret_cast<const dd*>(L), n,
                                                                        reinterpret_cast<dd*>(Xall));
  HP_LAUNCH_CHECK();
  return HP_OK;
}

size_t dd_block_inverses_bytes(size_t n) { return ((n + TB - 1) / TB) * TB * TB * 16; }

int dd_trsv_blocked(const double* L, const double* Xall, double* v, size_t n, bool upper_t, cudaStream_t s) {
  if (n == 0) return HP_OK;
  const dd* Lp = reinterpret_cast<const dd*>(L);
  const dd* Xp = reinterpret_cast<const dd*>(Xall);
  dd* vp = reinterpret_cast<dd*>(v);
  int64_t nn = (int64_t)n;
  void* args[] = {(void*)&Lp, (void*)&Xp, (void*)&vp, (void*)&nn};
  const void* fn = upper_t ? (const void*)trsv_blocked_kernel<true> : (const void*)trsv_blocked_kernel<false>;
  const int grid = coop_grid(fn, 256);
  HP_CUDA_TRY(cudaLaunchCooperativeKernel(fn, grid, 256, args, 0, s));
  return HP_OK;
}

}  // namespace hp
