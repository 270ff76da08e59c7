// Plain (CUDA-core) f128 and f256 GEMM: the reference's algorithm, one
// sequential k-ordered accumulation per C entry, made fast by tiling.
//
// Reference: crates/quad/src/linalg.rs:150-182 (gemm, gemm_atb) and
// crates/quad/src/multifloat/linalg.rs:39-85 (mf_gemm, mf_gemm_atb):
//     s = 0; for p in 0..k { s += a(i,p) * b(p,j) }; c(i,j) = s
// Each thread owns whole C entries and runs that loop in p order with the
// reference's Mul and Add (hp_arith.cuh), so C is bit-identical to the
// reference. No split-k: splitting would change the summation order.
//
// Layout: operands are read in the reference's AoS layout with 16-byte
// (f128) / 2x16-byte (f256) vector loads, which are fully coalesced along a
// row; shared memory holds each limb as its own plane so the inner loop
// reads 8-byte words without bank conflicts.
//
// Bound: the FP64 pipe. One f128 multiply-add is 29 FP64 instructions
// (Mul: 2 MUL + 1 FMA + 5 ADD/SUB; Add: 20 ADD/SUB), so the ceiling is
// P64_instr / 29 * 2 flops.
#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
namespace {

constexpr int DD_BM = 64, DD_BN = 64, DD_BK = 16, DD_TX = 16, DD_TY = 16;
constexpr int DD_RM = DD_BM / DD_TY, DD_RN = DD_BN / DD_TX;  // 4 x 4 entries per thread

// C (m x n) = op(A) * B. op(A)(i,p) = A[i*k+p] (ATB=false) or A[p*m+i].
template <bool ATB>
__global__ void __launch_bounds__(DD_TX* DD_TY, 1)
    dd_gemm_plain_kernel(const double2* __restrict__ A, const double2* __restrict__ B,
                         double2* __restrict__ C, int64_t m, int64_t n, int64_t k) {
  __shared__ double As_hi[DD_BK][DD_BM + 1], As_lo[DD_BK][DD_BM + 1];
  __shared__ double Bs_hi[DD_BK][DD_BN], Bs_lo[DD_BK][DD_BN];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * DD_TX + tx;
  const int64_t m0 = (int64_t)blockIdx.y * DD_BM, n0 = (int64_t)blockIdx.x * DD_BN;

  dd acc[DD_RM][DD_RN];
#pragma unroll
  for (int i = 0; i < DD_RM; i++)
#pragma unroll
    for (int j = 0; j < DD_RN; j++) acc[i][j] = dd{0.0, 0.0};

  // Register staging for the next k-tile: 1024 A and 1024 B entries per
  // tile, 4 of each per thread.
  double2 ra[4], rb[4];
  auto load_tile = [&](int64_t k0) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int e = tid + q * 256;
      int64_t gi, gp;
      if (!ATB) {  // tile is BM rows x BK cols, read along k
        gi = m0 + e / DD_BK;
        gp = k0 + e % DD_BK;
      } else {     // tile is BK rows x BM cols of the k x m matrix, read along m
        gp = k0 + e / DD_BM;
        gi = m0 + e % DD_BM;
      }
      ra[q] = (gi < m && gp < k) ? (ATB ? A[gp * m + gi] : A[gi * k + gp]) : make_double2(0.0, 0.0);
      int64_t bp = k0 + e / DD_BN, bj = n0 + e % DD_BN;
      rb[q] = (bp < k && bj < n) ? B[bp * n + bj] : make_double2(0.0, 0.0);
    }
  };
  auto store_tile = [&]() {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int e = tid + q * 256;
      int r, c;
      if (!ATB) {
        r = e % DD_BK;
        c = e / DD_BK;
      } else {
        r = e / DD_BM;
        c = e % DD_BM;
      }
      As_hi[r][c] = ra[q].x;
      As_lo[r][c] = ra[q].y;
      Bs_hi[e / DD_BN][e % DD_BN] = rb[q].x;
      Bs_lo[e / DD_BN][e % DD_BN] = rb[q].y;
    }
  };

  load_tile(0);
  for (int64_t k0 = 0; k0 < k; k0 += DD_BK) {
    __syncthreads();
    store_tile();
    __syncthreads();
    if (k0 + DD_BK < k) load_tile(k0 + DD_BK);
    const int kmax = (int)((k - k0) < DD_BK ? (k - k0) : DD_BK);
    for (int kk = 0; kk < kmax; kk++) {
      dd a[DD_RM], b[DD_RN];
#pragma unroll
      for (int i = 0; i < DD_RM; i++) a[i] = dd{As_hi[kk][ty + DD_TY * i], As_lo[kk][ty + DD_TY * i]};
#pragma unroll
      for (int j = 0; j < DD_RN; j++) b[j] = dd{Bs_hi[kk][tx + DD_TX * j], Bs_lo[kk][tx + DD_TX * j]};
#pragma unroll
      for (int i = 0; i < DD_RM; i++)
#pragma unroll
        for (int j = 0; j < DD_RN; j++) acc[i][j] = dd_add(acc[i][j], dd_mul(a[i], b[j]));
    }
  }
#pragma unroll
  for (int i = 0; i < DD_RM; i++) {
    int64_t gi = m0 + ty + DD_TY * i;
    if (gi >= m) continue;
#pragma unroll
    for (int j = 0; j < DD_RN; j++) {
      int64_t gj = n0 + tx + DD_TX * j;
      if (gj < n) C[gi * n + gj] = make_double2(acc[i][j].hi, acc[i][j].lo);
    }
  }
}

// f256: one C entry per thread, 16 x 16 tile, k-tiles of 16.
constexpr int QD_T = 16, QD_BK = 16;

template <bool ATB>
__global__ void __launch_bounds__(QD_T* QD_T)
    qd_gemm_plain_kernel(const double4* __restrict__ A, const double4* __restrict__ B,
                         double4* __restrict__ C, int64_t m, int64_t n, int64_t k) {
  __shared__ double As[4][QD_BK][QD_T + 1];
  __shared__ double Bs[4][QD_BK][QD_T];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t gi = (int64_t)blockIdx.y * QD_T + ty, gj = (int64_t)blockIdx.x * QD_T + tx;
  const int64_t m0 = (int64_t)blockIdx.y * QD_T;
  qd acc = qd_zero();
  for (int64_t k0 = 0; k0 < k; k0 += QD_BK) {
    __syncthreads();
    {
      // A tile: 16 rows (i) x 16 k. Thread (ty, tx) loads op(A)(m0+ty, k0+tx).
      int64_t ai = m0 + ty, ap = k0 + tx;
      double4 v = make_double4(0, 0, 0, 0);
      if (ai < m && ap < k) v = ATB ? A[ap * m + ai] : A[ai * k + ap];
      As[0][tx][ty] = v.x;
      As[1][tx][ty] = v.y;
      As[2][tx][ty] = v.z;
      As[3][tx][ty] = v.w;
      int64_t bp = k0 + ty, bj = gj;
      double4 w = make_double4(0, 0, 0, 0);
      if (bp < k && bj < n) w = B[bp * n + bj];
      Bs[0][ty][tx] = w.x;
      Bs[1][ty][tx] = w.y;
      Bs[2][ty][tx] = w.z;
      Bs[3][ty][tx] = w.w;
    }
    __syncthreads();
    const int kmax = (int)((k - k0) < QD_BK ? (k - k0) : QD_BK);
    for (int kk = 0; kk < kmax; kk++) {
      qd a = qd{{As[0][kk][ty], As[1][kk][ty], As[2][kk][ty], As[3][kk][ty]}};
      qd b = qd{{Bs[0][kk][tx], Bs[1][kk][tx], Bs[2][kk][tx], Bs[3][kk][tx]}};
      acc = qd_add(acc, qd_mul(a, b));
    }
  }
  if (gi < m && gj < n) C[gi * n + gj] = make_double4(acc.l[0], acc.l[1], acc.l[2], acc.l[3]);
}

}  // namespace

int dd_gemm_plain(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                  bool atb, cudaStream_t s) {
  if (m == 0 || n == 0) return HP_OK;
  if (k == 0) {
    HP_CUDA_TRY(cudaMemsetAsync(c, 0, m * n * 16, s));
    return HP_OK;
  }
  if ((m + DD_BM - 1) / DD_BM > 65535) {
    set_error("f128 gemm: m = %zu exceeds the grid limit", m);
    return HP_ERR_INVALID_ARG;
  }
  dim3 grid((unsigned)((n + DD_BN - 1) / DD_BN), (unsigned)((m + DD_BM - 1) / DD_BM));
  dim3 block(DD_TX, DD_TY);
  if (atb)
    dd_gemm_plain_kernel<true><<<grid, block, 0, s>>>((const double2*)a, (const double2*)b,
                                                      (double2*)c, m, n, k);
  else
    dd_gemm_plain_kernel<false><<<grid, block, 0, s>>>((const double2*)a, (const double2*)b,
                                                       (double2*)c, m, n, k);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

int qd_gemm_plain(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                  bool atb, cudaStream_t s) {
  if (m == 0 || n == 0) return HP_OK;
  if (k == 0) {
    HP_CUDA_TRY(cudaMemsetAsync(c, 0, m * n * 32, s));
    return HP_OK;
  }
  if ((m + QD_T - 1) / QD_T > 65535) {
    set_error("f256 gemm: m = %zu exceeds the grid limit", m);
    return HP_ERR_INVALID_ARG;
  }
  dim3 grid((unsigned)((n + QD_T - 1) / QD_T), (unsigned)((m + QD_T - 1) / QD_T));
  dim3 block(QD_T, QD_T);
  if (atb)
    qd_gemm_plain_kernel<true><<<grid, block, 0, s>>>((const double4*)a, (const double4*)b,
                                                      (double4*)c, m, n, k);
  else
    qd_gemm_plain_kernel<false><<<grid, block, 0, s>>>((const double4*)a, (const double4*)b,
                                                       (double4*)c, m, n, k);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace hp
