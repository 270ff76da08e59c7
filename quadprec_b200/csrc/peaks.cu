// Roofline denominators measured on the device itself (no reference
// counterpart): the FP64 pipe (a DFMA loop) and the int8 tensor pipe (a
// tcgen05.mma kind::i8 loop). The library's kernels are reported as fractions
// of these rates, so each loop issues the same instruction the hot kernels
// are bound by, at full occupancy, with nothing else in the way.
//
// FP64: every thread runs 8 independent DFMA chains (enough in flight to
// cover the pipe's latency at 8 warps per scheduler), 2 flops per DFMA.
// int8: one CTA per SM (the dynamic shared memory keeps a second one out),
// one thread issues M = 128, N = 256, K = 32 unsigned MMAs from 128-byte
// swizzled K-major tiles in shared memory into two TMEM accumulators
// (2 * 128 * 256 * 32 ops each), then commits once and waits (bounded) for
// them to finish. The operands are zero: the rate does not depend on values.
#include <algorithm>

#include "hp_runtime.cuh"
#include "sm100_ptx.cuh"

namespace hp {
namespace {

constexpr int F64_CHAINS = 8;

__global__ void __launch_bounds__(256) fp64_peak_kernel(double* out, int iters, double a, double b) {
  double acc[F64_CHAINS];
#pragma unroll
  for (int c = 0; c < F64_CHAINS; c++) acc[c] = threadIdx.x * 1e-9 + c;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int c = 0; c < F64_CHAINS; c++) acc[c] = __fma_rn(acc[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < F64_CHAINS; c++) s += acc[c];
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains live; never true for these inputs
}

constexpr int PK_M = 128, PK_N = 256, PK_KB = 128;  // K bytes per tile (4 MMAs of K = 32)
constexpr int PK_SMEM = 1024 + PK_M * PK_KB + PK_N * PK_KB;
constexpr int PK_SMEM_LAUNCH = 160 * 1024;  // one CTA per SM

__global__ void __launch_bounds__(128, 1) i8_mma_peak_kernel(int iters, uint32_t* status) {
  using namespace sm100;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t* sA = smem_raw + pad;
  uint8_t* sB = sA + PK_M * PK_KB;
  __shared__ uint64_t done;
  __shared__ uint32_t tmem_slot;
  for (int i = threadIdx.x; i < (PK_M + PK_N) * PK_KB / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(sA)[i] = make_uint4(0, 0, 0, 0);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  const int warp = threadIdx.x / 32;
  if (threadIdx.x == 0) {
    mbar_init(&done, 1);
    fence_mbarrier_init();
  }
  if (warp == 0) {
    tmem_alloc(&tmem_slot, 2 * PK_N);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  if (threadIdx.x == 0) {
    const uint32_t idesc = idesc_i8(PK_M, PK_N, true);
    const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
    for (int i = 0; i < iters; i++) {
      const uint32_t d = tmem + (uint32_t)(i & 1) * PK_N;
#pragma unroll
      for (int kk = 0; kk < PK_KB / 32; kk++)
        mma_i8(d, desc_k_sw128(a0 + kk * 32), desc_k_sw128(b0 + kk * 32), idesc, (i > 1 || kk) ? 1u : 0u);
    }
    mma_commit(&done);
    mbar_wait(&done, 0, status, DEV_STATUS_TIMEOUT);
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * PK_N);
  }
}

}  // namespace
}  // namespace hp

extern "C" int hp_measure_peaks(int reps, double* fp64_tflops, double* i8_tops, double* fp64_ms, double* i8_ms) {
  using namespace hp;
  if (reps <= 0) reps = 5;
  int dev = 0, sms = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  HP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  cudaStream_t s = library_stream();
  uint32_t* status = device_status(s);
  if (!status) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  DevBuf out(sizeof(double) * 4096, s);
  if (!out.p) return HP_ERR_CUDA;
  cudaEvent_t e0, e1;
  HP_CUDA_TRY(cudaEventCreate(&e0));
  HP_CUDA_TRY(cudaEventCreate(&e1));
  // FP64: 8 CTAs of 256 threads per SM
  const int f_blocks = sms * 8, f_iters = 1 << 15;
  float best = 1e30f, ms = 0.0f;
  for (int r = 0; r < reps + 1; r++) {
    HP_CUDA_TRY(cudaEventRecord(e0, s));
    fp64_peak_kernel<<<f_blocks, 256, 0, s>>>(out.as<double>(), f_iters, 0.999999, 1e-7);
    HP_LAUNCH_CHECK();
    HP_CUDA_TRY(cudaEventRecord(e1, s));
    HP_CUDA_TRY(cudaEventSynchronize(e1));
    HP_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    if (r > 0) best = std::min(best, ms);  // the first run loads the module
  }
  const double f_flops = 2.0 * F64_CHAINS * (double)f_iters * 256.0 * f_blocks;
  if (fp64_tflops) *fp64_tflops = f_flops / (best * 1e-3) / 1e12;
  if (fp64_ms) *fp64_ms = best;
  // int8 tensor pipe
  HP_CUDA_TRY(cudaFuncSetAttribute(i8_mma_peak_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PK_SMEM_LAUNCH));
  static_assert(PK_SMEM <= PK_SMEM_LAUNCH, "tiles fit the launch's shared memory");
  const int i_iters = 1 << 13;
  best = 1e30f;
  for (int r = 0; r < reps + 1; r++) {
    HP_CUDA_TRY(cudaEventRecord(e0, s));
    i8_mma_peak_kernel<<<sms, 128, PK_SMEM_LAUNCH, s>>>(i_iters, status);
    HP_LAUNCH_CHECK();
    HP_CUDA_TRY(cudaEventRecord(e1, s));
    HP_CUDA_TRY(cudaEventSynchronize(e1));
    HP_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    if (r > 0) best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  HP_TRY(consume_device_status(s));
  const double i_ops = 2.0 * PK_M * PK_N * PK_KB * (double)i_iters * sms;
  if (i8_tops) *i8_tops = i_ops / (best * 1e-3) / 1e12;
  if (i8_ms) *i8_ms = best;
  return HP_OK;
}
