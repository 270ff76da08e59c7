// Blocked f128 triangular solves for refinement loops: L y = b and L^T x = y
// with the inverses X_k = L_kk^-1 of the 64 x 64 diagonal blocks of L
// precomputed once per factorisation:
//   forward:  y_k = X_k (b_k - sum_{j<k} L_kj y_j)
//   backward: x_k = X_k^T (y_k - sum_{j>k} L_jk^T x_j)
// One launch, one CTA per block row, no grid-wide barrier: CTAs take block
// rows in dependency order from a ticket counter; each accumulates the
// products with the solved blocks as they appear (its L tile is loaded
// before the wait), then applies X_k and publishes its block. A CTA only
// ever waits for CTAs that took earlier tickets, so the wavefront makes
// progress whatever the residency.
//
// Publication without flags: a solved block is written (relaxed, gpu scope)
// to an exchange buffer whose entries hold a sentinel bit pattern (both
// limbs all ones, a NaN no result can carry: published NaNs are written as
// the canonical NaN) until then, and a consumer polls the values themselves,
// so a dependency costs one store-to-load latency instead of a fence, a flag
// and a second load. Two exchange buffers alternate by launch parity; every
// launch refills the other one with sentinels for the next, and the last
// CTA to finish resets the ticket counter. Every wait is bounded (2 s of
// global time, or an abort raised by another CTA) and a CTA that gives up
// records DEV_STATUS_TIMEOUT in the status word the host reads.
//
// Same operations as the reference's substitutions (crates/quad/src/
// linalg.rs:99-120) grouped by blocks, in another order: f128-level accuracy,
// not bit-identical. Used where a solve is repeated (refinement), with the
// reference-order kernels in solve.cu kept for the single-solve entry points.
#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"
#include "sm100_ptx.cuh"

namespace hp {
namespace {

constexpr int TB = 64;         // block size
constexpr int INV_COLS = 8;    // columns of X_k per CTA of block_inverse_kernel (one warp each)
constexpr unsigned long long SENTINEL = ~0ull;

// Wavefront bookkeeping behind the inverses in the same workspace, followed
// by the two exchange buffers (nblk * TB entries each).
struct TrsvSync {
  unsigned ticket;  // next block row to hand out (0 when a launch starts)
  unsigned done;    // CTAs finished in the current launch
  unsigned launch;  // launches completed on this workspace; parity picks the exchange buffer
  unsigned abort;   // a CTA gave up: the others stop waiting
  unsigned status;  // DEV_STATUS_* bits, read by the host
  unsigned pad[3];
};
static_assert(sizeof(TrsvSync) % 16 == 0, "exchange buffers stay 16-byte aligned");
inline size_t nblocks(size_t n) { return (n + TB - 1) / TB; }
inline size_t inverses_bytes(size_t n) { return nblocks(n) * TB * TB * 16; }

__device__ __forceinline__ void ld_relaxed_v2(const dd* p, unsigned long long& a, unsigned long long& b) {
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}
__device__ __forceinline__ void st_relaxed_v2(dd* p, unsigned long long a, unsigned long long b) {
  asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}
__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long canonical_bits(double x) {
  return x != x ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(x);
}

// X_k = L_kk^-1, column by column: CTA (k, g) computes columns
// g*INV_COLS .. g*INV_COLS + INV_COLS - 1 of block k, one warp per column
// (lane l holds rows l and l + 32). Column c is a forward substitution
// L_kk x = e_c: x_i is final once rows < i have been applied, is scaled by
// 1/l_ii, broadcast by shuffle, and subtracted (times column i of L_kk)
// from the rows below; the strictly lower copy of L_kk in shared memory
// makes the update unconditional. Xall[k] is row-major 64 x 64; rows and
// columns beyond the last block's size are zero. The CTAs of column group 0
// also fill both exchange buffers with sentinels and CTA (0, 0) clears the
// wavefront bookkeeping, so the solves need no memset.
__global__ void __launch_bounds__(INV_COLS * 32) block_inverse_kernel(const dd* __restrict__ L, int64_t n,
                                                                      dd* __restrict__ Xall, TrsvSync* sync,
                                                                      dd* __restrict__ xchg, int nblk) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  dd(*A)[TB + 1] = reinterpret_cast<dd(*)[TB + 1]>(sm_raw);  // [TB][TB + 1], strictly lower
  __shared__ dd inv[TB];
  const int t = threadIdx.x, lane = t % 32, w = t / 32;
  const int64_t k0 = (int64_t)blockIdx.x * TB;
  const int jb = (int)min((int64_t)TB, n - k0);
  for (int q = t; q < TB * TB; q += blockDim.x) {
    const int r = q / TB, c = q % TB;
    A[r][c] = (r < jb && c < r) ? L[(k0 + r) * n + k0 + c] : dd{0.0, 0.0};
  }
  if (t < TB) inv[t] = t < jb ? dd_recip(L[(k0 + t) * n + k0 + t]) : dd_from(1.0);
  if (blockIdx.y == 0) {
    for (int q = t; q < 2 * TB; q += blockDim.x)
      st_relaxed_v2(xchg + (size_t)(q / TB) * nblk * TB + k0 + q % TB, SENTINEL, SENTINEL);
    if (blockIdx.x == 0 && t == 0) *sync = TrsvSync{0, 0, 0, 0, 0, {0, 0, 0}};
  }
  __syncthreads();
  const int c = blockIdx.y * INV_COLS + w;
  dd x0 = dd_from(lane == c ? 1.0 : 0.0), x1 = dd_from(lane + 32 == c ? 1.0 : 0.0);
  for (int i = c; i < 32; i++) {  // pivot rows 0..31 live in x0
    dd xi = {__shfl_sync(0xffffffffu, x0.hi, i), __shfl_sync(0xffffffffu, x0.lo, i)};
    xi = dd_mul(xi, inv[i]);
    if (lane == i) x0 = xi;
    x0 = dd_fms_fast(x0, A[lane][i], xi);
    x1 = dd_fms_fast(x1, A[lane + 32][i], xi);
  }
  for (int i = max(c, 32); i < TB; i++) {  // pivot rows 32..63: only x1 moves
    dd xi = {__shfl_sync(0xffffffffu, x1.hi, i - 32), __shfl_sync(0xffffffffu, x1.lo, i - 32)};
    xi = dd_mul(xi, inv[i]);
    if (lane == i - 32) x1 = xi;
    x1 = dd_fms_fast(x1, A[lane + 32][i], xi);
  }
  dd* out = Xall + (size_t)blockIdx.x * TB * TB;
  const bool live = c < jb;
  out[lane * TB + c] = live && lane < jb ? x0 : dd{0.0, 0.0};
  out[(lane + 32) * TB + c] = live && lane + 32 < jb ? x1 : dd{0.0, 0.0};
}

// Poll an exchange entry until both limbs hold a published value; false if
// the wait gave up (wait_ns of global time, or another CTA's abort).
__device__ __forceinline__ bool poll_entry(const dd* p, dd& out, TrsvSync* sync, uint64_t wait_ns) {
  const uint64_t t0 = sm100::globaltimer_ns();
  for (unsigned it = 1;; it++) {
    unsigned long long h, l;
    ld_relaxed_v2(p, h, l);
    if (h != SENTINEL && l != SENTINEL) {
      out = dd{__longlong_as_double((long long)h), __longlong_as_double((long long)l)};
      return true;
    }
    if ((it & 31) == 0 && (ld_relaxed_u32(&sync->abort) || sm100::globaltimer_ns() - t0 > wait_ns)) {
      atomicOr(&sync->status, (unsigned)DEV_STATUS_TIMEOUT);
      atomicExch(&sync->abort, 1u);
      return false;
    }
  }
}

// Block row k: thread (r, q) = (t / 4, t % 4) owns row r of the block and
// the columns c = q (mod 4) of each 64 x 64 tile it multiplies; the four
// partial sums of a row sit on neighbouring lanes and are combined by
// shuffles (dd_add is commutative bit for bit, so all four agree).
// withheld >= 0 names one block row that is solved but not published: the
// diagnostic entry point uses this to make the waits of the CTAs after it
// run out (with a short wait_ns) and checks that the launch ends with
// DEV_STATUS_TIMEOUT; the solver passes -1.
template <bool UPPER_T>
__global__ void __launch_bounds__(256) trsv_wave_kernel(const dd* __restrict__ L, const dd* __restrict__ Xall,
                                                        dd* v, int64_t n, int nblk, TrsvSync* sync, dd* xchg,
                                                        uint64_t wait_ns, int withheld) {
  __shared__ unsigned my, par;
  __shared__ int bad[2];  // per dependency parity: a poll gave up
  __shared__ dd vj[2][TB], sv[TB];
  const int t = threadIdx.x, r = t / 4, q = t % 4;
  if (t == 0) {
    my = atomicAdd(&sync->ticket, 1u);
    par = ld_relaxed_u32(&sync->launch) & 1u;
    bad[0] = bad[1] = 0;
  }
  __syncthreads();
  const int s = (int)my;  // < nblk: the grid has one CTA per block row
  const int k = UPPER_T ? nblk - 1 - s : s;
  const int64_t k0 = (int64_t)k * TB;
  const int jb = (int)min((int64_t)TB, n - k0);
  dd* cur = xchg + (size_t)par * nblk * TB;           // this launch's exchange buffer
  dd* nxt = xchg + (size_t)(par ^ 1u) * nblk * TB;    // the next launch's, refilled here
  if (t < TB) st_relaxed_v2(nxt + k0 + t, SENTINEL, SENTINEL);
  const dd br = (q == 0 && r < jb) ? v[k0 + r] : dd{0.0, 0.0};  // only this CTA touches v's block k
  // X_k row r (forward) or column r (backward), loaded before any wait
  const dd* X = Xall + (size_t)k * TB * TB;
  dd xr[TB / 4];
#pragma unroll
  for (int m = 0; m < TB / 4; m++) {
    const int c = q + 4 * m;
    xr[m] = UPPER_T ? X[c * TB + r] : X[r * TB + c];
  }
  dd acc0 = {0.0, 0.0}, acc1 = {0.0, 0.0};
  bool ok = true;
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
    if (t < TB) {
      dd val = {0.0, 0.0};
      if (t < jbj && !poll_entry(cur + j0 + t, val, sync, wait_ns)) bad[d & 1] = 1;
      vj[d & 1][t] = val;
    }
    __syncthreads();
    if (bad[d & 1]) {  // every thread reads the same word after the same barrier
      ok = false;
      break;
    }
    const dd* y = vj[d & 1];
#pragma unroll
    for (int m = 0; m < TB / 4; m += 2) {
      acc0 = dd_fms_fast(acc0, dd{-lv[m].hi, -lv[m].lo}, y[q + 4 * m]);
      acc1 = dd_fms_fast(acc1, dd{-lv[m + 1].hi, -lv[m + 1].lo}, y[q + 4 * m + 4]);
    }
  }
  if (ok) {
    dd a = dd_add(acc0, acc1);
    a = dd_add(a, dd{__shfl_xor_sync(0xffffffffu, a.hi, 1), __shfl_xor_sync(0xffffffffu, a.lo, 1)});
    a = dd_add(a, dd{__shfl_xor_sync(0xffffffffu, a.hi, 2), __shfl_xor_sync(0xffffffffu, a.lo, 2)});
    if (q == 0) sv[r] = r < jb ? dd_sub(br, a) : dd{0.0, 0.0};
    __syncthreads();
    acc0 = acc1 = dd{0.0, 0.0};
#pragma unroll
    for (int m = 0; m < TB / 4; m += 2) {
      acc0 = dd_fms_fast(acc0, dd{-xr[m].hi, -xr[m].lo}, sv[q + 4 * m]);
      acc1 = dd_fms_fast(acc1, dd{-xr[m + 1].hi, -xr[m + 1].lo}, sv[q + 4 * m + 4]);
    }
    a = dd_add(acc0, acc1);
    a = dd_add(a, dd{__shfl_xor_sync(0xffffffffu, a.hi, 1), __shfl_xor_sync(0xffffffffu, a.lo, 1)});
    a = dd_add(a, dd{__shfl_xor_sync(0xffffffffu, a.hi, 2), __shfl_xor_sync(0xffffffffu, a.lo, 2)});
    if (q == 0 && r < jb && k != withheld) {
      st_relaxed_v2(cur + k0 + r, canonical_bits(a.hi), canonical_bits(a.lo));
      v[k0 + r] = a;
    }
  }
  // the last CTA out resets the ticket counter and flips the buffer parity
  __syncthreads();
  if (t == 0) {
    __threadfence();
    if (atomicAdd(&sync->done, 1u) == (unsigned)nblk - 1) {
      sync->ticket = 0;
      sync->done = 0;
      sync->launch += 1;
    }
  }
}

}  // namespace

int dd_block_inverses(const double* L, size_t n, double* Xall, cudaStream_t s) {
  if (n == 0) return HP_OK;
  const int smem = TB * (TB + 1) * 16;
  HP_CUDA_TRY(cudaFuncSetAttribute(block_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int nblk = (int)nblocks(n);
  char* tail = reinterpret_cast<char*>(Xall) + inverses_bytes(n);
  block_inverse_kernel<<<dim3((unsigned)nblk, TB / INV_COLS), INV_COLS * 32, smem, s>>>(
      reinterpret_cast<const dd*>(L), n, reinterpret_cast<dd*>(Xall), reinterpret_cast<TrsvSync*>(tail),
      reinterpret_cast<dd*>(tail + sizeof(TrsvSync)), nblk);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

size_t dd_block_inverses_bytes(size_t n) { return inverses_bytes(n) + sizeof(TrsvSync) + 2 * nblocks(n) * TB * 16; }

int dd_trsv_blocked(const double* L, const double* Xall, double* v, size_t n, bool upper_t, cudaStream_t s,
                    uint64_t wait_ns, int withheld) {
  if (n == 0) return HP_OK;
  char* tail = const_cast<char*>(reinterpret_cast<const char*>(Xall)) + inverses_bytes(n);
  TrsvSync* sync = reinterpret_cast<TrsvSync*>(tail);
  dd* xchg = reinterpret_cast<dd*>(tail + sizeof(TrsvSync));
  const int nblk = (int)nblocks(n);
  const dd* Lp = reinterpret_cast<const dd*>(L);
  const dd* Xp = reinterpret_cast<const dd*>(Xall);
  dd* vp = reinterpret_cast<dd*>(v);
  if (upper_t)
    trsv_wave_kernel<true><<<nblk, 256, 0, s>>>(Lp, Xp, vp, (int64_t)n, nblk, sync, xchg, wait_ns, withheld);
  else
    trsv_wave_kernel<false><<<nblk, 256, 0, s>>>(Lp, Xp, vp, (int64_t)n, nblk, sync, xchg, wait_ns, withheld);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

const unsigned* dd_trsv_status_word(const double* Xall, size_t n) {
  const TrsvSync* sync = reinterpret_cast<const TrsvSync*>(reinterpret_cast<const char*>(Xall) + inverses_bytes(n));
  return &sync->status;
}

}  // namespace hp

extern "C" int hp_debug_trsv_wavefront(const double* l, const double* b, double* x, size_t n, int upper_t,
                                       uint64_t wait_ns, int withheld_block) {
  using namespace hp;
  if (n == 0) return HP_OK;
  size_t t, bytes;
  if (hp::mul_overflows(n, n, &t) || hp::mul_overflows(t, 16, &bytes)) {
    set_error("matrix size overflows size_t");
    return HP_ERR_INVALID_ARG;
  }
  if (!l || !b || !x) {
    set_error("null pointer with non-zero size");
    return HP_ERR_INVALID_ARG;
  }
  if (withheld_block >= (int)nblocks(n)) {
    set_error("withheld_block %d is not a block of the %zu-row solve", withheld_block, n);
    return HP_ERR_INVALID_ARG;
  }
  cudaStream_t s = library_stream();
  DevBuf dl(bytes, s), dv(n * 16, s), dx(dd_block_inverses_bytes(n), s);
  if (!dl.p || !dv.p || !dx.p) {
    set_error("device allocation failed");
    return HP_ERR_CUDA;
  }
  HP_CUDA_TRY(cudaMemcpyAsync(dl.p, l, bytes, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dv.p, b, n * 16, cudaMemcpyHostToDevice, s));
  HP_TRY(dd_block_inverses(dl.as<double>(), n, dx.as<double>(), s));
  HP_TRY(dd_trsv_blocked(dl.as<double>(), dx.as<double>(), dv.as<double>(), n, upper_t != 0, s,
                         wait_ns ? wait_ns : TRSV_WAIT_NS, withheld_block));
  unsigned st = 0;
  HP_CUDA_TRY(cudaMemcpyAsync(&st, dd_trsv_status_word(dx.as<double>(), n), sizeof(st), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(x, dv.p, n * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (st & DEV_STATUS_TIMEOUT) {
    set_error("wavefront solve: a bounded wait gave up (status 0x%x)", st);
    return HP_ERR_TIMEOUT;
  }
  return HP_OK;
}
