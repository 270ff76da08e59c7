// Exact extended-precision GEMM on the int8 tensor cores (Ozaki scheme II:
// residue number system + Chinese remainder reconstruction).
//
// For C = op(A) * B with f128 entries:
//  1. Row i of op(A) and column j of B are scaled by powers of two so that
//     every entry becomes an integer of at most BETA bits:
//        X_ip = rint(A_ip * 2^sa_i),  Y_pj = rint(B_pj * 2^sb_j).
//     This rounding is the only approximation (|error| <= 2^-BETA of the
//     row/column maximum, per limb).
//  2. For each of L pairwise-coprime moduli m_l <= 256, X and Y are reduced
//     to balanced int8 residues (exact integer arithmetic).
//  3. One int8 GEMM per modulus on tcgen05 (int32 accumulation in TMEM,
//     exact while k * 2^14 < 2^31); the epilogue reduces each int32 to its
//     residue mod m_l and stores one byte.
//  4. The CRT combines the L residues into the exact integer
//     Z_ij = sum_p X_ip Y_pj (|Z| < M/4, M = prod m_l), which is rounded
//     once to f128 and scaled by 2^-(sa_i + sb_j).
// L is the smallest count with log2 M >= 2*BETA + ceil(log2 k) + 2.
//
// The reference computes the same product with f128 multiply-adds
// (crates/quad/src/linalg.rs:150-182); this path returns that product to
// within 2^-(BETA-3) normwise, i.e. inside the 4*k*2^-104 tolerance.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "hp_arith.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"
#include "sm100_ptx.cuh"

namespace hp {
// Launch kernel k; with pdl set, as a programmatic dependent launch: the
// kernel may be scheduled while its predecessor in the stream still runs
// and waits for it (griddep_wait) before touching the predecessor's
// output. The Ozaki GEMM's phases and the residue-domain Cholesky's
// diagonal path are chained this way, so that each launch's set-up
// overlaps the tail of the previous kernel.
template <typename... P, typename... A>
static cudaError_t launch_k(bool pdl, void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? at : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

namespace ozaki {

constexpr int MAXL = 49;        // number of pairwise-coprime moduli <= 256 in the table
constexpr int NDIG = 5;         // base-2^22 digits of a scaled integer (110 bits)
constexpr int NDIG2 = 10;       // digits of the 220-bit integers of the residue-domain Cholesky
constexpr int CRT_BITS = 39;    // chunk width of the CRT accumulators
constexpr int NCMAX = 10;       // chunks needed for M < 2^342
constexpr int BETA_DD = 106;    // bits kept per f128 operand entry
constexpr int EXP_NONFINITE = 0x7FF;

struct ModTable {
  int mod[MAXL];
  uint32_t magic[MAXL];   // floor(2^32 / m)
  uint32_t offset[MAXL];  // m * ceil(2^31 / m): makes |x| <= 2^30 + 2^27 non-negative
  int pw[MAXL][NDIG2];    // 2^(22 c) mod m, balanced into [-m/2, m/2]
  int pw21[MAXL][5];      // 2^(21 c) mod m, balanced (digits of the f256 operands)
};
__constant__ ModTable c_tab;

struct CrtTable {
  int L, nc;
  double w[MAXL][NCMAX];  // W_l = (M/m_l) * ((M/m_l)^-1 mod m_l) in 39-bit chunks
  double mchunk[NCMAX];   // M in 39-bit chunks
  double inv_m;           // 1 / M (rounded)
};

// CRT tables of the moduli counts the f128 GEMM uses (k <= 2^20 at beta =
// 106), in constant memory so that the specialised CRT kernel's weights
// are immediate operands of its multiply-adds.
constexpr int CRT_CONST_L0 = 28, CRT_CONST_N = 5;
__constant__ CrtTable c_crt[CRT_CONST_N];  // L = CRT_CONST_L0 + i

// Tables of the tensor-core CRT (crt_tc_kernel), for the same moduli counts:
// the bytes of every weight W_l (the B operand of a u8 MMA: row q holds byte
// q of W_0 .. W_{L-1}), the 16-bit limbs of M and 2^192 / M.
struct CrtTcTable {
  uint8_t wb[32][32];
  int32_t mlimb[16];
  double k192;
};
__constant__ CrtTcTable c_crt_tc[CRT_CONST_N];  // L = CRT_CONST_L0 + i

// ---------------------------------------------------------------------------
// Host tables
// ---------------------------------------------------------------------------
struct HostTables {
  ModTable mt;
  std::vector<CrtTable> crt;  // index L (1..MAXL)
  CrtTcTable crt_tc[CRT_CONST_N];
  double cum_log2[MAXL + 1];
};

// Little-endian base-2^32 unsigned big integer (host only, table set-up).
struct Big {
  std::vector<uint32_t> d;
};
static void big_mul_small(Big& a, uint32_t m) {
  uint64_t carry = 0;
  for (auto& x : a.d) {
    uint64_t t = (uint64_t)x * m + carry;
    x = (uint32_t)t;
    carry = t >> 32;
  }
  if (carry) a.d.push_back((uint32_t)carry);
}
static uint32_t big_mod_small(const Big& a, uint32_t m) {
  uint64_t r = 0;
  for (size_t i = a.d.size(); i-- > 0;) r = ((r << 32) | a.d[i]) % m;
  return (uint32_t)r;
}
static Big big_div_small(const Big& a, uint32_t m) {
  Big q;
  q.d.assign(a.d.size(), 0);
  uint64_t r = 0;
  for (size_t i = a.d.size(); i-- > 0;) {
    uint64_t cur = (r << 32) | a.d[i];
    q.d[i] = (uint32_t)(cur / m);
    r = cur % m;
  }
  while (!q.d.empty() && q.d.back() == 0) q.d.pop_back();
  return q;
}
static double big_chunk(const Big& a, int c) {  // bits [39c, 39c+39) as a double
  uint64_t v = 0;
  for (int b = 0; b < CRT_BITS; b++) {
    int bit = c * CRT_BITS + b;
    size_t w = bit / 32;
    if (w < a.d.size() && ((a.d[w] >> (bit % 32)) & 1u)) v |= (1ull << b);
  }
  return (double)v;
}
static int64_t modinv(int64_t a, int64_t m) {
  int64_t g = m, x = 0, x1 = 1, a1 = a % m;
  while (a1) {
    int64_t q = g / a1;
    int64_t t = g - q * a1;
    g = a1;
    a1 = t;
    t = x - q * x1;
    x = x1;
    x1 = t;
  }
  return ((x % m) + m) % m;
}

static const HostTables& host_tables() {
  static HostTables T;
  static std::once_flag once;
  std::call_once(once, [] {
    // Greedy pairwise-coprime moduli from 256 down.
    std::vector<int> mods;
    for (int m = 256; m > 1 && (int)mods.size() < MAXL; m--) {
      bool ok = true;
      for (int x : mods)
        if (std::__gcd(x, m) != 1) ok = false;
      if (ok) mods.push_back(m);
    }
    T.cum_log2[0] = 0;
    for (int l = 0; l < MAXL; l++) {
      int m = mods[l];
      T.mt.mod[l] = m;
      T.mt.magic[l] = (uint32_t)((1ull << 32) / (uint64_t)m);
      T.mt.offset[l] = (uint32_t)((((1ull << 31) + m - 1) / m) * m);
      for (int c = 0; c < NDIG2; c++) {
        // 2^(22c) mod m, balanced
        uint64_t r = 1;
        for (int t = 0; t < 22 * c; t++) r = (r * 2) % m;
        int b = (int)r;
        if (b > m / 2) b -= m;
        T.mt.pw[l][c] = b;
      }
      for (int c = 0; c < 5; c++) {
        uint64_t r = 1;
        for (int t = 0; t < 21 * c; t++) r = (r * 2) % m;
        int b = (int)r;
        if (b > m / 2) b -= m;
        T.mt.pw21[l][c] = b;
      }
      T.cum_log2[l + 1] = T.cum_log2[l] + std::log2((double)m);
    }
    T.crt.resize(MAXL + 1);
    for (int L = 1; L <= MAXL; L++) {
      CrtTable& ct = T.crt[L];
      std::memset(&ct, 0, sizeof(ct));
      ct.L = L;
      Big M;
      M.d = {1};
      for (int l = 0; l < L; l++) big_mul_small(M, (uint32_t)mods[l]);
      int bits = (int)M.d.size() * 32;
      while (bits > 0 && !((M.d[(bits - 1) / 32] >> ((bits - 1) % 32)) & 1u)) bits--;
      ct.nc = (bits + CRT_BITS - 1) / CRT_BITS;
      for (int c = 0; c < ct.nc; c++) ct.mchunk[c] = big_chunk(M, c);
      {  // 1/M, rounded
        long double mv = 0;
        for (size_t i = M.d.size(); i-- > 0;) mv = mv * 4294967296.0L + (long double)M.d[i];
        ct.inv_m = (double)(1.0L / mv);
      }
      for (int l = 0; l < L; l++) {
        Big P = big_div_small(M, (uint32_t)mods[l]);
        int64_t pm = big_mod_small(P, (uint32_t)mods[l]);
        int64_t inv = modinv(pm, mods[l]);
        Big W = P;
        big_mul_small(W, (uint32_t)inv);  // < M since inv < m_l
        for (int c = 0; c < ct.nc; c++) ct.w[l][c] = big_chunk(W, c);
        if (L >= CRT_CONST_L0 && L < CRT_CONST_L0 + CRT_CONST_N) {
          CrtTcTable& tc = T.crt_tc[L - CRT_CONST_L0];
          for (int q = 0; q < 32; q++) {
            const size_t w = (size_t)q / 4;
            tc.wb[q][l] = w < W.d.size() ? (uint8_t)(W.d[w] >> (8 * (q % 4))) : 0;
          }
        }
      }
      if (L >= CRT_CONST_L0 && L < CRT_CONST_L0 + CRT_CONST_N) {
        CrtTcTable& tc = T.crt_tc[L - CRT_CONST_L0];
        for (int h = 0; h < 16; h++) {
          const size_t w = (size_t)h / 2;
          tc.mlimb[h] = w < M.d.size() ? (int32_t)((M.d[w] >> (16 * (h % 2))) & 0xFFFFu) : 0;
        }
        long double mv = 0;
        for (size_t i = M.d.size(); i-- > 0;) mv = mv * 4294967296.0L + (long double)M.d[i];
        tc.k192 = (double)(std::ldexp(1.0L, 192) / mv);
      }
    }
  });
  return T;
}

// Per-device upload of the tables (once per device).
struct DevTables {
  bool ready = false;
  CrtTable* crt = nullptr;
  int num_sms = 0;
};
static DevTables g_dev[64];
static std::mutex g_dev_mu;

static int device_tables(DevTables** out) {
  int d = 0;
  HP_CUDA_TRY(cudaGetDevice(&d));
  std::lock_guard<std::mutex> lk(g_dev_mu);
  DevTables& D = g_dev[d];
  if (!D.ready) {
    const HostTables& T = host_tables();
    HP_CUDA_TRY(cudaMemcpyToSymbol(c_tab, &T.mt, sizeof(ModTable)));
    HP_CUDA_TRY(cudaMemcpyToSymbol(c_crt, &T.crt[CRT_CONST_L0], sizeof(CrtTable) * CRT_CONST_N));
    HP_CUDA_TRY(cudaMemcpyToSymbol(c_crt_tc, T.crt_tc, sizeof(CrtTcTable) * CRT_CONST_N));
    HP_CUDA_TRY(cudaMalloc(&D.crt, sizeof(CrtTable) * (MAXL + 1)));
    HP_CUDA_TRY(cudaMemcpy(D.crt, T.crt.data(), sizeof(CrtTable) * (MAXL + 1), cudaMemcpyHostToDevice));
    HP_CUDA_TRY(cudaDeviceGetAttribute(&D.num_sms, cudaDevAttrMultiProcessorCount, d));
    D.ready = true;
  }
  *out = &D;
  return HP_OK;
}

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int exp_field(double x) {
  return (int)((__double_as_longlong(x) >> 52) & 0x7FF);
}
// x * 2^s for any s in [-2100, 2100], exact when the result is a normal
// number (the scaled integers of this file always are, or are discarded).
__device__ __forceinline__ double scale_pow2(double x, int s) {
  while (s > 1000) {
    x = __dmul_rn(x, 0x1p1000);
    s -= 1000;
  }
  while (s < -1000) {
    x = __dmul_rn(x, 0x1p-1000);
    s += 1000;
  }
  return __dmul_rn(x, __longlong_as_double((long long)(s + 1023) << 52));
}
__device__ __forceinline__ uint32_t mod_reduce(int32_t x, int l) {
  uint32_t u = (uint32_t)(x + (int32_t)0) + c_tab.offset[l];  // x + offset, as unsigned
  uint32_t m = (uint32_t)c_tab.mod[l];
  uint32_t q = __umulhi(u, c_tab.magic[l]);
  uint32_t r = u - q * m;
  return r >= m ? r - m : r;
}

// Exponent pass of the f128 Ozaki GEMM in one launch. A (RA x CA,
// row-major) contributes one exponent per row (a_rows) or per column, B
// (RB x CB) one per column; an entry's exponent is max(e(hi), e(lo) + 1),
// or the non-finite marker. Row blocks: 8 warps, each one chunk of `chunk`
// entries of a row, MAXEXP_U loads in flight per lane. Column blocks: 256
// consecutive columns, one per thread, over a slab of `slab` rows, so a
// block's loads of one row cover 256 contiguous entries (DRAM pages are
// opened for 4-8 KB, not 512 B). Partial maxima merge with atomicMax into
// outputs zeroed beforehand. Blocks [0, na) serve A, the rest B.
__device__ __forceinline__ int entry_exp(double2 v) {
  const int el = exp_field(v.y);
  return el == EXP_NONFINITE ? EXP_NONFINITE : max(exp_field(v.x), min(el + 1, EXP_NONFINITE));
}
// f256 entries: the same from limbs 0 and 1; any non-finite limb marks the entry
__device__ __forceinline__ int entry_exp(double4 v) {
  const int el = exp_field(v.y);
  if (el == EXP_NONFINITE || exp_field(v.z) == EXP_NONFINITE || exp_field(v.w) == EXP_NONFINITE) return EXP_NONFINITE;
  return max(exp_field(v.x), min(el + 1, EXP_NONFINITE));
}
constexpr int MAXEXP_U = 8;       // loads in flight per lane
constexpr int MAXEXP_ROUNDS = 4;  // rounds of MAXEXP_U loads per thread (a row chunk, a column slab)
constexpr int MAXEXP_COLS = 256;  // columns of a column block
template <class T>
__global__ void __launch_bounds__(256) maxexp_kernel(const T* __restrict__ A, int64_t RA, int64_t CA, bool a_rows,
                                                     int* __restrict__ outA, const T* __restrict__ B, int64_t RB,
                                                     int64_t CB, int* __restrict__ outB, int64_t slab, int64_t chunk,
                                                     unsigned na) {
  sm100::griddep_launch_dependents();
  const bool isA = blockIdx.x < na;
  const unsigned bid = isA ? blockIdx.x : blockIdx.x - na;
  const T* src = isA ? A : B;
  const int64_t R = isA ? RA : RB, C = isA ? CA : CB;
  int* out = isA ? outA : outB;
  const int lane = threadIdx.x % 32, wy = threadIdx.x / 32;
  if (isA && a_rows) {
    const int64_t nch = (C + chunk - 1) / chunk;
    const int64_t item = (int64_t)bid * 8 + wy, row = item / nch;
    if (row >= R) return;
    const T* rp = src + row * C;
    const int64_t p0 = (item % nch) * chunk, p1 = min(C, p0 + chunk);
    int e = 0;
    for (int64_t p = p0 + lane; p < p1; p += 32 * MAXEXP_U) {
      T v[MAXEXP_U];
#pragma unroll
      for (int u = 0; u < MAXEXP_U; u++) v[u] = p + 32 * u < p1 ? rp[p + 32 * u] : T{};
#pragma unroll
      for (int u = 0; u < MAXEXP_U; u++) e = max(e, entry_exp(v[u]));
    }
    for (int o = 16; o; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
    if (lane == 0) atomicMax(out + row, e);
    return;
  }
  const int64_t ncb = (C + MAXEXP_COLS - 1) / MAXEXP_COLS;
  const int64_t c = (int64_t)(bid % ncb) * MAXEXP_COLS + threadIdx.x;
  const int64_t r0 = (int64_t)(bid / ncb) * slab, r1 = min(R, r0 + slab);
  if (c >= C) return;
  int e = 0;
  for (int64_t r = r0; r < r1; r += MAXEXP_U) {
    T v[MAXEXP_U];
#pragma unroll
    for (int u = 0; u < MAXEXP_U; u++) v[u] = r + u < r1 ? src[(r + u) * C + c] : T{};
#pragma unroll
    for (int u = 0; u < MAXEXP_U; u++) e = max(e, entry_exp(v[u]));
  }
  atomicMax(out + c, e);
}
// Exponents of the f128 GEMM's operands: expA per row of A (per column when
// atb, A being k x m) and expB per column of B (k x n), both zeroed by the
// caller.
template <class T>
static int launch_maxexp(const T* A, const T* B, size_t m, size_t n, size_t k, bool atb, int* expA, int* expB,
                         cudaStream_t s) {
  const int64_t slab = MAXEXP_ROUNDS * MAXEXP_U, chunk = MAXEXP_ROUNDS * MAXEXP_U * 32;
  const int64_t kslabs = ((int64_t)k + slab - 1) / slab, kchunks = ((int64_t)k + chunk - 1) / chunk;
  const int64_t na = atb ? ((int64_t)m + MAXEXP_COLS - 1) / MAXEXP_COLS * kslabs : ((int64_t)m * kchunks + 7) / 8;
  const int64_t nb = ((int64_t)n + MAXEXP_COLS - 1) / MAXEXP_COLS * kslabs;
  if (na + nb > INT32_MAX) {
    set_error("ozaki: exponent pass grid too large");
    return HP_ERR_INVALID_ARG;
  }
  if (na + nb == 0) return HP_OK;  // nothing to scan (k, or both m and n, zero)
  maxexp_kernel<T><<<(unsigned)(na + nb), 256, 0, s>>>(A, atb ? (int64_t)k : (int64_t)m, atb ? (int64_t)m : (int64_t)k,
                                                    !atb, expA, B, (int64_t)k, (int64_t)n, expB, slab, chunk,
                                                    (unsigned)na);
  HP_LAUNCH_CHECK();
  return HP_OK;
}

// Balanced base-2^22 digits of rint(v) for |v| < 2^108 (exact).
__device__ __forceinline__ void int_digits(double v, int32_t* d) {
  double a = fabs(rint(v));
  double t4 = floor(__dmul_rn(a, 0x1p-88));
  double r = __dsub_rn(a, __dmul_rn(t4, 0x1p88));
  double t3 = floor(__dmul_rn(r, 0x1p-66));
  r = __dsub_rn(r, __dmul_rn(t3, 0x1p66));
  double t2 = floor(__dmul_rn(r, 0x1p-44));
  r = __dsub_rn(r, __dmul_rn(t2, 0x1p44));
  double t1 = floor(__dmul_rn(r, 0x1p-22));
  r = __dsub_rn(r, __dmul_rn(t1, 0x1p22));
  int32_t s = signbit(v) ? -1 : 1;
  d[0] = s * (int32_t)r;
  d[1] = s * (int32_t)t1;
  d[2] = s * (int32_t)t2;
  d[3] = s * (int32_t)t3;
  d[4] = s * (int32_t)t4;
}

// Residues of the scaled operand. Logical operand is R x K (row r, reduction
// index p); element (r, p) is src[r*K + p] (P_CONTIG) or src[p*R + r].
// Writes out[l][r][p] (int8), row stride ld, plane stride plane_stride, for
// every (r, p) the grid covers (64 gridDim.y rows, 32 gridDim.x columns;
// zero outside R x K); blockIdx.z takes the moduli l = z (mod gridDim.z).
// Block tile: 64 rows x 32 p; each thread owns one row and 8 consecutive p,
// so its 8 residues of one modulus pack into two 32-bit words.
//   P_CONTIG: thread reads 8 consecutive f128 (128 B) and stores its 8 bytes
//             straight to global (a warp writes 8 full 32-byte sectors).
//   else:     loads are coalesced along r; the bytes are transposed through
//             shared memory so the global stores run along p.
constexpr int RT_R = 64, RT_P = 32;
__device__ __forceinline__ void element_digits(double2 v, int s, int32_t* D) {
  int32_t dh[NDIG], dl[NDIG];
  int_digits(scale_pow2(v.x, s), dh);
  int_digits(scale_pow2(v.y, s), dl);
#pragma unroll
  for (int c = 0; c < NDIG; c++) D[c] = dh[c] + dl[c];
#pragma unroll
  for (int c = 0; c < NDIG - 1; c++) {
    int32_t carry = (D[c] + (1 << 21)) >> 22;
    D[c] -= carry << 22;
    D[c + 1] += carry;
  }
}
__device__ __forceinline__ uint32_t balanced_byte(const int32_t* D, int l, int m) {
  int32_t x = 0;
#pragma unroll
  for (int c = 0; c < NDIG; c++) x += D[c] * c_tab.pw[l][c];
  int r = (int)mod_reduce(x, l);
  if (r > 127) r -= m;
  return (uint32_t)(r & 0xFF);
}
// One RT_R x (4 EPR) tile (block coordinates bx, by) of the residue planes
// of a scaled f128 operand: EPR entries per thread (8 or 4: fewer digits
// live through the moduli loop, more warps per SM), all L moduli.
// the residue in [0, m) as an unsigned byte (operands of the unsigned MMA)
__device__ __forceinline__ uint32_t unsigned_byte(const int32_t* D, int l) {
  int32_t x = D[0];  // 2^0 mod m = 1
#pragma unroll
  for (int c = 1; c < NDIG; c++) x += D[c] * c_tab.pw[l][c];
  return mod_reduce(x, l);
}
// LC > 0: the number of moduli is the compile-time LC (== L), the moduli
// loop is unrolled (each modulus' constants are immediate operands) and the
// transposed tile keeps all LC planes in shared memory until one barrier.
template <bool P_CONTIG, int EPR, bool U8, int LC = 0>
__device__ __forceinline__ void residue_tile(const double2* __restrict__ src, int64_t R, int64_t K,
                                             const int* __restrict__ expf, int beta, int L, int64_t ld,
                                             int64_t plane_stride, int8_t* __restrict__ out, unsigned bx,
                                             unsigned by) {
  constexpr int NW = EPR / 4;  // 32-bit words (and 16-byte row chunks of the transposed store) per thread
  __shared__ __align__(16) uint32_t T[2][RT_R][EPR + 1];
  const int t = threadIdx.x;
  const int rl = P_CONTIG ? t / 4 : t % 64;
  const int quad = P_CONTIG ? t % 4 : t / 64;
  const int64_t r = (int64_t)by * RT_R + rl;
  const int64_t p0 = (int64_t)bx * (4 * EPR) + EPR * quad;
  int32_t dig[EPR][NDIG];
#pragma unroll
  for (int e = 0; e < EPR; e++)
#pragma unroll
    for (int c = 0; c < NDIG; c++) dig[e][c] = 0;
  // the entries do not depend on the preceding exponent pass: load them
  // before waiting for it
  double2 v[EPR];
#pragma unroll
  for (int e = 0; e < EPR; e++) {
    const int64_t p = p0 + e;
    v[e] = r < R && p < K ? (P_CONTIG ? src[r * K + p] : src[p * R + r]) : make_double2(0.0, 0.0);
  }
  sm100::griddep_launch_dependents();
  sm100::griddep_wait();
  if (r < R) {
    const int ex = expf[r];
    if (ex != EXP_NONFINITE) {
      const int s = beta + 1022 - ex;
#pragma unroll
      for (int e = 0; e < EPR; e++)
        if (p0 + e < K) element_digits(v[e], s, dig[e]);
    }
  }
  int8_t* const base = out + (size_t)by * RT_R * ld + (size_t)bx * (4 * EPR);
  if constexpr (LC > 0) {
    constexpr int TROWS = P_CONTIG ? 1 : RT_R;
    __shared__ uint32_t TT[P_CONTIG ? 1 : LC][TROWS][EPR + 1];
#pragma unroll
    for (int l = 0; l < LC; l++) {
      uint32_t w[NW];
#pragma unroll
      for (int q = 0; q < NW; q++) {
        w[q] = 0;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const uint32_t byte =
              U8 ? unsigned_byte(dig[4 * q + e], l) : balanced_byte(dig[4 * q + e], l, c_tab.mod[l]);
          w[q] |= byte << (8 * e);
        }
      }
      if constexpr (P_CONTIG) {
        int8_t* dst = base + (size_t)l * plane_stride + (size_t)rl * ld + EPR * quad;
        if (NW == 2)
          *reinterpret_cast<uint2*>(dst) = make_uint2(w[0], w[NW - 1]);
        else
          *reinterpret_cast<uint32_t*>(dst) = w[0];
      } else {
#pragma unroll
        for (int q = 0; q < NW; q++) TT[l][rl][NW * quad + q] = w[q];
      }
    }
    if constexpr (!P_CONTIG) {
      __syncthreads();
      for (int u = t; u < LC * RT_R * NW; u += blockDim.x) {
        const int l = u / (RT_R * NW), rem = u % (RT_R * NW), row = rem / NW, half = rem % NW;
        const uint32_t* sw = &TT[l][row][4 * half];
        *reinterpret_cast<uint4*>(base + (size_t)l * plane_stride + (size_t)row * ld + 16 * half) =
            make_uint4(sw[0], sw[1], sw[2], sw[3]);
      }
    }
  } else {
    int it = 0;
    for (int l = 0; l < L; l++, it++) {
      const int m = c_tab.mod[l];
      uint32_t w[NW];
#pragma unroll
      for (int q = 0; q < NW; q++) {
        w[q] = 0;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const uint32_t byte = U8 ? unsigned_byte(dig[4 * q + e], l) : balanced_byte(dig[4 * q + e], l, m);
          w[q] |= byte << (8 * e);
        }
      }
      int8_t* plane = base + (size_t)l * plane_stride;
      if (P_CONTIG) {
        if (NW == 2)
          *reinterpret_cast<uint2*>(plane + (size_t)rl * ld + EPR * quad) = make_uint2(w[0], w[NW - 1]);
        else
          *reinterpret_cast<uint32_t*>(plane + (size_t)rl * ld + EPR * quad) = w[0];
      } else {
#pragma unroll
        for (int q = 0; q < NW; q++) T[it & 1][rl][NW * quad + q] = w[q];
        __syncthreads();
        if (t < NW * RT_R) {
          const int row = t / NW, half = t % NW;
          const uint32_t* src_w = &T[it & 1][row][4 * half];
          *reinterpret_cast<uint4*>(plane + (size_t)row * ld + 16 * half) =
              make_uint4(src_w[0], src_w[1], src_w[2], src_w[3]);
        }
      }
    }
  }
}

// Residues of both operands of the f128 Ozaki GEMM in one launch: block
// rows [0, tiles_ay) cover A (row-contiguous when A_CONTIG), the rest B.
template <bool A_CONTIG, int EPR, bool U8, int LC = 0>
__global__ void __launch_bounds__(256) residue_ab_kernel(const double2* __restrict__ A, int64_t RA,
                                                         const int* __restrict__ expA, int8_t* __restrict__ outA,
                                                         int64_t planeA, unsigned tiles_ay,
                                                         const double2* __restrict__ B, int64_t RB,
                                                         const int* __restrict__ expB, int8_t* __restrict__ outB,
                                                         int64_t planeB, int64_t K, int beta, int L, int64_t ld) {
  if (blockIdx.y < tiles_ay)
    residue_tile<A_CONTIG, EPR, U8, LC>(A, RA, K, expA, beta, L, ld, planeA, outA, blockIdx.x, blockIdx.y);
  else
    residue_tile<false, EPR, U8, LC>(B, RB, K, expB, beta, L, ld, planeB, outB, blockIdx.x, blockIdx.y - tiles_ay);
}

// ---------------------------------------------------------------------------
// Residues on the tensor core (the unsigned residue planes of the f128 GEMM,
// L = 28..32 moduli). An entry's scaled integer X = rint(hi 2^s) +
// rint(lo 2^s), |X| < 2^109, is offset to X' = X + 2^111 in (0, 2^112), and
// its 16 bytes x_0 .. x_13, x_14 = 1, x_15 = 0 form one K-chunk of an MMA
// operand. With the weights w_lb = 2^(8b) mod m_l (b < 14), w_l14 = -2^111
// mod m_l and w_l15 = 0, the sum S_l = sum_b x_b w_lb is congruent to X mod
// m_l, and S_l < 16 * 255^2 < 2^20, so one multiply-high by ceil(2^32 / m_l)
// gives floor(S_l / m_l) exactly and S_l - m_l floor(S_l / m_l) is X's
// residue in [0, m_l), the byte the integer kernel (residue_tile) writes.
// A tile is 8 operand rows x 128 consecutive reduction indices p: TMA brings
// its entries into a 3-stage ring, each thread turns 4 entries into bytes
// (row p of a 128-byte-swizzled 128 x 128 byte tile, 16-byte slot j for
// operand row j), and four M = 128, N = 128, K = 32 MMAs place the sums of
// slot 4a + g, modulus l at TMEM lane 32 g + l of accumulator a: the weight
// tile holds w_l in 16-byte chunk g of row 32 g + l. Warp w then reads lane
// quarter g = w % 4 of accumulator a = w / 4: lane l owns modulus l and 128
// consecutive p of one operand row, reduces them and stores 128 bytes.
// ---------------------------------------------------------------------------
constexpr int RC_THREADS = 256, RC_STAGES = 2, RC_ROWS = 8, RC_P = 128;
constexpr int RC_IN_BYTES = RC_ROWS * RC_P * 16;
constexpr int RC_OUT_PLANE = RC_ROWS * RC_P + 16;  // staged bytes of one modulus (padded: no bank conflicts)
constexpr int RC_SMEM = 1024 + 2 * 128 * 128 + RC_STAGES * RC_IN_BYTES + 32 * RC_OUT_PLANE;

struct ResidueOperand {  // one GEMM operand as the residue kernel sees it
  int8_t* out;           // L planes of rows x ld bytes
  int64_t plane, ld;     // plane stride, row stride (bytes)
  const int* exps;       // per-row exponents
  int64_t row_tiles, p_tiles;  // tiles of RC_ROWS (f256: 4) rows x RC_P reduction indices
  int64_t half;          // f256: byte offset of a row's second half (the two 105-bit halves)
};

// The tiles of a persistent CTA (first, first + stride, ...) in a grid of
// `cols` tiles per row, walked without a division per step.
struct TileWalk {
  int64_t r, c, dr, dc, cols;
  __device__ __forceinline__ TileWalk(int64_t first, int64_t stride, int64_t cols_)
      : r(first / cols_), c(first % cols_), dr(stride / cols_), dc(stride % cols_), cols(cols_) {}
  __device__ __forceinline__ void next() {
    c += dc;
    r += dr;
    if (c >= cols) {
      c -= cols;
      r++;
    }
  }
};
// A ring position: stage index and the parity of its current use.
struct RingPos {
  int st = 0;
  uint32_t ph = 0;
  template <int S>
  __device__ __forceinline__ void next() {
    if (++st == S) {
      st = 0;
      ph ^= 1u;
    }
  }
};

// |x| < 2^108, integer-valued: x as a two's-complement 128-bit integer
__device__ __forceinline__ void int128_of(double x, uint64_t& lo, uint64_t& hi) {
  const double a = fabs(x);
  const double th = floor(__dmul_rn(a, 0x1p-64));        // exact
  const double rh = __dsub_rn(a, __dmul_rn(th, 0x1p64));  // a mod 2^64, exact
  lo = __double2ull_rz(rh);
  hi = __double2ull_rz(th);
  if (signbit(x)) {
    lo = ~lo + 1ull;
    hi = ~hi + (lo == 0ull ? 1ull : 0ull);
  }
}

// 128-bit two's-complement (lo, hi) += (a0, a1)
__device__ __forceinline__ void add128(uint64_t& lo, uint64_t& hi, uint64_t a0, uint64_t a1) {
  lo += a0;
  hi += a1 + (lo < a0 ? 1ull : 0ull);
}

// QD: the f256 operands. An entry is 4 limbs; its scaled integer
// X = sum_q rint(limb_q 2^s), |X| <= 2^210 + 2^157, is split exactly as
// X = Xh 2^105 + Xl with Xl = X mods 2^105 in [-2^104, 2^104): each limb's
// integer v is split by truncation, v = vh 2^105 + vl (both exact doubles),
// the vh and the vl are summed in 128-bit integers, and the vl sum is brought
// into range with its carry moved to Xh. Xh and Xl each take one 16-byte slot
// of the entry-byte tile (tiles of 4 operand rows x 128 p: 8 slots), and go
// to the two halves of the row (A: [Xh | Xl], B: [Yl | Yh], `half` bytes
// apart), as the f256 GEMM's residue GEMMs read them.
template <int LC, bool A_CONTIG, bool QD = false>
__global__ void __launch_bounds__(RC_THREADS, 2)
    residue_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                      ResidueOperand opA, ResidueOperand opB, int beta, uint32_t* status) {
  using namespace sm100;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t* sW = smem_raw + pad;    // weights: 128 rows x 128 bytes, swizzled
  uint8_t* sE = sW + 128 * 128;    // entry bytes: 128 rows (p) x 8 slots (operand rows), swizzled
  uint8_t* sIn = sE + 128 * 128;   // RC_STAGES x 1024 entries as loaded
  uint8_t* sOut = sIn + RC_STAGES * RC_IN_BYTES;  // the tile's residue bytes, per modulus 8 rows x 128
  __shared__ uint64_t full[RC_STAGES], mdone;
  __shared__ uint32_t tmem_slot;
  const int t = threadIdx.x, warp = t / 32, lane = t % 32;
  auto swz = [](int row, int chunk) { return (row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4); };
  // weight tile: row 32 g + l, 16-byte chunk g = w_l (modulus l < LC); zero elsewhere
  for (int e = t; e < 128 * 8; e += RC_THREADS) *reinterpret_cast<uint4*>(sW + 16 * e) = make_uint4(0, 0, 0, 0);
  __syncthreads();
  if (t < 128 && t % 32 < LC) {
    const int g = t / 32, l = t % 32;
    const uint32_t m = (uint32_t)c_tab.mod[l];
    uint32_t w[4] = {0, 0, 0, 0}, p = 1, p104 = 1;
    for (int b = 0; b < 14; b++) {
      w[b / 4] |= p << (8 * (b % 4));
      p104 = p;
      p = (p * 256u) % m;
    }
    const uint32_t c111 = (p104 * 128u) % m;  // 2^111 mod m
    w[3] |= ((m - c111) % m) << 16;           // byte 14
    *reinterpret_cast<uint4*>(sW + swz(t, g)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  if (t == 0) {
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
    for (int s = 0; s < RC_STAGES; s++) mbar_init(&full[s], 1);
    mbar_init(&mdone, 1);
    fence_mbarrier_init();
  }
  if (warp == 0) {
    tmem_alloc(&tmem_slot, 256);
    tmem_relinquish();
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  // this thread's modulus in the epilogue
  const int el = lane;
  const uint32_t em = el < LC ? (uint32_t)c_tab.mod[el] : 1u;
  const uint32_t emag = el < LC ? 0xFFFFFFFFu / em + 1u : 0u;  // ceil(2^32 / m)
  griddep_launch_dependents();
  griddep_wait();  // the exponents come from the preceding pass
  // tiles: row tiles of A then of B (both with opA.p_tiles reduction tiles), reduction tile fastest
  const int64_t P = opA.p_tiles, rowsA = opA.row_tiles, ntiles = (rowsA + opB.row_tiles) * P;
  const int64_t cnt = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  TileWalk prod(blockIdx.x, gridDim.x, P), cons(blockIdx.x, gridDim.x, P);
  RingPos pring, cring;
  auto issue = [&]() {  // thread 0: entries of the next tile into the next stage
    const bool isA = prod.r < rowsA;
    const int rt = (int)(isA ? prod.r : prod.r - rowsA), pt = (int)prod.c;
    uint8_t* dst = sIn + pring.st * RC_IN_BYTES;
    mbar_arrive_expect_tx(&full[pring.st], (uint32_t)RC_IN_BYTES);
    if constexpr (QD) {  // 3-D view: 4 limbs x entries x rows
      if (isA && A_CONTIG)
        tma_load_3d(dst, &mapA, &full[pring.st], 0, RC_P * pt, 4 * rt);
      else
        tma_load_3d(dst, isA ? &mapA : &mapB, &full[pring.st], 0, 4 * rt, RC_P * pt);
    } else {
      if (isA && A_CONTIG)
        tma_load_2d(dst, &mapA, &full[pring.st], 2 * RC_P * pt, RC_ROWS * rt);
      else
        tma_load_2d(dst, isA ? &mapA : &mapB, &full[pring.st], 2 * RC_ROWS * rt, RC_P * pt);
    }
    prod.next();
    pring.next<RC_STAGES>();
  };
  int64_t issued = 0;
  if (t == 0)
    for (; issued < cnt && issued < RC_STAGES; issued++) issue();
  const uint32_t idesc = idesc_i8(128, 128, true);
  bool ok = true;
  int64_t mma_issued = 0, mma_seen = 0;
  for (int64_t u = 0; u < cnt; u++) {
    const bool isA = cons.r < rowsA;
    const ResidueOperand& o = isA ? opA : opB;
    const int64_t rt = isA ? cons.r : cons.r - rowsA, pt = cons.c;
    cons.next();
    const bool contig = isA && A_CONTIG;
    constexpr int TR = QD ? 4 : RC_ROWS, NE = QD ? 2 : 4;  // operand rows per tile, entries per thread
    int exs[NE];  // the exponents of this thread's entries' rows, loaded before the wait
#pragma unroll
    for (int i = 0; i < NE; i++) {
      const int k = t + RC_THREADS * i;
      exs[i] = o.exps[rt * TR + (contig ? k / RC_P : k % TR)];
    }
    const int st = cring.st;
    if (!mbar_wait(&full[st], cring.ph, status, DEV_STATUS_TIMEOUT)) ok = false;
    cring.next<RC_STAGES>();
    if constexpr (QD) {
      if (ok) {
        const double4* in = reinterpret_cast<const double4*>(sIn + st * RC_IN_BYTES);
#pragma unroll
        for (int i = 0; i < NE; i++) {
          const int k = t + RC_THREADS * i;
          const int j = contig ? k / RC_P : k % TR, n = contig ? k % RC_P : k / TR;
          const double4 v = in[k];
          const int ex = exs[i];
          uint64_t h0 = 0, h1 = 0, x0 = 0, x1 = 0;  // Xh, Xl (zero for a non-finite row)
          if (ex != EXP_NONFINITE) {
            const int s = beta + 1022 - ex;
            const double lim[4] = {v.x, v.y, v.z, v.w};
            uint64_t l0 = 0, l1 = 0;
#pragma unroll
            for (int q = 0; q < 4; q++) {
              const double xq = rint(scale_pow2(lim[q], s));
              const double vh = trunc(__dmul_rn(xq, 0x1p-105));        // exact
              const double vl = __dsub_rn(xq, __dmul_rn(vh, 0x1p105));  // exact, |vl| < 2^105
              uint64_t a0, a1;
              int128_of(vh, a0, a1);
              add128(h0, h1, a0, a1);
              int128_of(vl, a0, a1);
              add128(l0, l1, a0, a1);
            }
            x0 = l0;  // Xl: the low 105 bits, sign-extended from bit 104
            x1 = l1 & ((1ull << 41) - 1);
            if (x1 >> 40) x1 |= ~((1ull << 41) - 1);
            const int64_t carry = (int64_t)(l1 - x1) >> 41;  // (sum - Xl) / 2^105 (low word cancels)
            add128(h0, h1, (uint64_t)carry, carry < 0 ? ~0ull : 0ull);
          }
          // X' = X + 2^111 for each half; A: slot 2j = Xh, 2j + 1 = Xl; B: slot 2j = Yl, 2j + 1 = Yh
          const uint64_t hw1 = h1 + (1ull << 47), xw1 = x1 + (1ull << 47);
          const uint4 bh = make_uint4((uint32_t)h0, (uint32_t)(h0 >> 32), (uint32_t)hw1,
                                      (uint32_t)((hw1 >> 32) & 0xFFFFu) | 0x10000u);
          const uint4 bl = make_uint4((uint32_t)x0, (uint32_t)(x0 >> 32), (uint32_t)xw1,
                                      (uint32_t)((xw1 >> 32) & 0xFFFFu) | 0x10000u);
          *reinterpret_cast<uint4*>(sE + swz(n, 2 * j)) = isA ? bh : bl;
          *reinterpret_cast<uint4*>(sE + swz(n, 2 * j + 1)) = isA ? bl : bh;
        }
      }
    } else {
      if (ok) {
        const double2* in = reinterpret_cast<const double2*>(sIn + st * RC_IN_BYTES);
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int k = t + RC_THREADS * i;
          const int j = contig ? k / RC_P : k % RC_ROWS, n = contig ? k % RC_P : k / RC_ROWS;
          const double2 v = in[k];
          const int ex = exs[i];
          uint64_t w0 = 0, w1 = 1ull << 47;  // X' = X + 2^111 (X = 0 for a non-finite row)
          if (ex != EXP_NONFINITE) {
            const int s = beta + 1022 - ex;
            uint64_t hl, hh, ll, lh;
            int128_of(rint(scale_pow2(v.x, s)), hl, hh);
            int128_of(rint(scale_pow2(v.y, s)), ll, lh);
            w0 = hl + ll;
            w1 = hh + lh + (w0 < hl ? 1ull : 0ull) + (1ull << 47);
          }
          *reinterpret_cast<uint4*>(sE + swz(n, j)) =
              make_uint4((uint32_t)w0, (uint32_t)(w0 >> 32), (uint32_t)w1, (uint32_t)((w1 >> 32) & 0xFFFFu) | 0x10000u);
        }
    
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    ok = __syncthreads_and(ok) != 0;  // entry tile written; the previous tile's TMEM read out
    tc_fence_after();
    if (!ok) break;
    if (t == 0) {
      const uint32_t wa = smem_u32(sW), ea = smem_u32(sE);
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int c = 0; c < 2; c++)
          mma_i8(tmem + (uint32_t)a * 128u, desc_k_sw128(wa + 32 * c), desc_k_sw128(ea + 32 * (2 * a + c)), idesc,
                 (uint32_t)c);
      mma_commit(&mdone);
      mma_issued++;
      if (issued < cnt) {  // refill the stage just read
        issue();
        issued++;
      }
    }
    bool got = mbar_wait(&mdone, (uint32_t)(u & 1), status, DEV_STATUS_TIMEOUT);
    if (!__syncthreads_and(got)) {
      ok = false;
      break;
    }
    mma_seen = u + 1;
    tc_fence_after();
    // epilogue: lane quarter g of accumulator a = operand row 4 a + g of the
    // tile; the bytes are staged so that the global stores run along rows
    const int g = warp % 4, a = warp / 4;
    uint8_t* so = sOut + el * RC_OUT_PLANE + (4 * a + g) * RC_P;
#pragma unroll
    for (int c2 = 0; c2 < 4; c2 += 2) {
      uint32_t v[2][32];
      const uint32_t col = tmem + (uint32_t)a * 128u + 32u * c2 + ((uint32_t)(32 * g) << 16);
      tmem_ld_32x32b_x32(col, v[0]);
      tmem_ld_32x32b_x32(col + 32u, v[1]);
      tmem_wait_ld();
      if (el < LC) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
          uint32_t wds[8];
#pragma unroll
          for (int q = 0; q < 8; q++) {
            uint32_t r[4];
#pragma unroll
            for (int e = 0; e < 4; e++) r[e] = v[h][4 * q + e] - __umulhi(v[h][4 * q + e], emag) * em;
            wds[q] = __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
          }
          uint8_t* d = so + 32 * (c2 + h);
          *reinterpret_cast<uint4*>(d) = make_uint4(wds[0], wds[1], wds[2], wds[3]);
          *reinterpret_cast<uint4*>(d + 16) = make_uint4(wds[4], wds[5], wds[6], wds[7]);
        }
      }
    }
    tc_fence_before();
    __syncthreads();  // the tile's bytes staged (and its TMEM read out)
    // full 128-byte rows of every plane, 8 threads per row
    int8_t* ob = o.out + (size_t)(rt * TR) * o.ld + (size_t)pt * RC_P;
#pragma unroll 2
    for (int e = t; e < LC * RC_ROWS * 8; e += RC_THREADS) {
      const int l = e >> 6, j = (e >> 3) & 7, c = e & 7;  // plane, slot, 16-byte piece
      const uint4 val = *reinterpret_cast<const uint4*>(sOut + l * RC_OUT_PLANE + j * RC_P + 16 * c);
      const size_t at = QD ? (size_t)(j >> 1) * o.ld + (size_t)(j & 1) * o.half : (size_t)j * o.ld;
      *reinterpret_cast<uint4*>(ob + (size_t)l * o.plane + at + 16 * c) = val;
    }
  }
  if (!ok && t == 0) {
    // a wait gave up: let the copies and the MMAs still in flight land (bounded) before the buffers go
    for (int64_t u = mma_issued; u < issued; u++)
      mbar_wait(&full[(int)(u % RC_STAGES)], (uint32_t)((u / RC_STAGES) & 1), status, DEV_STATUS_TIMEOUT,
                100000000ull);
    if (mma_issued > mma_seen)
      mbar_wait(&mdone, (uint32_t)((mma_issued - 1) & 1), status, DEV_STATUS_TIMEOUT, 100000000ull);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// ---------------------------------------------------------------------------
// tcgen05 int8 GEMM, one modulus per output tile:
//   cres[l][i][j] = (sum_p Ares[l][i][p] * Bres[l][j][p]) mod m_l   (uint8)
// Persistent, warp-specialised: warp 0 = TMA producer, warp 1 = MMA issuer,
// warp 2 = TMEM owner, warps 4-7 = epilogue (TMEM -> residue bytes).
// Tile 128 x BN (GemmCfg), K-block 128 bytes, smem ring, 2 TMEM accumulators.
// ---------------------------------------------------------------------------
constexpr int GB_M = 128, GB_N = 256, GB_K = 128, GSTAGES = 4;
constexpr int A_STAGE = GB_M * GB_K, B_STAGE = GB_N * GB_K, STAGE_BYTES = A_STAGE + B_STAGE;
constexpr int GEMM_SMEM = GSTAGES * STAGE_BYTES + 1024 + 256;
constexpr int MAX_K_CHUNK = 65536;  // signed operands: |int32 accumulator| <= 2^16 * 2^14 = 2^30
// unsigned operands (residues in [0, m)): accumulator <= 2^15 * 255^2 < 2^31,
// and mod_reduce's offset keeps it below 2^32
constexpr int MAX_K_CHUNK_U8 = 32768;

// Tile shapes: BN = 256 (4-stage ring, the general GEMM) or BN = 64 (8-stage
// ring, for the 64-column panels of the residue-domain Cholesky). The
// accumulators take 2 * BN TMEM columns (two tiles in flight).
template <int BN>
struct GemmCfg {
  static constexpr int STAGES = BN >= 256 ? 4 : 8;
  static constexpr int B_STAGE = BN * GB_K;
  static constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
  static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + 256;
  static constexpr int TMEM_COLS = 2 * BN;
};
static_assert(GemmCfg<256>::SMEM == GEMM_SMEM, "BN = 256 keeps the general GEMM's layout");

template <int BN, bool U8 = false>
__global__ void __launch_bounds__(256, 1)
    i8_gemm_mod_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int L,
                       int tiles_m, int tiles_n, int kb0, int kb1, int kb_off_b, int acc_mode,
                       uint8_t* __restrict__ cres,
                       int64_t ldc, int64_t plane, int64_t c_row0, int64_t c_col0, uint32_t* status) {
  using namespace sm100;
  using Cfg = GemmCfg<BN>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t* smem = smem_raw + pad;
  uint8_t* sA = smem;
  uint8_t* sB = smem + Cfg::STAGES * A_STAGE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::STAGES * Cfg::STAGE_BYTES);
  uint64_t* full = bars;
  uint64_t* empty = bars + Cfg::STAGES;
  uint64_t* tfull = bars + 2 * Cfg::STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 128);
    }
    mbar_init(drain, 1);
    fence_mbarrier_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
  }
  if (warp == 2) {
    tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  // set-up done; inputs and the residues it updates may come from the
  // preceding kernel of a programmatic launch
  griddep_launch_dependents();
  griddep_wait();

  const int nkb = kb1 - kb0;
  const int per_l = tiles_m * tiles_n;
  const int num_tiles = L * per_l;

  if (warp == 0) {
    if (lane == 0) {
      uint32_t stage = 0, phase = 0;
      bool ok = true;
      int filled_phase[Cfg::STAGES];
      for (int s = 0; s < Cfg::STAGES; s++) filled_phase[s] = -1;
      for (int t = blockIdx.x; t < num_tiles && ok; t += gridDim.x) {
        const int l = t / per_l, rem = t % per_l, tm = rem / tiles_n, tn = rem % tiles_n;
        for (int kb = 0; kb < nkb; kb++) {
          if (!mbar_wait(&empty[stage], phase ^ 1, status, DEV_STATUS_TIMEOUT)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[stage], Cfg::STAGE_BYTES);
          tma_load_3d(sA + stage * A_STAGE, &mapA, &full[stage], (kb0 + kb) * GB_K, tm * GB_M, l);
          tma_load_3d(sB + stage * Cfg::B_STAGE, &mapB, &full[stage], (kb0 + kb + kb_off_b) * GB_K, tn * BN, l);
          filled_phase[stage] = (int)phase;
          if (++stage == Cfg::STAGES) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
      if (!ok) {  // let loads still in flight land before the CTA exits
        for (int s = 0; s < Cfg::STAGES; s++)
          if (filled_phase[s] >= 0) mbar_wait(&full[s], (uint32_t)filled_phase[s], status, DEV_STATUS_TIMEOUT, 100000000ull);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t stage = 0, phase = 0, it = 0;
      bool ok = true;
      bool issued = false;
      const uint32_t idesc = idesc_i8(GB_M, BN, U8);
      for (int t = blockIdx.x; t < num_tiles && ok; t += gridDim.x, it++) {
        const uint32_t acc = it & 1, aph = (it >> 1) & 1;
        if (!mbar_wait(&tempty[acc], aph ^ 1, status, DEV_STATUS_TIMEOUT)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + acc * BN;
        for (int kb = 0; kb < nkb; kb++) {
          if (!mbar_wait(&full[stage], phase, status, DEV_STATUS_TIMEOUT)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(sA + stage * A_STAGE), b0 = smem_u32(sB + stage * Cfg::B_STAGE);
#pragma unroll
          for (int kk = 0; kk < GB_K / 32; kk++)
            mma_i8(d, desc_k_sw128(a0 + kk * 32), desc_k_sw128(b0 + kk * 32), idesc, (kb | kk) ? 1u : 0u);
          issued = true;
          mma_commit(&empty[stage]);
          if (++stage == Cfg::STAGES) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (!ok) break;
        mma_commit(&tfull[acc]);
      }
      if (!ok && issued) {  // wait for issued MMAs before TMEM is released
        mma_commit(drain);
        mbar_wait(drain, 0, status, DEV_STATUS_TIMEOUT, 100000000ull);
      }
    }
  } else if (warp >= 4) {
    const int ew = warp - 4;
    uint32_t it = 0;
    for (int t = blockIdx.x; t < num_tiles; t += gridDim.x, it++) {
      const int l = t / per_l, rem = t % per_l, tm = rem / tiles_n, tn = rem % tiles_n;
      const uint32_t acc = it & 1, aph = (it >> 1) & 1;
      const uint32_t m = (uint32_t)c_tab.mod[l];
      const int64_t row = c_row0 + (int64_t)tm * GB_M + ew * 32 + lane;
      uint8_t* dst = cres + (size_t)l * plane + (size_t)row * ldc + (size_t)(c_col0 + (int64_t)tn * BN);
      // read-modify-write tiles: fetch this row's 256 old bytes before waiting
      // for the accumulator, so the loads overlap the MMAs
      uint4 prev[BN / 16];
      if (acc_mode) {
#pragma unroll
        for (int q = 0; q < BN / 16; q++) prev[q] = *reinterpret_cast<const uint4*>(dst + 16 * q);
      }
      bool ok = mbar_wait(&tfull[acc], aph, status, DEV_STATUS_TIMEOUT);
      if (!__all_sync(0xffffffffu, ok)) break;
      tc_fence_after();
#pragma unroll
      for (int ch = 0; ch < BN / 32; ch++) {
        uint32_t v[32];
        tmem_ld_32x32b_x32(tmem_base + ((uint32_t)(ew * 32) << 16) + acc * BN + ch * 32, v);
        tmem_wait_ld();
        uint32_t packed[8];
        uint4 prev0 = make_uint4(0, 0, 0, 0), prev1 = make_uint4(0, 0, 0, 0);
        if (acc_mode) {
#pragma unroll
          for (int q = 0; q < BN / 32; q++)
            if (q == ch) {
              prev0 = prev[2 * q];
              prev1 = prev[2 * q + 1];
            }
        }
        const uint32_t pv[8] = {prev0.x, prev0.y, prev0.z, prev0.w, prev1.x, prev1.y, prev1.z, prev1.w};
#pragma unroll
        for (int w = 0; w < 8; w++) {
          uint32_t word = 0;
#pragma unroll
          for (int b = 0; b < 4; b++) {
            uint32_t r = mod_reduce((int32_t)v[4 * w + b], l);
            if (acc_mode == 1) {  // C = (C + AB) mod m
              r += (pv[w] >> (8 * b)) & 0xFFu;
              if (r >= m) r -= m;
            } else if (acc_mode == 2) {  // C = (C - AB) mod m
              const uint32_t old = (pv[w] >> (8 * b)) & 0xFFu;
              r = old >= r ? old - r : old + m - r;
            }
            word |= r << (8 * b);
          }
          packed[w] = word;
        }
        *reinterpret_cast<uint4*>(dst + ch * 32) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        *reinterpret_cast<uint4*>(dst + ch * 32 + 16) = make_uint4(packed[4], packed[5], packed[6], packed[7]);
      }
      tc_fence_before();
      mbar_arrive(&tempty[acc]);
    }
  }
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    tmem_dealloc(tmem_base, Cfg::TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// The same residue GEMM on CTA pairs (a cluster of 2, tcgen05 cta_group::2):
// a pair computes a 256 x 256 tile of one modulus; each CTA holds 128 rows
// of the A tile and 128 rows of the B tile per K-block and its 128 x 256
// half of the accumulator. Against the one-CTA kernel (128 x 256 per SM)
// every SM stages half as many B bytes per MMA, so the shared memory that
// TMA writes and the tensor core reads carries 8 KB instead of 12 KB per
// 2 M int8 multiply-adds. Roles: warp 0 of each CTA issues its own TMA
// loads, counted on the even CTA's barrier (which expects both CTAs'
// bytes); warp 1 of the even CTA issues the pair MMAs and commits to both
// CTAs' barriers; warps 4-11 of each CTA reduce their half of the
// accumulator mod m (warps 4-7 columns 0-127, warps 8-11 columns 128-255:
// TMEM lane group = warp index mod 4) and arrive on the even CTA's
// accumulator-free barrier.
// Waits are bounded as in the one-CTA kernel; every thread of both CTAs
// meets at a cluster barrier before the TMEM is released.
// ---------------------------------------------------------------------------
constexpr int GP_M = 256, GP_N = 256, GP_HALF = 128, GP_STAGES = 6;
constexpr int GP_THREADS = 384, GP_EPI_THREADS = 256;  // per CTA: warps 4-11 run the epilogue
constexpr int GP_STAGE = 2 * GP_HALF * GB_K;  // A half + B half, bytes per CTA per stage
constexpr int GP_SMEM = GP_STAGES * GP_STAGE + 1024 + 256;
static_assert(GP_SMEM <= 227 * 1024, "pair GEMM stages fit the shared memory of one CTA");

template <bool U8>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(GP_THREADS, 1)
    i8_gemm_pair_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int L,
                        int tiles_m, int tiles_n, int kb0, int kb1, int acc_mode, uint8_t* __restrict__ cres,
                        int64_t ldc, int64_t plane, uint32_t* status) {
  using namespace sm100;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t* smem = smem_raw + pad;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + GP_STAGES * GP_STAGE);
  uint64_t* full = bars;
  uint64_t* empty = bars + GP_STAGES;
  uint64_t* tfull = bars + 2 * GP_STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  if (threadIdx.x == 0) {
    for (int st = 0; st < GP_STAGES; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 2 * GP_EPI_THREADS);
    }
    mbar_init(drain, 1);
    fence_mbarrier_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
  }
  if (warp == 2) {
    tmem_alloc_pair(tmem_slot, 2 * GP_N);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync_all();  // barriers initialised and TMEM allocated in both CTAs
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  griddep_launch_dependents();
  griddep_wait();

  const int pair = blockIdx.x / 2, npairs = gridDim.x / 2;
  const int nkb = kb1 - kb0;
  const int per_l = tiles_m * tiles_n;
  const int num_tiles = L * per_l;
  bool stalled = false;  // this thread gave up a wait

  if (warp == 0) {
    if (lane == 0) {
      uint32_t stage = 0, phase = 0;
      const uint32_t full0 = mapa_shared(smem_u32(full), 0);
      for (int t = pair; t < num_tiles && !stalled; t += npairs) {
        const int l = t / per_l, rem = t % per_l, tm = rem / tiles_n, tn = rem % tiles_n;
        for (int kb = 0; kb < nkb; kb++) {
          if (!mbar_wait(&empty[stage], phase ^ 1, status, DEV_STATUS_TIMEOUT)) {
            stalled = true;
            break;
          }
          if (leader) mbar_arrive_expect_tx(&full[stage], 2 * GP_STAGE);
          uint8_t* sA = smem + stage * GP_STAGE;
          const uint32_t bar = full0 + stage * (uint32_t)sizeof(uint64_t);
          tma_load_3d_pair(sA, &mapA, bar, (kb0 + kb) * GB_K, tm * GP_M + (int)rank * GP_HALF, l);
          tma_load_3d_pair(sA + GP_HALF * GB_K, &mapB, bar, (kb0 + kb) * GB_K, tn * GP_N + (int)rank * GP_HALF, l);
          if (++stage == GP_STAGES) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && leader) {
      uint32_t stage = 0, phase = 0, it = 0;
      bool issued = false;
      const uint32_t idesc = idesc_i8(GP_M, GP_N, U8);
      for (int t = pair; t < num_tiles && !stalled; t += npairs, it++) {
        const uint32_t acc = it & 1, aph = (it >> 1) & 1;
        if (!mbar_wait(&tempty[acc], aph ^ 1, status, DEV_STATUS_TIMEOUT)) {
          stalled = true;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + acc * GP_N;
        for (int kb = 0; kb < nkb; kb++) {
          if (!mbar_wait(&full[stage], phase, status, DEV_STATUS_TIMEOUT)) {
            stalled = true;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(smem + stage * GP_STAGE), b0 = a0 + GP_HALF * GB_K;
#pragma unroll
          for (int kk = 0; kk < GB_K / 32; kk++)
            mma_i8_pair(d, desc_k_sw128(a0 + kk * 32), desc_k_sw128(b0 + kk * 32), idesc, (kb | kk) ? 1u : 0u);
          issued = true;
          mma_commit_pair(&empty[stage], 0x3);
          if (++stage == GP_STAGES) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (stalled) break;
        mma_commit_pair(&tfull[acc], 0x3);
      }
      if (stalled && issued) {  // wait for issued MMAs before TMEM is released
        mma_commit_pair(drain, 0x1);
        mbar_wait(drain, 0, status, DEV_STATUS_TIMEOUT, 100000000ull);
      }
    }
  } else if (warp >= 4) {
    const int ew = warp % 4;                  // TMEM lane group
    const int cbase = warp >= 8 ? GP_N / 2 : 0;  // this warp's 128 columns
    constexpr int EC = GP_N / 2;
    uint32_t it = 0;
    const uint32_t tempty0 = mapa_shared(smem_u32(tempty), 0);
    for (int t = pair; t < num_tiles; t += npairs, it++) {
      const int l = t / per_l, rem = t % per_l, tm = rem / tiles_n, tn = rem % tiles_n;
      const uint32_t acc = it & 1, aph = (it >> 1) & 1;
      const uint32_t m = (uint32_t)c_tab.mod[l];
      const int64_t row = (int64_t)tm * GP_M + (int64_t)rank * GP_HALF + ew * 32 + lane;
      uint8_t* dst = cres + (size_t)l * plane + (size_t)row * ldc + (size_t)tn * GP_N + cbase;
      uint4 prev[EC / 16];
      if (acc_mode) {
#pragma unroll
        for (int q = 0; q < EC / 16; q++) prev[q] = *reinterpret_cast<const uint4*>(dst + 16 * q);
      }
      const bool ok = mbar_wait(&tfull[acc], aph, status, DEV_STATUS_TIMEOUT);
      if (!__all_sync(0xffffffffu, ok)) break;
      tc_fence_after();
#pragma unroll
      for (int ch = 0; ch < EC / 32; ch++) {
        uint32_t v[32];
        tmem_ld_32x32b_x32(tmem_base + ((uint32_t)(ew * 32) << 16) + acc * GP_N + cbase + ch * 32, v);
        tmem_wait_ld();
        uint4 prev0 = make_uint4(0, 0, 0, 0), prev1 = make_uint4(0, 0, 0, 0);
        if (acc_mode) {
#pragma unroll
          for (int q = 0; q < EC / 32; q++)
            if (q == ch) {
              prev0 = prev[2 * q];
              prev1 = prev[2 * q + 1];
            }
        }
        const uint32_t pv[8] = {prev0.x, prev0.y, prev0.z, prev0.w, prev1.x, prev1.y, prev1.z, prev1.w};
        uint32_t packed[8];
#pragma unroll
        for (int w = 0; w < 8; w++) {
          uint32_t word = 0;
#pragma unroll
          for (int b = 0; b < 4; b++) {
            uint32_t r = mod_reduce((int32_t)v[4 * w + b], l);
            if (acc_mode) {  // C = (C + AB) mod m (a later K-chunk)
              r += (pv[w] >> (8 * b)) & 0xFFu;
              if (r >= m) r -= m;
            }
            word |= r << (8 * b);
          }
          packed[w] = word;
        }
        *reinterpret_cast<uint4*>(dst + ch * 32) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        *reinterpret_cast<uint4*>(dst + ch * 32 + 16) = make_uint4(packed[4], packed[5], packed[6], packed[7]);
      }
      tc_fence_before();
      mbar_arrive_cluster(tempty0 + acc * (uint32_t)sizeof(uint64_t));
    }
  }
  if (stalled) {  // let loads this CTA issued land before its shared memory goes away
    for (int q = 0; q < 1000; q++) __nanosleep(1000);
  }
  __syncthreads();
  tc_fence_before();
  cluster_sync_all();  // both CTAs done with the MMAs and their TMEM halves
  if (warp == 2) {
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, 2 * GP_N);
  }
}

// ---------------------------------------------------------------------------
// CRT reconstruction: residues -> exact integer -> f128, scaled back.
// Each thread reconstructs 4 consecutive entries of a row (one 4-byte load
// per modulus). With NC chunks of 39 bits, every accumulator stays an exact
// integer below 2^53: 255 * (2^39 - 1) * L < 2^53 for L <= 64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double byte_to_double(uint32_t b) {
  // exact: 2^52 + b has b in its low mantissa bits
  return __dsub_rn(__hiloint2double(0x43300000, (int)b), 4503599627370496.0);
}
template <int NC>
__device__ __forceinline__ void carry_normalise(double* acc) {
#pragma unroll
  for (int c = 0; c < NC; c++) {
    double carry = floor(__dmul_rn(acc[c], 0x1p-39));
    acc[c] = __fma_rn(-carry, 0x1p39, acc[c]);
    acc[c + 1] = __dadd_rn(acc[c + 1], carry);
  }
}
// acc[0..NC) hold the weighted residue sums, each an exact integer in
// [0, 2^52) (L * 255 * 2^39 with L <= 32), acc[NC] = 0. The quotient
// estimate needs only the top two chunks (the lower ones move X / M by less
// than 2^-26); q < 2^13, so acc[c] - q mch[c] stays exact and every carry
// below fits as well.
template <int NC>
__device__ __forceinline__ dd crt_finish(double* acc, const double* mch, double inv_m, bool* neg_out) {
  // q = round(X / M): the true value is X - qM with |X - qM| <= M/4
  double xa = __fma_rn(acc[NC], 0x1p39, acc[NC - 1]);
  xa = __fma_rn(xa, 0x1p39, acc[NC - 2]);
  const double q = rint(__dmul_rn(__dmul_rn(xa, scale_pow2(1.0, CRT_BITS * (NC - 2))), inv_m));
#pragma unroll
  for (int c = 0; c < NC; c++) acc[c] = __fma_rn(-q, mch[c], acc[c]);
  carry_normalise<NC>(acc);
  bool neg = acc[NC] < 0.0;
  if (neg) {
#pragma unroll
    for (int c = 0; c <= NC; c++) acc[c] = -acc[c];
    carry_normalise<NC>(acc);
  }
  // sum the non-negative, non-overlapping chunks from the top into f128:
  // s.hi is 0 or above every chunk still to come, so quick_two_sum gives
  // two_sum's exact pair with half the operations
  dd s = dd{0.0, 0.0};
#pragma unroll
  for (int c = NC - 1; c >= 0; c--) {
    double v = scale_pow2(acc[c], CRT_BITS * c);
    double hs, he;
    quick_two_sum(s.hi, v, hs, he);
    s = dd_renorm(hs, __dadd_rn(he, s.lo));
  }
  *neg_out = neg;
  return s;
}
// EPT consecutive entries of a row per thread (one 2- or 4-byte load per
// modulus); fewer entries per thread hold fewer accumulators, so more warps
// fit on an SM. The per-entry arithmetic does not depend on EPT.
// LC > 0: L == LC at compile time, the tables come from c_crt (weights as
// immediate operands) and the moduli loop is unrolled.
template <int NC, int EPT, int LC = 0>
__global__ void __launch_bounds__(256) crt_dd_kernel(const uint8_t* __restrict__ cres, int64_t plane, int64_t Np,
                                                     int64_t m, int64_t n, const int* __restrict__ expA,
                                                     const int* __restrict__ expB, int beta,
                                                     const CrtTable* __restrict__ tab, double2* __restrict__ C) {
  __shared__ double w_sm[LC > 0 ? 1 : MAXL][NC];
  __shared__ double mch_sm[NC];
  const int L = LC > 0 ? LC : tab->L;
  if constexpr (LC == 0) {
    for (int i = threadIdx.x; i < L * NC; i += blockDim.x) w_sm[i / NC][i % NC] = tab->w[i / NC][i % NC];
    if (threadIdx.x < NC) mch_sm[threadIdx.x] = tab->mchunk[threadIdx.x];
  }
  const double(*w_s)[NCMAX] = LC > 0 ? c_crt[LC > 0 ? LC - CRT_CONST_L0 : 0].w : nullptr;
  const double(*w_d)[NC] = w_sm;
  const double* mch_s = LC > 0 ? c_crt[LC > 0 ? LC - CRT_CONST_L0 : 0].mchunk : mch_sm;
  sm100::griddep_launch_dependents();
  sm100::griddep_wait();  // the product residues come from the preceding GEMM
  if constexpr (LC == 0) __syncthreads();
  const double inv_m = LC > 0 ? c_crt[LC > 0 ? LC - CRT_CONST_L0 : 0].inv_m : tab->inv_m;
  const int64_t qpr = (n + EPT - 1) / EPT;  // EPT-entry groups per row
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= m * qpr) return;
  const int64_t i = g / qpr, j0 = EPT * (g % qpr);
  const int ea = expA[i];
  double acc[EPT][NC + 1];
#pragma unroll
  for (int e = 0; e < EPT; e++)
#pragma unroll
    for (int c = 0; c <= NC; c++) acc[e][c] = 0.0;
  const uint8_t* rp = cres + (size_t)i * Np + j0;
  // Issue the residue loads of 8 moduli back to back, then consume them, so
  // each thread waits for memory once per 8 moduli rather than once each.
#pragma unroll(LC > 0 ? 8 : 1)
  for (int l0 = 0; l0 < L; l0 += 8) {
    uint32_t v[8];
#pragma unroll
    for (int u = 0; u < 8; u++)
      v[u] = l0 + u >= L    ? 0u
             : EPT == 4 ? __ldg(reinterpret_cast<const uint32_t*>(rp + (size_t)(l0 + u) * plane))
             : EPT == 2 ? (uint32_t)__ldg(reinterpret_cast<const unsigned short*>(rp + (size_t)(l0 + u) * plane))
                        : (uint32_t)__ldg(rp + (size_t)(l0 + u) * plane);
#pragma unroll
    for (int u = 0; u < 8; u++) {
      if (l0 + u >= L) break;
#pragma unroll
      for (int e = 0; e < EPT; e++) {
        const double r = byte_to_double((v[u] >> (8 * e)) & 0xFFu);
#pragma unroll
        for (int c = 0; c < NC; c++)
          acc[e][c] = __fma_rn(r, LC > 0 ? w_s[l0 + u][c] : w_d[l0 + u][c], acc[e][c]);
      }
    }
  }
#pragma unroll
  for (int e = 0; e < EPT; e++) {
    const int64_t j = j0 + e;
    if (j >= n) break;
    const int eb = expB[j];
    if (ea == EXP_NONFINITE || eb == EXP_NONFINITE) {
      C[i * n + j] = make_double2(__longlong_as_double(0x7ff8000000000000ll), 0.0);
      continue;
    }
    bool neg;
    dd s = crt_finish<NC>(acc[e], mch_s, inv_m, &neg);
    const int shift = -((beta + 1022 - ea) + (beta + 1022 - eb));
    dd o = dd_renorm(scale_pow2(s.hi, shift), scale_pow2(s.lo, shift));
    if (neg) o = dd_neg(o);
    C[i * n + j] = make_double2(o.hi, o.lo);
  }
}

// ---------------------------------------------------------------------------
// CRT on the tensor core (the f128 GEMM, L = 28..32 moduli). For an entry
// with product residues r_l, the CRT value V = sum_l r_l W_l is split by the
// bytes of the weights: V = sum_q 2^(8q) S_q with S_q = sum_l r_l w_lq, an
// exact u8 x u8 dot product (< 30 * 255^2 < 2^21). A persistent CTA walks
// tiles of 256 consecutive entries of a row: TMA brings each tile's residue
// rows (one 256-byte row per modulus) into a 4-stage ring, the CTA
// transposes them into two 128 x 32 byte K-major tiles (32-byte swizzle) and
// multiplies each by the 32 x 32 byte matrix of the weights with one M = 128,
// N = 32, K = 32 tcgen05 MMA. Each thread then finishes two entries (ILP
// for the serial parts) from the 32 sums it reads from TMEM, in integer
// arithmetic: 16-bit limbs U_h = S_2h + 2^8 S_2h+1, the quotient q =
// round(V / M) from the top limbs (|V - q M| <= M/4 leaves a wide margin for
// the estimate), the digits d_h = U_h - q M_h, their exact 48-bit chunks
// with balanced carries, and the chunks summed from the top into a
// double-double. The MMA of a tile runs while the previous tile is finished.
// ---------------------------------------------------------------------------
constexpr int CT_THREADS = 128, CT_STAGES = 4, CT_TILE = 256;
constexpr int CT_SMEM = 1024 + 2 * 128 * 32 + 32 * 32 + CT_STAGES * 32 * CT_TILE;

// byte offset of (row, logical byte k < 32) in a K-major tile of 32-byte rows, 32-byte swizzle
__device__ __forceinline__ int swz32(int row, int k) {
  return (row >> 3) * 256 + (row & 7) * 32 + ((((k >> 4) ^ (row >> 2)) & 1) << 4) + (k & 15);
}

// the balanced 48-bit chunks b_k (|b_k| <= 2^47) of one entry's C = sum_k b_k 2^(48 k), from its 32 weight-byte sums
__device__ __forceinline__ void crt_tc_chunks(const uint32_t (&acc)[32], const CrtTcTable& T, int64_t (&b)[6]) {
  int32_t U[16];
#pragma unroll
  for (int h = 0; h < 16; h++) U[h] = (int32_t)(acc[2 * h] + (acc[2 * h + 1] << 8));
  // q = round(V / M) from the top limbs (the rest moves V / M by < 2^-29)
  const double vt = __dadd_rn(__dadd_rn(__dmul_rn((double)U[15], 0x1p48), __dmul_rn((double)U[14], 0x1p32)),
                              __dadd_rn(__dmul_rn((double)U[13], 0x1p16), (double)U[12]));
  const int32_t q = (int32_t)rint(__dmul_rn(vt, T.k192));
  // C = V - q M = sum_h d_h 2^(16 h), |d_h| < 2^31
  int32_t d[18];
#pragma unroll
  for (int h = 0; h < 16; h++) d[h] = U[h] - q * T.mlimb[h];
  d[16] = d[17] = 0;
  int64_t carry = 0;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const int64_t c = (int64_t)d[3 * k] + (int64_t)d[3 * k + 1] * 65536 + (int64_t)d[3 * k + 2] * 4294967296ll + carry;
    carry = k < 5 ? (c + (1ll << 47)) >> 48 : 0;
    b[k] = c - carry * 281474976710656ll;
  }
}

// the f128 value of one entry from its 32 weight-byte sums
__device__ __forceinline__ double2 crt_tc_entry(const uint32_t (&acc)[32], const CrtTcTable& T, int shift) {
  int64_t b[6];
  crt_tc_chunks(acc, T, b);
  double v[6];
#pragma unroll
  for (int k = 0; k < 6; k++) v[k] = scale_pow2((double)b[k], 48 * k);  // exact
  // from the top: a nonzero partial sum is a multiple of 2^(48 (k+1)) and
  // |b_k 2^(48 k)| < 2^(48 k + 48), so the quick two-sums are exact
  dd s = dd{v[5], 0.0};
#pragma unroll
  for (int k = 4; k >= 0; k--) {
    double hs, he;
    quick_two_sum(s.hi, v[k], hs, he);
    s = dd_renorm(hs, __dadd_rn(he, s.lo));
  }
  const dd o = dd_renorm(scale_pow2(s.hi, shift), scale_pow2(s.lo, shift));
  return make_double2(o.hi, o.lo);
}

// the f256 value of G1 2^105 + G2 from the two groups' weight-byte sums.
// 105 = 2 x 48 + 9: G1's chunk k times 2^9 (|512 b| <= 2^56) joins G2's
// chunk k + 2, and one balanced carry pass leaves nine chunks |c_k| <= 2^47
// (the top one small) with C = sum_k c_k 2^(48 k) exactly. They are added
// from the top into four limbs by a two-sum cascade (every step exact but
// the last limb's additions, ~2^-212 of |C| each) and renormalised by
// two-sum passes; the top nonzero chunk bounds |C| from below by half its
// weight, so the error is relative to |C|.
__device__ __forceinline__ double4 crt_tc_entry_qd(const uint32_t (&acc1)[32], const uint32_t (&acc2)[32],
                                                   const CrtTcTable& T, int shift) {
  int64_t b1[6], b2[6], c[9];
  crt_tc_chunks(acc1, T, b1);
  crt_tc_chunks(acc2, T, b2);
#pragma unroll
  for (int k = 0; k < 9; k++) c[k] = (k < 6 ? b2[k] : 0) + (k >= 2 && k < 8 ? b1[k - 2] * 512 : 0);
  int64_t carry = 0;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const int64_t x = c[k] + carry;
    carry = k < 8 ? (x + (1ll << 47)) >> 48 : 0;
    c[k] = x - carry * 281474976710656ll;
  }
  double x0 = 0.0, x1 = 0.0, x2 = 0.0, x3 = 0.0;
#pragma unroll
  for (int k = 8; k >= 0; k--) {
    const double v = scale_pow2((double)c[k], 48 * k);  // exact
    double e;
    two_sum(x0, v, x0, e);
    two_sum(x1, e, x1, e);
    two_sum(x2, e, x2, e);
    x3 = __dadd_rn(x3, e);
  }
  two_sum(x2, x3, x2, x3);
  two_sum(x1, x2, x1, x2);
  two_sum(x0, x1, x0, x1);
  two_sum(x1, x2, x1, x2);
  two_sum(x2, x3, x2, x3);
  return make_double4(scale_pow2(x0, shift), scale_pow2(x1, shift), scale_pow2(x2, shift), scale_pow2(x3, shift));
}

// QD: the f256 GEMM's CRT. A tile is 128 entries of a row and the map spans
// both groups' planes (G1's L planes, then G2's): the stage holds G1's box
// and then G2's, each group is transposed into its own 128 x 32 tile and
// multiplied by the weights, and each thread finishes one entry from both
// groups' sums (crt_tc_entry_qd), writing four limbs.
template <int LC, bool QD = false>
__global__ void __launch_bounds__(CT_THREADS, 4)
    crt_tc_kernel(const __grid_constant__ CUtensorMap map, int64_t m, int64_t n, const int* __restrict__ expA,
                  const int* __restrict__ expB, int beta, std::conditional_t<QD, double4, double2>* __restrict__ C,
                  int64_t ldc, uint32_t* status) {
  using namespace sm100;
  constexpr int TW = QD ? 128 : CT_TILE;        // entries of a row per tile
  constexpr int PS = QD ? 128 : CT_TILE;        // bytes between two moduli's residues in a stage
  constexpr int HALF = QD ? 32 * 128 : 128;     // stage offset of the second MMA tile's residues
  extern __shared__ uint8_t smem_raw[];
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t* sA = smem_raw + pad;  // 2 x (128 rows (entries) x 32 bytes (moduli)), swizzled
  uint8_t* sB = sA + 2 * 128 * 32;   // 32 rows (weight bytes q) x 32 bytes (moduli), swizzled
  uint8_t* sR = sB + 32 * 32;        // CT_STAGES x (LC planes x 256 residues, or 2 x LC planes x 128), as loaded
  __shared__ uint64_t full[CT_STAGES], mdone[2];
  __shared__ uint32_t tmem_slot;
  const CrtTcTable& T = c_crt_tc[LC - CRT_CONST_L0];
  const int t = threadIdx.x, warp = t / 32, lane = t % 32;
  for (int e = t; e < 32 * 32; e += CT_THREADS) sB[swz32(e / 32, e % 32)] = T.wb[e / 32][e % 32];
  if (t == 0) {
    prefetch_tmap(&map);
    for (int s = 0; s < CT_STAGES; s++) mbar_init(&full[s], 1);
    mbar_init(&mdone[0], 1);
    mbar_init(&mdone[1], 1);
    fence_mbarrier_init();
  }
  if (warp == 0) {
    tmem_alloc(&tmem_slot, 128);
    tmem_relinquish();
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  griddep_launch_dependents();
  griddep_wait();  // the product residues come from the preceding GEMM
  const int64_t tpr = (n + TW - 1) / TW, ntiles = m * tpr;
  const int64_t cnt = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;  // this CTA's tiles
  constexpr uint32_t TILE_BYTES = (uint32_t)CT_TILE * LC;  // QD: 2 x 128 x LC
  TileWalk prod(blockIdx.x, gridDim.x, tpr), cons(blockIdx.x, gridDim.x, tpr);
  RingPos pring, cring;
  auto issue = [&]() {  // thread 0: residues of the next tile into the next stage
    uint8_t* dst = sR + pring.st * 32 * CT_TILE;
    mbar_arrive_expect_tx(&full[pring.st], TILE_BYTES);
    tma_load_3d(dst, &map, &full[pring.st], (int)(prod.c * TW), (int)prod.r, 0);
    if constexpr (QD) tma_load_3d(dst + HALF, &map, &full[pring.st], (int)(prod.c * TW), (int)prod.r, LC);
    prod.next();
    pring.next<CT_STAGES>();
  };
  int64_t issued = 0;
  if (t == 0)
    for (; issued < cnt && issued < CT_STAGES; issued++) issue();
  const uint32_t idesc = idesc_i8(128, 32, true);
  bool ok = true;
  int64_t mma_issued = 0, mma_seen = 0;  // thread 0's count of MMAs issued; every thread's count of MMAs awaited
  int shift_prev[2] = {0, 0};            // the previous tile's scale shifts (or the non-finite marker)
  int64_t i_prev = 0, j0_prev = 0;       // the previous tile's row and first column
  // Iteration u waits for tile u - 1's MMAs, stages tile u, issues its MMAs
  // and finishes tile u - 1 while they run.
  for (int64_t u = 0; u <= cnt; u++) {
    if (u >= 1) {
      const int64_t v1 = u - 1;
      if (!mbar_wait(&mdone[v1 & 1], (uint32_t)((v1 >> 1) & 1), status, DEV_STATUS_TIMEOUT)) ok = false;
      else mma_seen = u;
    }
    int shift_cur[2] = {0, 0};
    const int64_t i_cur = cons.r, j0_cur = cons.c * TW;
    if (u < cnt) {
      const int ea = expA[i_cur];
#pragma unroll
      for (int h = 0; h < (QD ? 1 : 2); h++) {
        const int64_t j = j0_cur + 128 * h + t;
        const int eb = j < n ? expB[j] : 0;
        // QD: the groups hold X Y / 2^105
        shift_cur[h] = (ea == EXP_NONFINITE || eb == EXP_NONFINITE)
                           ? INT32_MIN
                           : (QD ? 105 : 0) - ((beta + 1022 - ea) + (beta + 1022 - eb));
      }
      const int st = cring.st;
      if (ok && !mbar_wait(&full[st], cring.ph, status, DEV_STATUS_TIMEOUT)) ok = false;
      cring.next<CT_STAGES>();
      cons.next();
      if (ok) {
        // warp w takes moduli 8w .. 8w+7, lane the entries 4 lane .. 4 lane + 3 of each half (QD: each group)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const uint8_t* r = sR + st * 32 * CT_TILE + HALF * h + 4 * lane;
          uint32_t wv[8];
#pragma unroll
          for (int v = 0; v < 8; v++) {
            const int l = 8 * warp + v;
            wv[v] = l < LC ? *reinterpret_cast<const uint32_t*>(r + l * PS) : 0u;
          }
          // entry e's bytes of moduli 8w .. 8w+7 -> row 4 lane + e, bytes 8w .. 8w+7
          uint8_t* a = sA + h * 128 * 32;
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const uint32_t sel = (uint32_t)e | ((uint32_t)(e + 4) << 4);
            const uint32_t lo = __byte_perm(__byte_perm(wv[0], wv[1], sel), __byte_perm(wv[2], wv[3], sel), 0x5410);
            const uint32_t hi = __byte_perm(__byte_perm(wv[4], wv[5], sel), __byte_perm(wv[6], wv[7], sel), 0x5410);
            *reinterpret_cast<uint2*>(a + swz32(4 * lane + e, 8 * warp)) = make_uint2(lo, hi);
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    tc_fence_before();
    // tile u staged and its residues read; tile u - 2's TMEM columns read out
    ok = __syncthreads_and(ok) != 0;
    tc_fence_after();
    if (!ok) break;
    if (u < cnt && t == 0) {
      const uint32_t d = tmem + (uint32_t)(u & 1) * 64u;
      mma_i8(d, desc_k_sw32(smem_u32(sA)), desc_k_sw32(smem_u32(sB)), idesc, 0u);
      mma_i8(d + 32u, desc_k_sw32(smem_u32(sA + 128 * 32)), desc_k_sw32(smem_u32(sB)), idesc, 0u);
      mma_commit(&mdone[u & 1]);
      mma_issued++;
      if (issued < cnt) {  // refill the stage just read
        issue();
        issued++;
      }
    }
    if (u >= 1) {
      // finish tile u - 1 (its MMAs were awaited above)
      const int64_t v1 = u - 1;
      const int64_t i = i_prev, j0 = j0_prev;
      uint32_t acc0[32], acc1[32];
      const uint32_t col = tmem + (uint32_t)(v1 & 1) * 64u + ((uint32_t)(warp * 32) << 16);
      tmem_ld_32x32b_x32(col, acc0);
      tmem_ld_32x32b_x32(col + 32u, acc1);
      tmem_wait_ld();
      const double nan = __longlong_as_double(0x7ff8000000000000ll);
      const int64_t ja = j0 + t, jb = j0 + 128 + t;
      if constexpr (QD) {
        const double4 r = shift_prev[0] == INT32_MIN ? make_double4(nan, 0.0, 0.0, 0.0)
                                                     : crt_tc_entry_qd(acc0, acc1, T, shift_prev[0]);
        if (ja < n) C[i * ldc + ja] = r;
      } else {
        const double2 nan2 = make_double2(nan, 0.0);
        const double2 ra = shift_prev[0] == INT32_MIN ? nan2 : crt_tc_entry(acc0, T, shift_prev[0]);
        const double2 rb = shift_prev[1] == INT32_MIN ? nan2 : crt_tc_entry(acc1, T, shift_prev[1]);
        if (ja < n) C[i * ldc + ja] = ra;
        if (jb < n) C[i * ldc + jb] = rb;
      }
    }
    shift_prev[0] = shift_cur[0];
    shift_prev[1] = shift_cur[1];
    i_prev = i_cur;
    j0_prev = j0_cur;
  }
  if (!ok && t == 0) {
    // a wait gave up: let the copies and the MMAs still in flight land (bounded) before the buffers go
    for (int64_t u = mma_issued; u < issued; u++)
      mbar_wait(&full[(int)(u % CT_STAGES)], (uint32_t)((u / CT_STAGES) & 1), status, DEV_STATUS_TIMEOUT,
                100000000ull);
    if (mma_issued > mma_seen) {
      const int64_t v1 = mma_issued - 1;
      mbar_wait(&mdone[v1 & 1], (uint32_t)((v1 >> 1) & 1), status, DEV_STATUS_TIMEOUT, 100000000ull);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 128);
  }
}

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// Planes of R rows x K bytes; consecutive planes are plane_stride bytes apart
// (K * R when 0) and rows row_pitch bytes apart (K when 0). Boxes reaching
// past K bytes or R rows read zeros.
static int make_map(CUtensorMap* map, const void* base, uint64_t K, uint64_t R, uint64_t L, uint32_t box_r,
                    uint64_t plane_stride = 0, uint64_t row_pitch = 0) {
  auto fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return HP_ERR_CUDA;
  }
  const uint64_t pitch = row_pitch ? row_pitch : K;
  cuuint64_t dims[3] = {K, R, L};
  cuuint64_t strides[2] = {pitch, plane_stride ? plane_stride : pitch * R};
  cuuint32_t box[3] = {(cuuint32_t)GB_K, box_r, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult rc = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)rc);
    return HP_ERR_CUDA;
  }
  return HP_OK;
}

constexpr int RES_EPR = 4;  // entries per thread of the f128 GEMM's residue kernel
constexpr int CRT_EPT = 2;  // entries per thread of crt_dd_kernel (measured best of 1, 2, 4)
static int launch_crt_dd(const uint8_t* cres, size_t Mp, size_t Np, size_t m, size_t n, const int* expA,
                         const int* expB, int beta, const CrtTable* tab, int nc, double2* C, cudaStream_t s,
                         bool pdl = false, int L = 0) {
  const int64_t groups = (int64_t)m * (int64_t)((n + CRT_EPT - 1) / CRT_EPT);
  const unsigned grid = (unsigned)((groups + 255) / 256);
#define HP_CRT_LC(LCV, NCV)                                                                                   \
  if (L == LCV && nc == NCV) {                                                                                \
    HP_CUDA_TRY(launch_k(pdl, crt_dd_kernel<NCV, CRT_EPT, LCV>, dim3(grid), dim3(256), 0, s, cres,            \
                         (int64_t)(Mp * Np), (int64_t)Np, (int64_t)m, (int64_t)n, expA, expB, beta, tab, C)); \
    return HP_OK;                                                                                             \
  }
  HP_CRT_LC(28, 6) HP_CRT_LC(28, 7) HP_CRT_LC(29, 6) HP_CRT_LC(29, 7) HP_CRT_LC(30, 6) HP_CRT_LC(30, 7)
  HP_CRT_LC(31, 6) HP_CRT_LC(31, 7) HP_CRT_LC(32, 6) HP_CRT_LC(32, 7)
#undef HP_CRT_LC
#define HP_CRT_CASE(NC)                                                                                       \
  case NC:                                                                                                    \
    HP_CUDA_TRY(launch_k(pdl, crt_dd_kernel<NC, CRT_EPT>, dim3(grid), dim3(256), 0, s, cres, (int64_t)(Mp * Np), \
                         (int64_t)Np, (int64_t)m, (int64_t)n, expA, expB, beta, tab, C));                      \
    break;
  switch (nc) {
    HP_CRT_CASE(3) HP_CRT_CASE(4) HP_CRT_CASE(5) HP_CRT_CASE(6) HP_CRT_CASE(7) HP_CRT_CASE(8) HP_CRT_CASE(9)
    default:
      set_error("ozaki: unsupported CRT chunk count %d", nc);
      return HP_ERR_UNSUPPORTED;
  }
#undef HP_CRT_CASE
  return HP_OK;
}

// The tensor-core CRT for L = 28..32 (the counts k <= 2^20 needs at beta =
// 106); HP_ERR_UNSUPPORTED for other L. Np must be a multiple of 256. Row i
// of the m x n result goes to C + i ldc (ldc = n when 0).
static int launch_crt_tc(const uint8_t* cres, size_t Mp, size_t Np, size_t m, size_t n, const int* expA,
                         const int* expB, int beta, int L, double2* C, int num_sms, uint32_t* status, cudaStream_t s,
                         bool pdl, size_t ldc = 0) {
  if (L < CRT_CONST_L0 || L >= CRT_CONST_L0 + CRT_CONST_N || Np % CT_TILE != 0) {
    set_error("ozaki: no tensor-core CRT for %d moduli", L);
    return HP_ERR_UNSUPPORTED;
  }
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<28>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<29>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<30>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<31>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    attr_set[dev & 63] = true;
  }
  // product residue planes L x Mp x Np bytes; one box is 256 residues of one row in every plane
  auto fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return HP_ERR_CUDA;
  }
  CUtensorMap map;
  cuuint64_t dims[3] = {Np, Mp, (cuuint64_t)L};
  cuuint64_t strides[2] = {Np, Np * Mp};
  cuuint32_t box[3] = {(cuuint32_t)CT_TILE, 1, (cuuint32_t)L};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult rc = fn(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t*>(cres), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)rc);
    return HP_ERR_CUDA;
  }
  const int grid = num_sms * 4;
#define HP_CRT_TC(LCV)                                                                                        \
  if (L == LCV) {                                                                                             \
    HP_CUDA_TRY(launch_k(pdl, crt_tc_kernel<LCV>, dim3(grid), dim3(CT_THREADS), CT_SMEM, s, map, (int64_t)m,  \
                         (int64_t)n, expA, expB, beta, C, (int64_t)(ldc ? ldc : n), status));                 \
    return HP_OK;                                                                                             \
  }
  HP_CRT_TC(28) HP_CRT_TC(29) HP_CRT_TC(30) HP_CRT_TC(31) HP_CRT_TC(32)
#undef HP_CRT_TC
  return HP_ERR_UNSUPPORTED;
}

// The f256 GEMM's CRT on the tensor core: g holds G1's L planes of Mp x Np
// bytes followed by G2's; row i of the m x n result goes to C + i ldc (ldc =
// n when 0). HP_ERR_UNSUPPORTED (nothing launched) for L outside 28..32 or
// Np not a multiple of 128.
static int launch_crt_tc_qd(const uint8_t* g, size_t Mp, size_t Np, size_t m, size_t n, const int* expA,
                            const int* expB, int beta, int L, double4* C, int num_sms, uint32_t* status,
                            cudaStream_t s, size_t ldc = 0) {
  if (L < CRT_CONST_L0 || L >= CRT_CONST_L0 + CRT_CONST_N || Np % 128 != 0) {
    set_error("ozaki f256: no tensor-core CRT for %d moduli", L);
    return HP_ERR_UNSUPPORTED;
  }
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<28, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<29, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<30, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<31, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(crt_tc_kernel<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM));
    attr_set[dev & 63] = true;
  }
  // 2L planes of Mp x Np bytes; one box is 128 residues of one row in L consecutive planes
  auto fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return HP_ERR_CUDA;
  }
  CUtensorMap map;
  cuuint64_t dims[3] = {Np, Mp, (cuuint64_t)(2 * L)};
  cuuint64_t strides[2] = {Np, Np * Mp};
  cuuint32_t box[3] = {128, 1, (cuuint32_t)L};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult rc = fn(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t*>(g), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)rc);
    return HP_ERR_CUDA;
  }
  const int grid = num_sms * 4;
#define HP_CRT_TCQ(LCV)                                                                                       \
  if (L == LCV) {                                                                                             \
    HP_CUDA_TRY(launch_k(true, crt_tc_kernel<LCV, true>, dim3(grid), dim3(CT_THREADS), CT_SMEM, s, map,        \
                         (int64_t)m, (int64_t)n, expA, expB, beta, C, (int64_t)(ldc ? ldc : n), status));     \
    return HP_OK;                                                                                             \
  }
  HP_CRT_TCQ(28) HP_CRT_TCQ(29) HP_CRT_TCQ(30) HP_CRT_TCQ(31) HP_CRT_TCQ(32)
#undef HP_CRT_TCQ
  return HP_ERR_UNSUPPORTED;
}

// Residue planes of the f128 GEMM's operands on the tensor core (unsigned
// bytes, L = 28..32): A is m x k (k x m when atb), B is k x n, both f128
// row-major; either may be null (its planes are not written). Writes the
// same bytes as residue_tile<..., U8 = true> over Mp x Kp and Np x Kp.
// HP_ERR_UNSUPPORTED (nothing launched) for other L or an operand not
// 16-byte aligned.
static int launch_residues_tc(bool atb, int L, const double2* A, size_t m, const int* expA, int8_t* outA, size_t Mp,
                              const double2* B, size_t n, const int* expB, int8_t* outB, size_t Np, size_t k,
                              size_t Kp, int beta, int num_sms, uint32_t* status, cudaStream_t s, bool pdl) {
  if (L < CRT_CONST_L0 || L >= CRT_CONST_L0 + CRT_CONST_N || (!A && !B) ||
      ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15u) || Mp % RC_ROWS || Np % RC_ROWS ||
      Kp % RC_P)
    return HP_ERR_UNSUPPORTED;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
#define HP_RC_ATTR(LCV)                                                                                           \
  HP_CUDA_TRY(cudaFuncSetAttribute(residue_tc_kernel<LCV, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                   RC_SMEM));                                                                     \
  HP_CUDA_TRY(cudaFuncSetAttribute(residue_tc_kernel<LCV, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, RC_SMEM));
    HP_RC_ATTR(28) HP_RC_ATTR(29) HP_RC_ATTR(30) HP_RC_ATTR(31) HP_RC_ATTR(32)
#undef HP_RC_ATTR
    attr_set[dev & 63] = true;
  }
  auto fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return HP_ERR_CUDA;
  }
  // f64 view of a row-major f128 matrix of `rows` rows and `cols` entries; a box is
  // box_e entries x box_r rows (the entries of 8 operand rows, or 128 reduction indices)
  auto map2d = [&](CUtensorMap* map, const double2* base, size_t rows, size_t cols, uint32_t box_e,
                   uint32_t box_r) -> int {
    cuuint64_t dims[2] = {2 * cols, rows};
    cuuint64_t strides[1] = {2 * cols * sizeof(double)};
    cuuint32_t box[2] = {2 * box_e, box_r};
    cuuint32_t estr[2] = {1, 1};
    CUresult rc = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double2*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (rc != CUDA_SUCCESS) {
      set_error("cuTensorMapEncodeTiled failed (%d)", (int)rc);
      return HP_ERR_CUDA;
    }
    return HP_OK;
  };
  CUtensorMap mapA, mapB;
  ResidueOperand oa{outA, (int64_t)(Mp * Kp), (int64_t)Kp, expA, A ? (int64_t)(Mp / RC_ROWS) : 0,
                    (int64_t)(Kp / RC_P), 0};
  ResidueOperand ob{outB, (int64_t)(Np * Kp), (int64_t)Kp, expB, B ? (int64_t)(Np / RC_ROWS) : 0,
                    (int64_t)(Kp / RC_P), 0};
  if (B) HP_TRY(map2d(&mapB, B, k, n, RC_ROWS, RC_P));
  if (A) {
    if (atb)
      HP_TRY(map2d(&mapA, A, k, m, RC_ROWS, RC_P));  // A is k x m: 8 operand rows x 128 reduction indices
    else
      HP_TRY(map2d(&mapA, A, m, k, RC_P, RC_ROWS));  // A is m x k: 128 reduction indices x 8 rows
  }
  if (!A) mapA = mapB;  // not read (no A tiles)
  if (!B) mapB = mapA;
  const int grid = num_sms * 2;
#define HP_RC(LCV)                                                                                                \
  if (L == LCV) {                                                                                                 \
    if (atb)                                                                                                      \
      HP_CUDA_TRY(launch_k(pdl, residue_tc_kernel<LCV, false>, dim3(grid), dim3(RC_THREADS), RC_SMEM, s, mapA,     \
                           mapB, oa, ob, beta, status));                                                          \
    else                                                                                                          \
      HP_CUDA_TRY(launch_k(pdl, residue_tc_kernel<LCV, true>, dim3(grid), dim3(RC_THREADS), RC_SMEM, s, mapA, mapB, \
                           oa, ob, beta, status));                                                                \
    return HP_OK;                                                                                                 \
  }
  HP_RC(28) HP_RC(29) HP_RC(30) HP_RC(31) HP_RC(32)
#undef HP_RC
  return HP_ERR_UNSUPPORTED;
}

static inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
static inline int ceil_log2(size_t x) {
  int b = 0;
  while (((size_t)1 << b) < x) b++;
  return b;
}

}  // namespace ozaki

int ozaki_moduli_for(size_t k, int beta) {
  const ozaki::HostTables& T = ozaki::host_tables();
  double need = 2.0 * beta + ozaki::ceil_log2(k) + 2.0;
  for (int L = 1; L <= ozaki::MAXL; L++)
    if (T.cum_log2[L] >= need) return L;
  return -1;
}

// Residue GEMM core shared by the f128 and f256 drivers: given int8 residue
// planes of op(A) (L x Mp x Kp) and B (L x Np x Kp), writes cres (L x Mp x Np).
int ozaki_residue_gemm(const int8_t* ares, const int8_t* bres, uint8_t* cres, int L, size_t Mp, size_t Np,
                       size_t Kp, cudaStream_t s) {
  return ozaki_residue_gemm_ex(ares, bres, cres, L, Mp, Np, Kp, Np, Mp * Np, 0, 0, 0, s, Mp, Np);
}

int ozaki_residue_gemm_ex(const int8_t* ares, const int8_t* bres, uint8_t* cres, int L, size_t Mp, size_t Np,
                          size_t Kp, size_t ldc, size_t plane, size_t c_row0, size_t c_col0, int acc_mode,
                          cudaStream_t s, size_t ra_rows, size_t rb_rows) {
  return ozaki_residue_gemm_k(ares, bres, cres, L, Mp, Np, Kp, Kp, 0, Kp, 0, ldc, plane, c_row0, c_col0, acc_mode, s,
                              ra_rows, rb_rows);
}

// General form: the residue planes have row length ka (A) / kb (B) bytes;
// the product runs over k_len bytes starting at byte a_k0 of A's rows and
// b_k0 of B's rows (multiples of 128).
int ozaki_residue_gemm_k(const int8_t* ares, const int8_t* bres, uint8_t* cres, int L, size_t Mp, size_t Np,
                         size_t ka, size_t kb_len_b, size_t a_k0, size_t k_len, size_t b_k0, size_t ldc,
                         size_t plane, size_t c_row0, size_t c_col0, int acc_mode, cudaStream_t s, size_t ra_rows,
                         size_t rb_rows, bool pdl, bool u8) {
  using namespace ozaki;
  DevTables* D;
  HP_TRY(device_tables(&D));
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev]) {
    HP_CUDA_TRY(cudaFuncSetAttribute(i8_gemm_mod_kernel<GB_N>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(i8_gemm_mod_kernel<GB_N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     GEMM_SMEM));
    attr_set[dev] = true;
  }
  CUtensorMap mapA, mapB;
  HP_TRY(make_map(&mapA, ares, ka, ra_rows ? ra_rows : Mp, L, GB_M));
  HP_TRY(make_map(&mapB, bres, kb_len_b, rb_rows ? rb_rows : Np, L, GB_N));
  uint32_t* status = device_status(s);
  if (!status) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  const int tiles_m = (int)(Mp / GB_M), tiles_n = (int)(Np / GB_N);
  const int num_tiles = L * tiles_m * tiles_n;
  const int grid = std::min(num_tiles, D->num_sms);
  const int kb_first = (int)(a_k0 / GB_K), nkb_total = (int)(k_len / GB_K);
  const int boff = (int)(b_k0 / GB_K) - kb_first;
  const int kb_chunk = (u8 ? MAX_K_CHUNK_U8 : MAX_K_CHUNK) / GB_K;
  for (int c0 = 0; c0 < nkb_total; c0 += kb_chunk) {
    const int kb0 = kb_first + c0, kb1 = kb_first + std::min(nkb_total, c0 + kb_chunk);
    const int mode = c0 > 0 ? (acc_mode == 2 ? 2 : 1) : acc_mode;
    if (u8)
      HP_CUDA_TRY(launch_k(pdl && c0 == 0, i8_gemm_mod_kernel<GB_N, true>, dim3(grid), dim3(256), GEMM_SMEM, s, mapA,
                           mapB, L, tiles_m, tiles_n, kb0, kb1, boff, mode, cres, (int64_t)ldc, (int64_t)plane,
                           (int64_t)c_row0, (int64_t)c_col0, status));
    else
      HP_CUDA_TRY(launch_k(pdl && c0 == 0, i8_gemm_mod_kernel<GB_N>, dim3(grid), dim3(256), GEMM_SMEM, s, mapA, mapB,
                           L, tiles_m, tiles_n, kb0, kb1, boff, mode, cres, (int64_t)ldc, (int64_t)plane,
                           (int64_t)c_row0, (int64_t)c_col0, status));
  }
  return HP_OK;
}

// Residue GEMM on CTA pairs: cres[l] = (A_l B_l^T) mod m_l for Mp x Np (Mp a
// multiple of 256, Np of 256) over ka bytes of K. Rows are pitch bytes long
// (ka when 0); the product takes A's bytes [a_k0, a_k0 + ka) and B's
// [b_k0, b_k0 + ka) of each row (offsets multiples of 128).
int ozaki_residue_gemm_pair(const int8_t* ares, const int8_t* bres, uint8_t* cres, int L, size_t Mp, size_t Np,
                            size_t ka, cudaStream_t s, bool pdl, bool u8, size_t pitch = 0, size_t a_k0 = 0,
                            size_t b_k0 = 0) {
  using namespace ozaki;
  DevTables* D;
  HP_TRY(device_tables(&D));
  static bool attr_set[64] = {};
  int dev = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 64 && !attr_set[dev]) {
    HP_CUDA_TRY(cudaFuncSetAttribute(i8_gemm_pair_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, GP_SMEM));
    HP_CUDA_TRY(cudaFuncSetAttribute(i8_gemm_pair_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, GP_SMEM));
    attr_set[dev] = true;
  }
  CUtensorMap mapA, mapB;
  HP_TRY(make_map(&mapA, ares + a_k0, ka, Mp, L, GP_HALF, pitch * Mp, pitch));
  HP_TRY(make_map(&mapB, bres + b_k0, ka, Np, L, GP_HALF, pitch * Np, pitch));
  uint32_t* status = device_status(s);
  if (!status) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  const int tiles_m = (int)(Mp / GP_M), tiles_n = (int)(Np / GP_N);
  const int num_tiles = L * tiles_m * tiles_n;
  const int grid = 2 * std::min(num_tiles, D->num_sms / 2);
  const int nkb_total = (int)(ka / GB_K);
  const int kb_chunk = (u8 ? MAX_K_CHUNK_U8 : MAX_K_CHUNK) / GB_K;
  for (int c0 = 0; c0 < nkb_total; c0 += kb_chunk) {
    const int kb1 = std::min(nkb_total, c0 + kb_chunk);
    const int mode = c0 > 0 ? 1 : 0;
    if (u8)
      HP_CUDA_TRY(launch_k(pdl && c0 == 0, i8_gemm_pair_kernel<true>, dim3(grid), dim3(GP_THREADS), GP_SMEM, s, mapA, mapB, L,
                           tiles_m, tiles_n, c0, kb1, mode, cres, (int64_t)Np, (int64_t)(Mp * Np), status));
    else
      HP_CUDA_TRY(launch_k(pdl && c0 == 0, i8_gemm_pair_kernel<false>, dim3(grid), dim3(GP_THREADS), GP_SMEM, s, mapA, mapB,
                           L, tiles_m, tiles_n, c0, kb1, mode, cres, (int64_t)Np, (int64_t)(Mp * Np), status));
  }
  return HP_OK;
}

namespace {
// The f128 GEMM's residue launch, specialised on the moduli count for the
// counts k <= 2^20 needs (28-32 at beta = 106; others take the runtime loop).
template <bool A_CONTIG, int LC>
cudaError_t launch_residues_lc(bool pdl, dim3 g, cudaStream_t s, const double2* A, int64_t RA, const int* expA,
                               int8_t* outA, int64_t planeA, unsigned tay, const double2* B, int64_t RB,
                               const int* expB, int8_t* outB, int64_t planeB, int64_t K, int beta, int L,
                               int64_t ld) {
  return launch_k(pdl, ozaki::residue_ab_kernel<A_CONTIG, ozaki::RES_EPR, true, LC>, g, dim3(256), 0, s, A, RA, expA,
                  outA, planeA, tay, B, RB, expB, outB, planeB, K, beta, L, ld);
}
template <bool A_CONTIG>
cudaError_t launch_residues_l(int L, bool pdl, dim3 g, cudaStream_t s, const double2* A, int64_t RA,
                              const int* expA, int8_t* outA, int64_t planeA, unsigned tay, const double2* B,
                              int64_t RB, const int* expB, int8_t* outB, int64_t planeB, int64_t K, int beta,
                              int64_t ld) {
#define HP_RES_CASE(N)                                                                                           \
  case N:                                                                                                         \
    return launch_residues_lc<A_CONTIG, N>(pdl, g, s, A, RA, expA, outA, planeA, tay, B, RB, expB, outB, planeB, \
                                           K, beta, L, ld);
  switch (L) {
    HP_RES_CASE(28)
    HP_RES_CASE(29)
    HP_RES_CASE(30)
    HP_RES_CASE(31)
    HP_RES_CASE(32)
    default:
      return launch_residues_lc<A_CONTIG, 0>(pdl, g, s, A, RA, expA, outA, planeA, tay, B, RB, expB, outB, planeB,
                                             K, beta, L, ld);
  }
#undef HP_RES_CASE
}
cudaError_t launch_residues_ab(bool atb, int L, bool pdl, dim3 g, cudaStream_t s, const double2* A, int64_t RA,
                               const int* expA, int8_t* outA, int64_t planeA, unsigned tay, const double2* B,
                               int64_t RB, const int* expB, int8_t* outB, int64_t planeB, int64_t K, int beta,
                               int64_t ld) {
  return atb ? launch_residues_l<false>(L, pdl, g, s, A, RA, expA, outA, planeA, tay, B, RB, expB, outB, planeB, K,
                                        beta, ld)
             : launch_residues_l<true>(L, pdl, g, s, A, RA, expA, outA, planeA, tay, B, RB, expB, outB, planeB, K,
                                       beta, ld);
}
}  // namespace

int ozaki_dd_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, bool atb,
                  cudaStream_t s) {
  using namespace ozaki;
  if (m == 0 || n == 0) return HP_OK;
  if (k == 0) {
    HP_CUDA_TRY(cudaMemsetAsync(c, 0, m * n * 16, s));
    return HP_OK;
  }
  DevTables* D;
  HP_TRY(device_tables(&D));
  const int beta = BETA_DD;
  const int L = ozaki_moduli_for(k, beta);
  if (L < 0) {
    set_error("ozaki: k = %zu needs more moduli than the table holds", k);
    return HP_ERR_UNSUPPORTED;
  }
  // rows padded to the CTA pair's 256-row tile (the padding holds zero residues)
  const size_t Mp = round_up(m, GP_M), Np = round_up(n, GB_N), Kp = round_up(k, GB_K);
  if (Mp / GB_M * (Np / GB_N) * (size_t)L > (size_t)INT32_MAX || Kp > (size_t)INT32_MAX) {
    set_error("ozaki: problem too large");
    return HP_ERR_INVALID_ARG;
  }
  DevBuf exps((Mp + Np) * sizeof(int), s);
  DevBuf ares((size_t)L * Mp * Kp, s), bres((size_t)L * Np * Kp, s), cres((size_t)L * Mp * Np, s);
  if (!exps.p || !ares.p || !bres.p || !cres.p) {
    set_error("ozaki: workspace allocation failed");
    return HP_ERR_CUDA;
  }
  int* expA = exps.as<int>();
  int* expB = expA + Mp;
  HP_CUDA_TRY(cudaMemsetAsync(exps.p, 0, (Mp + Np) * sizeof(int), s));
  // With profiling marks (events between the phases) the launches are not
  // chained programmatically.
  const bool pdl = !profiling_on();
  profile_mark(s, "start");
  const double2* A2 = reinterpret_cast<const double2*>(a);
  const double2* B2 = reinterpret_cast<const double2*>(b);
  // 1. exponents
  HP_TRY(launch_maxexp(A2, B2, m, n, k, atb, expA, expB, s));
  profile_mark(s, "exponents");
  // 2. residues (on the tensor core for the usual moduli counts)
  uint32_t* status = device_status(s);
  if (!status) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  const int rc = launch_residues_tc(atb, L, A2, m, expA, ares.as<int8_t>(), Mp, B2, n, expB, bres.as<int8_t>(), Np,
                                    k, Kp, beta, D->num_sms, status, s, pdl);
  if (rc == HP_ERR_UNSUPPORTED) {
    const unsigned tay = (unsigned)(Mp / RT_R);
    dim3 g((unsigned)(Kp / (4 * RES_EPR)), tay + (unsigned)(Np / RT_R));
    HP_CUDA_TRY(launch_residues_ab(atb, L, pdl, g, s, A2, (int64_t)m, (const int*)expA, ares.as<int8_t>(),
                                   (int64_t)(Mp * Kp), tay, B2, (int64_t)n, (const int*)expB, bres.as<int8_t>(),
                                   (int64_t)(Np * Kp), (int64_t)k, beta, (int64_t)Kp));
  } else if (rc != HP_OK) {
    return rc;
  }
  profile_mark(s, "residues");
  // 3. one int8 GEMM per modulus, on CTA pairs
  HP_TRY(ozaki_residue_gemm_pair(ares.as<int8_t>(), bres.as<int8_t>(), cres.as<uint8_t>(), L, Mp, Np, Kp, s, pdl, true));
  profile_mark(s, "i8_gemm");
  // 4. CRT (on the tensor core for the usual moduli counts)
  if (L >= CRT_CONST_L0 && L < CRT_CONST_L0 + CRT_CONST_N) {
    HP_TRY(launch_crt_tc(cres.as<uint8_t>(), Mp, Np, m, n, expA, expB, beta, L, reinterpret_cast<double2*>(c),
                         D->num_sms, status, s, pdl));
  } else {
    HP_TRY(launch_crt_dd(cres.as<uint8_t>(), Mp, Np, m, n, expA, expB, beta, D->crt + L, host_tables().crt[L].nc,
                         reinterpret_cast<double2*>(c), s, pdl, L));
  }
  profile_mark(s, "crt");
  return HP_OK;
}

// Host-pointer f128 GEMM C = op(A) B (chosen mode) with the PCIe copies
// overlapped. op(A) streams in as row panels (with atb, A's column panels,
// each copied into a compact k x rows matrix) and B as column panels (two for
// n >= 1024, else one) on a copy stream, in the order the blocks use them:
// B's first panel, A's first panel, B's other panels, A's other panels.
// Each panel's exponents and residue planes are formed once, as soon as its
// entries have landed. Each block of C (row panel x column panel) then takes
// a residue GEMM and the CRT on the library stream and goes back on a second
// copy stream while the next blocks are computed. Splitting B lets results
// start to flow back after half of B instead of all of it. The host link
// carries both directions at once, but at ~79 GB/s together against ~55 one
// way, so the time spent copying in before the first result can go back
// sets most of the overhead (2048^3: 3.2 -> 2.98 ms per call; four column
// panels measured 3.1). The arithmetic of every entry is that of
// ozaki_dd_gemm (same exponents, residues and CRT), so the result is
// bit-identical to the one-shot path.
namespace {
struct StreamsDrain {  // every stream idle before the buffers above it are freed
  cudaStream_t a, b, c;
  ~StreamsDrain() {
    cudaStreamSynchronize(a);
    cudaStreamSynchronize(b);
    cudaStreamSynchronize(c);
  }
};
// The calling thread's events on the current device, created once and
// reused by every later call (event creation would otherwise sit in front
// of the first copy of each call).
struct EventSet {
  std::vector<cudaEvent_t> ev;
  explicit EventSet(size_t count) {
    static thread_local std::vector<cudaEvent_t> pool[64];
    int dev = 0;
    cudaGetDevice(&dev);
    std::vector<cudaEvent_t>& p = pool[dev & 63];
    while (p.size() < count) {
      cudaEvent_t e = nullptr;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) break;
      p.push_back(e);
    }
    if (p.size() >= count) ev.assign(p.begin(), p.begin() + count);
  }
  bool ok() const { return !ev.empty(); }
};
}  // namespace

int ozaki_dd_gemm_host(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, bool atb) {
  using namespace ozaki;
  DevTables* D;
  HP_TRY(device_tables(&D));
  const int beta = BETA_DD;
  const int L = ozaki_moduli_for(k, beta);
  if (L < 0) {
    set_error("ozaki: k = %zu needs more moduli than the table holds", k);
    return HP_ERR_UNSUPPORTED;
  }
  const bool tc_crt = L >= CRT_CONST_L0 && L < CRT_CONST_L0 + CRT_CONST_N;
  const size_t Kp = round_up(k, GB_K);
  const size_t panels_wanted = m >= 2048 ? 16 : m >= 1024 ? 8 : 4;
  const size_t pr = round_up((m + panels_wanted - 1) / panels_wanted, GP_M);  // rows per A panel (CTA-pair tiles)
  const size_t np = (m + pr - 1) / pr;
  // B and C in column panels when n is wide: the first C blocks then need only
  // B's first panel and A's first panel, so results start to flow back while
  // most of the operands are still on their way in (the host link carries
  // both directions at once, but not at twice one direction's rate). The
  // FP64 CRT writes whole rows, so without the tensor-core CRT: one panel.
  const size_t nq_wanted = (tc_crt && n >= 1024) ? 2 : 1;  // four measured slower (more, smaller blocks)
  const size_t pc = round_up((n + nq_wanted - 1) / nq_wanted, GP_N);  // columns per B panel
  const size_t nq = (n + pc - 1) / pc;
  const size_t Mpa = np * pr;  // rows of A's residue planes, every panel padded to pr
  if (pr / GB_M * (pc / GB_N) * (size_t)L > (size_t)INT32_MAX || Kp > (size_t)INT32_MAX) {
    set_error("ozaki: problem too large");
    return HP_ERR_INVALID_ARG;
  }
  cudaStream_t s = library_stream(), sin = library_copy_stream(0), sout = library_copy_stream(1);
  DevBuf dA(m * k * 16, s), dB(k * n * 16, s), dC(m * n * 16, s);
  DevBuf exps((Mpa + nq * pc) * sizeof(int), s);
  DevBuf bres((size_t)L * nq * pc * Kp, s), ares((size_t)L * Mpa * Kp, s), cres((size_t)L * pr * pc, s);
  if (!dA.p || !dB.p || !dC.p || !exps.p || !bres.p || !ares.p || !cres.p) {
    set_error("ozaki: workspace allocation failed");
    return HP_ERR_CUDA;
  }
  EventSet ev(1 + nq + np + np * nq);
  if (!ev.ok()) {
    set_error("ozaki: event creation failed");
    return HP_ERR_CUDA;
  }
  StreamsDrain drain{s, sin, sout};
  cudaEvent_t ready = ev.ev[0];
  cudaEvent_t* eB = ev.ev.data() + 1;  // B panel j copied
  cudaEvent_t* eA = eB + nq;           // A panel i copied
  cudaEvent_t* eC = eA + np;           // C block (i, j) written
  int* expA = exps.as<int>();          // every row's exponent (panel i at i pr)
  int* expB = expA + Mpa;              // every column's (panel j at j pc)
  const bool pdl = !profiling_on();
  // the buffers exist (stream-ordered) before the copy streams touch them
  HP_CUDA_TRY(cudaEventRecord(ready, s));
  profile_mark(s, "start");  // with profiling on: a timeline of the copies in, the blocks and the copies out
  HP_CUDA_TRY(cudaStreamWaitEvent(sin, ready, 0));
  HP_CUDA_TRY(cudaStreamWaitEvent(sout, ready, 0));
  // copies in, in the order the blocks use them: B panel 0, A panel 0, B's
  // other panels, A's other panels. B panel j (columns j pc ..) is stored as
  // a compact k x nj matrix.
  auto copy_b = [&](size_t j) -> int {
    const size_t j0 = j * pc, nj = std::min(pc, n - j0);
    HP_CUDA_TRY(cudaMemcpy2DAsync(dB.as<char>() + j0 * k * 16, nj * 16, reinterpret_cast<const char*>(b) + j0 * 16,
                                  n * 16, nj * 16, k, cudaMemcpyHostToDevice, sin));
    HP_CUDA_TRY(cudaEventRecord(eB[j], sin));
    return HP_OK;
  };
  auto copy_a = [&](size_t i) -> int {  // rows r0 .. of op(A); with atb, A's columns r0 .. as a compact k x mi panel
    const size_t r0 = i * pr, mi = std::min(pr, m - r0);
    if (atb)
      HP_CUDA_TRY(cudaMemcpy2DAsync(dA.as<char>() + r0 * k * 16, mi * 16, reinterpret_cast<const char*>(a) + r0 * 16,
                                    m * 16, mi * 16, k, cudaMemcpyHostToDevice, sin));
    else
      HP_CUDA_TRY(cudaMemcpyAsync(dA.as<char>() + r0 * k * 16, reinterpret_cast<const char*>(a) + r0 * k * 16,
                                  mi * k * 16, cudaMemcpyHostToDevice, sin));
    HP_CUDA_TRY(cudaEventRecord(eA[i], sin));
    return HP_OK;
  };
  HP_TRY(copy_b(0));
  profile_mark(sin, "b0_in");
  HP_TRY(copy_a(0));
  for (size_t j = 1; j < nq; j++) HP_TRY(copy_b(j));
  for (size_t i = 1; i < np; i++) HP_TRY(copy_a(i));
  profile_mark(sin, "all_in");
  uint32_t* status = device_status(s);
  if (!status) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  HP_CUDA_TRY(cudaMemsetAsync(exps.p, 0, (Mpa + nq * pc) * sizeof(int), s));  // maxima merge by atomicMax
  const int nc = host_tables().crt[L].nc;
  for (size_t i = 0; i < np; i++) {
    const size_t r0 = i * pr, mi = std::min(pr, m - r0), Mpi = round_up(mi, GP_M);
    const double2* A2 = dA.as<const double2>() + r0 * k;
    int8_t* aresi = ares.as<int8_t>() + (size_t)L * r0 * Kp;  // L planes of Mpi x Kp
    HP_CUDA_TRY(cudaStreamWaitEvent(s, eA[i], 0));
    HP_TRY(launch_maxexp(A2, (const double2*)nullptr, mi, 0, k, atb, expA + r0, nullptr, s));
    int rc = launch_residues_tc(atb, L, A2, mi, expA + r0, aresi, Mpi, nullptr, 0, nullptr, nullptr, 0, k, Kp, beta,
                                D->num_sms, status, s, pdl);
    if (rc == HP_ERR_UNSUPPORTED) {
      const unsigned tay = (unsigned)(Mpi / RT_R);
      HP_CUDA_TRY(launch_residues_ab(atb, L, pdl, dim3((unsigned)(Kp / (4 * RES_EPR)), tay), s, A2, (int64_t)mi,
                                     expA + r0, aresi, (int64_t)(Mpi * Kp), tay, nullptr, 0, nullptr, nullptr, 0,
                                     (int64_t)k, beta, (int64_t)Kp));
    } else if (rc != HP_OK) {
      return rc;
    }
    for (size_t j = 0; j < nq; j++) {
      const size_t j0 = j * pc, nj = std::min(pc, n - j0);
      int8_t* bresj = bres.as<int8_t>() + (size_t)L * j0 * Kp;  // L planes of pc x Kp
      if (i == 0) {  // B panel j's column exponents and residue planes, once
        const double2* Bj = dB.as<const double2>() + j0 * k;
        HP_CUDA_TRY(cudaStreamWaitEvent(s, eB[j], 0));
        HP_TRY(launch_maxexp((const double2*)nullptr, Bj, 0, nj, k, false, nullptr, expB + j0, s));
        rc = launch_residues_tc(false, L, nullptr, 0, nullptr, nullptr, 0, Bj, nj, expB + j0, bresj, pc, k, Kp, beta,
                                D->num_sms, status, s, pdl);
        if (rc == HP_ERR_UNSUPPORTED)
          HP_CUDA_TRY(launch_residues_ab(false, L, pdl, dim3((unsigned)(Kp / (4 * RES_EPR)), (unsigned)(pc / RT_R)), s,
                                         nullptr, 0, nullptr, nullptr, 0, 0, Bj, (int64_t)nj, expB + j0, bresj,
                                         (int64_t)(pc * Kp), (int64_t)k, beta, (int64_t)Kp));
        else if (rc != HP_OK)
          return rc;
      }
      HP_TRY(ozaki_residue_gemm_pair(aresi, bresj, cres.as<uint8_t>(), L, Mpi, pc, Kp, s, pdl, true));
      double* Cij = dC.as<double>() + (r0 * n + j0) * 2;
      if (tc_crt)
        HP_TRY(launch_crt_tc(cres.as<uint8_t>(), Mpi, pc, mi, nj, expA + r0, expB + j0, beta, L,
                             reinterpret_cast<double2*>(Cij), D->num_sms, status, s, pdl, n));
      else  // one column panel (nj = n)
        HP_TRY(launch_crt_dd(cres.as<uint8_t>(), Mpi, pc, mi, n, expA + r0, expB, beta, D->crt + L, nc,
                             reinterpret_cast<double2*>(Cij), s, pdl, L));
      cudaEvent_t e = eC[i * nq + j];
      HP_CUDA_TRY(cudaEventRecord(e, s));
      HP_CUDA_TRY(cudaStreamWaitEvent(sout, e, 0));
      HP_CUDA_TRY(cudaMemcpy2DAsync(reinterpret_cast<char*>(c) + (r0 * n + j0) * 16, n * 16, Cij, n * 16, nj * 16, mi,
                                    cudaMemcpyDeviceToHost, sout));
      if (i == 0 && j == 0) profile_mark(sout, "c00_out");
    }
  }
  profile_mark(s, "blocks_done");
  profile_mark(sout, "all_out");
  HP_CUDA_TRY(cudaStreamSynchronize(sout));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return consume_device_status(s);
}

// ===========================================================================
// f256 (MultiFloat<4>) Ozaki-II GEMM.
// Entries are scaled to integers X of <= 210 bits and split X = Xh 2^105 + Xl
// (balanced base-2^21 digits, |Xh|, |Xl| <= 2^105). Two exact residue GEMM
// groups are formed,
//     G1 = Xh Yh  (k terms),   G2 = [Xh | Xl] [Yl ; Yh] = Xh Yl + Xl Yh (2k),
// each rebuilt by the CRT and rounded to f256, and since
// X Y = G1 2^210 + G2 2^105 + Xl Yl, C = (G1 2^105 + G2) 2^(105 - sa - sb).
// The omitted Xl Yl term is below 2^-209 of |A||B| (the f256 tolerance is
// 4k 2^-208 normwise). Residue rows are 2 Kp bytes: A = [Xh | Xl], B = [Yl | Yh].
// ===========================================================================
namespace ozaki {
constexpr int BETA_QD = 210;

// The f256 GEMM's residue rows on the tensor core (residue_tc_kernel<., ., QD>):
// A (m x k, or k x m when atb) and B (k x n) of 4-limb entries, either may be
// null (its planes are not written); rows of 2 Kp bytes, [Xh | Xl] for A and
// [Yl | Yh] for B, unsigned bytes. HP_ERR_UNSUPPORTED (nothing launched) for
// moduli counts other than 28..32 or operands not 32-byte aligned.
static int launch_residues_tc_qd(bool atb, int L, const double4* A, size_t m, const int* expA, int8_t* outA,
                                 size_t Mp, const double4* B, size_t n, const int* expB, int8_t* outB, size_t Np,
                                 size_t k, size_t Kp, int num_sms, uint32_t* status, cudaStream_t s) {
  if (L < CRT_CONST_L0 || L >= CRT_CONST_L0 + CRT_CONST_N || (!A && !B) || Mp % 4 || Np % 4 || Kp % RC_P ||
      ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 31u))
    return HP_ERR_UNSUPPORTED;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
#define HP_RQ_ATTR(LCV)                                                                                          \
  HP_CUDA_TRY(cudaFuncSetAttribute(residue_tc_kernel<LCV, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                   RC_SMEM));                                                                    \
  HP_CUDA_TRY(cudaFuncSetAttribute(residue_tc_kernel<LCV, false, true>,                                          \
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, RC_SMEM));
    HP_RQ_ATTR(28) HP_RQ_ATTR(29) HP_RQ_ATTR(30) HP_RQ_ATTR(31) HP_RQ_ATTR(32)
#undef HP_RQ_ATTR
    attr_set[dev & 63] = true;
  }
  auto fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return HP_ERR_CUDA;
  }
  // f64 view (4 limbs x cols x rows) of a row-major f256 matrix; a box is
  // 4 limbs x box_c entries x box_r rows
  auto map3d = [&](CUtensorMap* map, const double4* base, size_t rows, size_t cols, uint32_t box_c,
                   uint32_t box_r) -> int {
    cuuint64_t dims[3] = {4, cols, rows};
    cuuint64_t strides[2] = {32, cols * 32};
    cuuint32_t box[3] = {4, box_c, box_r};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult rc = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double4*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (rc != CUDA_SUCCESS) {
      set_error("cuTensorMapEncodeTiled failed (%d)", (int)rc);
      return HP_ERR_CUDA;
    }
    return HP_OK;
  };
  CUtensorMap mapA, mapB;
  if (B) HP_TRY(map3d(&mapB, B, k, n, 4, RC_P));  // B is k x n: 4 operand rows (columns) x 128 reduction indices
  if (A) {
    if (atb)
      HP_TRY(map3d(&mapA, A, k, m, 4, RC_P));  // A is k x m
    else
      HP_TRY(map3d(&mapA, A, m, k, RC_P, 4));  // A is m x k: 128 reduction indices x 4 rows
  }
  if (!A) mapA = mapB;  // not read (no A tiles)
  if (!B) mapB = mapA;
  ResidueOperand oa{outA, (int64_t)(Mp * 2 * Kp), (int64_t)(2 * Kp), expA, A ? (int64_t)(Mp / 4) : 0,
                    (int64_t)(Kp / RC_P), (int64_t)Kp};
  ResidueOperand ob{outB, (int64_t)(Np * 2 * Kp), (int64_t)(2 * Kp), expB, B ? (int64_t)(Np / 4) : 0,
                    (int64_t)(Kp / RC_P), (int64_t)Kp};
  const int grid = num_sms * 2;
#define HP_RQ(LCV)                                                                                                \
  if (L == LCV) {                                                                                                 \
    if (atb)                                                                                                      \
      HP_CUDA_TRY(launch_k(true, residue_tc_kernel<LCV, false, true>, dim3(grid), dim3(RC_THREADS), RC_SMEM, s,    \
                           mapA, mapB, oa, ob, BETA_QD, status));                                                 \
    else                                                                                                          \
      HP_CUDA_TRY(launch_k(true, residue_tc_kernel<LCV, true, true>, dim3(grid), dim3(RC_THREADS), RC_SMEM, s,     \
                           mapA, mapB, oa, ob, BETA_QD, status));                                                 \
    return HP_OK;                                                                                                 \
  }
  HP_RQ(28) HP_RQ(29) HP_RQ(30) HP_RQ(31) HP_RQ(32)
#undef HP_RQ
  return HP_ERR_UNSUPPORTED;
}

// Balanced base-2^21 digits of rint(v) for |v| < 2^212 (exact).
__device__ __forceinline__ void int_digits21x10(double v, int32_t* d) {
  double a = fabs(rint(v));
  const int32_t sg = signbit(v) ? -1 : 1;
#pragma unroll
  for (int c = 9; c >= 1; c--) {
    const double sc = scale_pow2(1.0, -21 * c), up = scale_pow2(1.0, 21 * c);
    const double t = floor(__dmul_rn(a, sc));
    a = __dsub_rn(a, __dmul_rn(t, up));
    d[c] = sg * (int32_t)t;
  }
  d[0] = sg * (int32_t)a;
}

// residues of a 5-digit (base 2^21) number
__device__ __forceinline__ uint32_t balanced_byte21(const int32_t* D, const int* w, int l, int m) {
  int32_t x = 0;
#pragma unroll
  for (int c = 0; c < 5; c++) x += D[c] * w[c];
  int r = (int)mod_reduce(x, l);
  if (r > 127) r -= m;
  return (uint32_t)(r & 0xFF);
}

// Operand residues for the f256 GEMM. Element (r, p) is src[r*K + p]
// (P_CONTIG) or src[p*R + r], 4 limbs. Writes hi digits at byte offset
// hi_off and lo digits at lo_off of each 2*Kp-byte row, planes of Rp rows.
// residue of a 5-digit (base 2^21) number in [0, m) (w[0] = 2^0 mod m = 1)
__device__ __forceinline__ uint32_t unsigned_byte21(const int32_t* D, const int* w, int l) {
  int32_t x = D[0];
#pragma unroll
  for (int c = 1; c < 5; c++) x += D[c] * w[c];
  return mod_reduce(x, l);
}

// One RT_R x (4 EPR) tile (block coordinates bx, by) of the f256 residue
// rows [Xh | Xl]: EPR entries per thread (8 or 4), all L moduli, residues
// balanced (signed bytes) or, with U8, in [0, m).
// LC > 0: L == LC at compile time; the moduli loop is unrolled with each
// modulus' constants (c_tab.pw21) as immediate operands, and the
// transposed tile stores its planes in groups of QG behind one barrier.
template <bool P_CONTIG, int EPR, bool U8, int LC = 0>
__device__ __forceinline__ void residue_qd_tile(const double4* __restrict__ src, int64_t R, int64_t K,
                                                const int* __restrict__ expf, int L, int64_t Rp, int64_t Kp,
                                                int64_t hi_off, int64_t lo_off, int8_t* __restrict__ out,
                                                unsigned bx, unsigned by, const int (*w21)[5]) {
  constexpr int NW = EPR / 4;  // 32-bit words per half per thread
  __shared__ __align__(16) uint32_t T[2][2][RT_R][EPR + 1];
  const int t = threadIdx.x;
  const int rl = P_CONTIG ? t / 4 : t % 64;
  const int quad = P_CONTIG ? t % 4 : t / 64;
  const int64_t r = (int64_t)by * RT_R + rl;
  const int64_t p0 = (int64_t)bx * (4 * EPR) + EPR * quad;
  int32_t dig[EPR][10];
#pragma unroll
  for (int e = 0; e < EPR; e++)
#pragma unroll
    for (int c = 0; c < 10; c++) dig[e][c] = 0;
  if (r < R) {
    const int ex = expf[r];
    if (ex != EXP_NONFINITE) {
      const int sh = BETA_QD + 1022 - ex;
#pragma unroll
      for (int e = 0; e < EPR; e++) {
        const int64_t p = p0 + e;
        if (p < K) {
          const double4 v = P_CONTIG ? src[r * K + p] : src[p * R + r];
          const double lim[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int q = 0; q < 4; q++) {
            int32_t d[10];
            int_digits21x10(scale_pow2(lim[q], sh), d);
#pragma unroll
            for (int c = 0; c < 10; c++) dig[e][c] += d[c];
          }
#pragma unroll
          for (int c = 0; c < 9; c++) {
            const int32_t carry = (dig[e][c] + (1 << 20)) >> 21;
            dig[e][c] -= carry << 21;
            dig[e][c + 1] += carry;
          }
        }
      }
    }
  }
  int8_t* const base = out + (size_t)by * RT_R * (2 * Kp) + (size_t)bx * (4 * EPR);
  if constexpr (LC > 0) {
    constexpr int QG = 8;  // planes per barrier of the transposed store
    __shared__ uint32_t TG[P_CONTIG ? 1 : QG][2][P_CONTIG ? 1 : RT_R][EPR + 1];
#pragma unroll
    for (int l = 0; l < LC; l++) {
      uint32_t wh[NW], wl[NW];
#pragma unroll
      for (int q = 0; q < NW; q++) {
        wh[q] = wl[q] = 0;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int32_t* dl = dig[4 * q + e];
          const uint32_t bl = U8 ? unsigned_byte21(dl, c_tab.pw21[l], l)
                                 : balanced_byte21(dl, c_tab.pw21[l], l, c_tab.mod[l]);
          const uint32_t bh = U8 ? unsigned_byte21(dl + 5, c_tab.pw21[l], l)
                                 : balanced_byte21(dl + 5, c_tab.pw21[l], l, c_tab.mod[l]);
          wl[q] |= bl << (8 * e);
          wh[q] |= bh << (8 * e);
        }
      }
      int8_t* plane = base + (size_t)l * Rp * (2 * Kp);
      if constexpr (P_CONTIG) {
        int8_t* row = plane + (size_t)rl * (2 * Kp) + EPR * quad;
        if (NW == 2) {
          *reinterpret_cast<uint2*>(row + hi_off) = make_uint2(wh[0], wh[NW - 1]);
          *reinterpret_cast<uint2*>(row + lo_off) = make_uint2(wl[0], wl[NW - 1]);
        } else {
          *reinterpret_cast<uint32_t*>(row + hi_off) = wh[0];
          *reinterpret_cast<uint32_t*>(row + lo_off) = wl[0];
        }
      } else {
#pragma unroll
        for (int q = 0; q < NW; q++) {
          TG[l % QG][0][rl][NW * quad + q] = wh[q];
          TG[l % QG][1][rl][NW * quad + q] = wl[q];
        }
        if (l % QG == QG - 1 || l == LC - 1) {  // a group of planes is complete
          const int g0 = l - l % QG, gn = l % QG + 1;
          __syncthreads();
          for (int u = t; u < gn * RT_R * 2 * NW; u += blockDim.x) {
            const int gl = u / (RT_R * 2 * NW), rem = u % (RT_R * 2 * NW);
            const int row = rem / (2 * NW), r2 = rem % (2 * NW), part = r2 / NW, half = r2 % NW;
            const uint32_t* sw = &TG[gl][part][row][4 * half];
            *reinterpret_cast<uint4*>(base + (size_t)(g0 + gl) * Rp * (2 * Kp) + (size_t)row * (2 * Kp) +
                                      (part ? lo_off : hi_off) + 16 * half) = make_uint4(sw[0], sw[1], sw[2], sw[3]);
          }
          __syncthreads();  // the group's buffers are rewritten by the next group
        }
      }
    }
  } else {
    for (int l = 0; l < L; l++) {
      const int m = c_tab.mod[l];
      uint32_t wh[NW], wl[NW];
#pragma unroll
      for (int q = 0; q < NW; q++) {
        wh[q] = wl[q] = 0;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int32_t* dl = dig[4 * q + e];
          const uint32_t bl = U8 ? unsigned_byte21(dl, w21[l], l) : balanced_byte21(dl, w21[l], l, m);
          const uint32_t bh = U8 ? unsigned_byte21(dl + 5, w21[l], l) : balanced_byte21(dl + 5, w21[l], l, m);
          wl[q] |= bl << (8 * e);
          wh[q] |= bh << (8 * e);
        }
      }
      int8_t* plane = base + (size_t)l * Rp * (2 * Kp);
      if (P_CONTIG) {
        int8_t* row = plane + (size_t)rl * (2 * Kp) + EPR * quad;
        if (NW == 2) {
          *reinterpret_cast<uint2*>(row + hi_off) = make_uint2(wh[0], wh[NW - 1]);
          *reinterpret_cast<uint2*>(row + lo_off) = make_uint2(wl[0], wl[NW - 1]);
        } else {
          *reinterpret_cast<uint32_t*>(row + hi_off) = wh[0];
          *reinterpret_cast<uint32_t*>(row + lo_off) = wl[0];
        }
      } else {
#pragma unroll
        for (int q = 0; q < NW; q++) {
          T[l & 1][0][rl][NW * quad + q] = wh[q];
          T[l & 1][1][rl][NW * quad + q] = wl[q];
        }
        __syncthreads();
        if (t < RT_R * 2 * NW) {
          const int row = t / (2 * NW), rem = t % (2 * NW), part = rem / NW, half = rem % NW;
          const uint32_t* sw = &T[l & 1][part][row][4 * half];
          *reinterpret_cast<uint4*>(plane + (size_t)row * (2 * Kp) + (part ? lo_off : hi_off) + 16 * half) =
              make_uint4(sw[0], sw[1], sw[2], sw[3]);
        }
      }
    }
  }
}

// Both f256 operands' residues in one launch: block rows [0, tiles_ay) cover
// A (row-contiguous when A_CONTIG; halves at hi 0, lo Kp), the rest B
// (transposed; halves at hi Kp, lo 0).
template <bool A_CONTIG, int EPR, bool U8, int LC = 0>
__global__ void __launch_bounds__(256, 3) residue_qd_ab_kernel(const double4* __restrict__ A, int64_t RA, int64_t RpA,
                                                            const int* __restrict__ expA, int8_t* __restrict__ outA,
                                                            unsigned tiles_ay, const double4* __restrict__ B,
                                                            int64_t RB, int64_t RpB, const int* __restrict__ expB,
                                                            int8_t* __restrict__ outB, int64_t K, int64_t Kp, int L) {
  const int(*w21)[5] = c_tab.pw21;  // 2^(21 c) mod m, balanced
  sm100::griddep_launch_dependents();
  sm100::griddep_wait();  // the exponents come from the preceding pass
  if (blockIdx.y < tiles_ay)
    residue_qd_tile<A_CONTIG, EPR, U8, LC>(A, RA, K, expA, L, RpA, Kp, 0, Kp, outA, blockIdx.x, blockIdx.y, w21);
  else
    residue_qd_tile<false, EPR, U8, LC>(B, RB, K, expB, L, RpB, Kp, Kp, 0, outB, blockIdx.x, blockIdx.y - tiles_ay,
                                        w21);
}

// f256 CRT: rebuild G1 and G2, C = (G1 2^105 + G2) 2^(105 - sa - sb).
// One group's weighted residue sums -> |G| as normalised 39-bit chunks
// acc[0..NC] (acc[NC] = 0 when |G| < M/2); returns the sign.
template <int NC, int LC = 0, class W>
__device__ __forceinline__ bool crt_group_chunks(const uint8_t* rp, int64_t plane, int L, W w_s, const double* mch,
                                                 double inv_m, double* acc) {
#pragma unroll
  for (int q = 0; q <= NC; q++) acc[q] = 0.0;
#pragma unroll(LC > 0 ? 8 : 1)
  for (int l0 = 0; l0 < L; l0 += 8) {
    uint32_t v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) v[u] = (l0 + u < L) ? (uint32_t)__ldg(rp + (size_t)(l0 + u) * plane) : 0u;
#pragma unroll
    for (int u = 0; u < 8; u++) {
      if (l0 + u >= L) break;
      const double x = byte_to_double(v[u]);
#pragma unroll
      for (int q = 0; q < NC; q++) acc[q] = __fma_rn(x, w_s[l0 + u][q], acc[q]);
    }
  }
  bool neg;
  (void)crt_finish<NC>(acc, mch, inv_m, &neg);  // leaves |G| in normalised chunks
  return neg;
}
// V = G1 2^105 + G2 as a quad-double. Both groups' signed chunks go on one
// 39-bit grid (105 = 2 x 39 + 27: chunk c of G1 splits exactly at 12 bits
// into cells c + 2 and c + 3), where every cell stays an exact integer below
// 2^41; the cells are carry-normalised (the top one takes the sign; if it
// is negative all are negated and normalised again), then added from the
// top into four limbs by a two_sum cascade (each cell and every error term
// exact except the last limb's additions, ~2^-212 of |V| each) and
// renormalised once by two_sum passes. A V that fits one double comes out
// exactly, with zero lower limbs. This is the chosen path's conversion (f256
// accuracy), not the reference's MultiFloat renormalisation and addition.
template <int NC>
__device__ __forceinline__ qd crt_combine_qd(const double* a1, bool n1, const double* a2, bool n2) {
  constexpr int NCELL = NC + 4;
  double cell[NCELL];
#pragma unroll
  for (int k = 0; k < NCELL; k++) cell[k] = 0.0;
  const double s1 = n1 ? -1.0 : 1.0, s2 = n2 ? -1.0 : 1.0;
#pragma unroll
  for (int c = 0; c <= NC; c++) cell[c] = s2 * a2[c];
#pragma unroll
  for (int c = 0; c <= NC; c++) {
    const double hi = floor(__dmul_rn(a1[c], 0x1p-12));  // < 2^27
    const double lo = __fma_rn(-hi, 0x1p12, a1[c]);      // < 2^12
    cell[c + 2] = __fma_rn(s1 * lo, 0x1p27, cell[c + 2]);
    cell[c + 3] = __dadd_rn(cell[c + 3], s1 * hi);
  }
  auto normalise = [&]() {
#pragma unroll
    for (int k = 0; k < NCELL - 1; k++) {
      const double carry = floor(__dmul_rn(cell[k], 0x1p-39));
      cell[k] = __fma_rn(-carry, 0x1p39, cell[k]);
      cell[k + 1] = __dadd_rn(cell[k + 1], carry);
    }
  };
  normalise();
  const bool neg = cell[NCELL - 1] < 0.0;
  if (neg) {
#pragma unroll
    for (int k = 0; k < NCELL; k++) cell[k] = -cell[k];
    normalise();
  }
  double x0 = 0.0, x1 = 0.0, x2 = 0.0, x3 = 0.0;
#pragma unroll
  for (int k = NCELL - 1; k >= 0; k--) {
    const double v = scale_pow2(cell[k], CRT_BITS * k);
    double e;
    two_sum(x0, v, x0, e);
    two_sum(x1, e, x1, e);
    two_sum(x2, e, x2, e);
    x3 = __dadd_rn(x3, e);
  }
  two_sum(x2, x3, x2, x3);
  two_sum(x1, x2, x1, x2);
  two_sum(x0, x1, x0, x1);
  two_sum(x1, x2, x1, x2);
  two_sum(x2, x3, x2, x3);
  qd r{{x0, x1, x2, x3}};
  return neg ? qd_neg(r) : r;
}
// LC > 0: L == LC at compile time, tables from c_crt (weights as immediate
// operands), moduli loop unrolled.
template <int NC, int LC = 0>
__global__ void __launch_bounds__(256, 4) crt_qd_kernel(const uint8_t* __restrict__ g1, const uint8_t* __restrict__ g2,
                                                     int64_t plane, int64_t Np, int64_t m, int64_t n,
                                                     const int* __restrict__ expA, const int* __restrict__ expB,
                                                     const CrtTable* __restrict__ tab, double4* __restrict__ C) {
  __shared__ double w_sm[LC > 0 ? 1 : MAXL][NC];
  __shared__ double mch_sm[NC];
  const int L = LC > 0 ? LC : tab->L;
  if constexpr (LC == 0) {
    for (int i = threadIdx.x; i < L * NC; i += blockDim.x) w_sm[i / NC][i % NC] = tab->w[i / NC][i % NC];
    if (threadIdx.x < NC) mch_sm[threadIdx.x] = tab->mchunk[threadIdx.x];
  }
  sm100::griddep_launch_dependents();
  sm100::griddep_wait();  // the product residues come from the preceding GEMM
  if constexpr (LC == 0) __syncthreads();
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= m * n) return;
  const int64_t i = idx / n, j = idx % n;
  const int ea = expA[i], eb = expB[j];
  if (ea == EXP_NONFINITE || eb == EXP_NONFINITE) {
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    C[idx] = make_double4(nan, 0.0, 0.0, 0.0);
    return;
  }
  const size_t o = (size_t)i * Np + j;
  double acc1[NC + 1], acc2[NC + 1];
  bool n1, n2;
  if constexpr (LC > 0) {
    const CrtTable& ct = c_crt[LC - CRT_CONST_L0];
    n1 = crt_group_chunks<NC, LC>(g1 + o, plane, LC, ct.w, ct.mchunk, ct.inv_m, acc1);
    n2 = crt_group_chunks<NC, LC>(g2 + o, plane, LC, ct.w, ct.mchunk, ct.inv_m, acc2);
  } else {
    const double(*w_d)[NC] = w_sm;
    n1 = crt_group_chunks<NC>(g1 + o, plane, L, w_d, mch_sm, tab->inv_m, acc1);
    n2 = crt_group_chunks<NC>(g2 + o, plane, L, w_d, mch_sm, tab->inv_m, acc2);
  }
  const qd c = crt_combine_qd<NC>(acc1, n1, acc2, n2);  // X Y / 2^105 = G1 2^105 + G2 (+ Xl Yl / 2^105, omitted)
  const int shift = 105 - ((BETA_QD + 1022 - ea) + (BETA_QD + 1022 - eb));
  C[idx] = make_double4(scale_pow2(c.l[0], shift), scale_pow2(c.l[1], shift), scale_pow2(c.l[2], shift),
                        scale_pow2(c.l[3], shift));
}

}  // namespace ozaki

int ozaki_qd_gemm(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, bool atb,
                  cudaStream_t s) {
  using namespace ozaki;
  if (m == 0 || n == 0) return HP_OK;
  if (k == 0) {
    HP_CUDA_TRY(cudaMemsetAsync(c, 0, m * n * 32, s));
    return HP_OK;
  }
  DevTables* D;
  HP_TRY(device_tables(&D));
  // |G| < 2k 2^210: need log2 M >= 210 + ceil(log2 2k) + 2
  const int L = ozaki_moduli_for(2 * k, BETA_QD / 2);
  if (L < 0) {
    set_error("ozaki f256: k = %zu needs more moduli than the table holds", k);
    return HP_ERR_UNSUPPORTED;
  }
  const size_t Mp = round_up(m, GP_M), Np = round_up(n, GP_N), Kp = round_up(k, GB_K);
  DevBuf exps((Mp + Np) * sizeof(int), s);
  DevBuf ares((size_t)L * Mp * 2 * Kp, s), bres((size_t)L * Np * 2 * Kp, s);
  DevBuf gg((size_t)2 * L * Mp * Np, s);  // G1's residue planes, then G2's
  if (!exps.p || !ares.p || !bres.p || !gg.p) {
    set_error("ozaki f256: workspace allocation failed");
    return HP_ERR_CUDA;
  }
  int* expAp = exps.as<int>();  // A's row (or column) exponents, then B's column exponents
  int* expBp = expAp + Mp;
  HP_CUDA_TRY(cudaMemsetAsync(exps.p, 0, (Mp + Np) * sizeof(int), s));
  const double4* A4 = reinterpret_cast<const double4*>(a);
  const double4* B4 = reinterpret_cast<const double4*>(b);
  HP_TRY(launch_maxexp(A4, B4, m, n, k, atb, expAp, expBp, s));
  uint32_t* status = device_status(s);
  if (!status) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  const int rq = launch_residues_tc_qd(atb, L, A4, m, expAp, ares.as<int8_t>(), Mp, B4, n, expBp, bres.as<int8_t>(),
                                       Np, k, Kp, D->num_sms, status, s);
  if (rq != HP_OK && rq != HP_ERR_UNSUPPORTED) return rq;
  if (rq == HP_ERR_UNSUPPORTED) {  // residues of both operands as unsigned bytes, 4 entries per thread
    const unsigned tay = (unsigned)(Mp / RT_R);
    dim3 g((unsigned)(Kp / 16), tay + (unsigned)(Np / RT_R));
#define HP_RESQ(AC, LCV)                                                                                        \
  HP_CUDA_TRY(launch_k(true, residue_qd_ab_kernel<AC, 4, true, LCV>, g, dim3(256), 0, s, A4, (int64_t)m,         \
                       (int64_t)Mp, (const int*)expAp, ares.as<int8_t>(), tay, B4, (int64_t)n, (int64_t)Np,       \
                       (const int*)expBp, bres.as<int8_t>(), (int64_t)k, (int64_t)Kp, L))
#define HP_RESQ_L(AC)              \
  switch (L) {                     \
    case 28: HP_RESQ(AC, 28); break; \
    case 29: HP_RESQ(AC, 29); break; \
    case 30: HP_RESQ(AC, 30); break; \
    case 31: HP_RESQ(AC, 31); break; \
    case 32: HP_RESQ(AC, 32); break; \
    default: HP_RESQ(AC, 0); break;  \
  }
    if (!atb) {
      HP_RESQ_L(true)
    } else {
      HP_RESQ_L(false)
    }
#undef HP_RESQ_L
#undef HP_RESQ
  }
  uint8_t* g1 = gg.as<uint8_t>();
  uint8_t* g2 = g1 + (size_t)L * Mp * Np;
  // on CTA pairs; G1 = Xh Yh: A bytes [0, Kp), B bytes [Kp, 2Kp) of rows 2Kp long
  HP_TRY(ozaki_residue_gemm_pair(ares.as<int8_t>(), bres.as<int8_t>(), g1, L, Mp, Np, Kp, s, true, true, 2 * Kp, 0,
                                 Kp));
  // G2 = [Xh | Xl] [Yl ; Yh]: both over [0, 2Kp)
  HP_TRY(ozaki_residue_gemm_pair(ares.as<int8_t>(), bres.as<int8_t>(), g2, L, Mp, Np, 2 * Kp, s, false, true));
  const int rc = launch_crt_tc_qd(g1, Mp, Np, m, n, expAp, expBp, BETA_QD, L, reinterpret_cast<double4*>(c),
                                  D->num_sms, status, s);
  if (rc != HP_ERR_UNSUPPORTED) return rc;
  const int nc = host_tables().crt[L].nc;  // the FP64 CRT for other moduli counts
  const unsigned grid = (unsigned)((m * n + 255) / 256);
#define HP_CRTQ_LC(NCV, LCV)                                                                                       \
  if (nc == NCV && L == LCV) {                                                                                     \
    HP_CUDA_TRY(launch_k(true, crt_qd_kernel<NCV, LCV>, dim3(grid), dim3(256), 0, s,                                \
                         (const uint8_t*)g1, (const uint8_t*)g2, (int64_t)(Mp * Np),                               \
                         (int64_t)Np, (int64_t)m, (int64_t)n, (const int*)expAp, (const int*)expBp,                 \
                         (const CrtTable*)(D->crt + L), reinterpret_cast<double4*>(c)));                            \
    return HP_OK;                                                                                                  \
  }
  HP_CRTQ_LC(6, 28) HP_CRTQ_LC(6, 29) HP_CRTQ_LC(6, 30) HP_CRTQ_LC(6, 31) HP_CRTQ_LC(6, 32)
  HP_CRTQ_LC(7, 28) HP_CRTQ_LC(7, 29) HP_CRTQ_LC(7, 30) HP_CRTQ_LC(7, 31) HP_CRTQ_LC(7, 32)
#undef HP_CRTQ_LC
#define HP_CRTQ(NC)                                                                                                  \
  case NC:                                                                                                           \
    HP_CUDA_TRY(launch_k(true, crt_qd_kernel<NC>, dim3(grid), dim3(256), 0, s, (const uint8_t*)g1,                   \
                         (const uint8_t*)g2, (int64_t)(Mp * Np), (int64_t)Np, (int64_t)m, (int64_t)n,  \
                         (const int*)expAp, (const int*)expBp, (const CrtTable*)(D->crt + L),               \
                         reinterpret_cast<double4*>(c)));                                                            \
    break;
  switch (nc) {
    HP_CRTQ(5) HP_CRTQ(6) HP_CRTQ(7) HP_CRTQ(8)
    default:
      set_error("ozaki f256: unsupported chunk count %d", nc);
      return HP_ERR_UNSUPPORTED;
  }
#undef HP_CRTQ
  return HP_OK;
}

// Host-pointer f256 GEMM C = op(A) B (chosen mode) with the PCIe copies
// overlapped, as ozaki_dd_gemm_host does for f128: op(A) in row panels (with
// atb, A's column panels copied into compact k x rows matrices), B and C in
// two column panels for n >= 1024, copies in the order B0, A0, B1, the rest
// of A. Each panel's exponents and residue rows are formed once; each block of
// C takes its two group GEMMs and the tensor-core CRT and goes back while later
// blocks compute. Every entry's arithmetic is that of ozaki_qd_gemm, so the
// result is bit-identical to the one-shot path. Moduli counts outside the
// tensor-core kernels' 28..32 take the one-shot path with plain copies.
int ozaki_qd_gemm_host(const double* a, const double* b, double* c, size_t m, size_t n, size_t k, bool atb) {
  using namespace ozaki;
  DevTables* D;
  HP_TRY(device_tables(&D));
  const int L = ozaki_moduli_for(2 * k, BETA_QD / 2);
  if (L < 0) {
    set_error("ozaki f256: k = %zu needs more moduli than the table holds", k);
    return HP_ERR_UNSUPPORTED;
  }
  cudaStream_t s = library_stream(), sin = library_copy_stream(0), sout = library_copy_stream(1);
  if (L < CRT_CONST_L0 || L >= CRT_CONST_L0 + CRT_CONST_N) {
    DevBuf da(m * k * 32, s), db(k * n * 32, s), dc(m * n * 32, s);
    if (!da.p || !db.p || !dc.p) {
      set_error("ozaki f256: workspace allocation failed");
      return HP_ERR_CUDA;
    }
    HP_CUDA_TRY(cudaMemcpyAsync(da.p, a, m * k * 32, cudaMemcpyHostToDevice, s));
    HP_CUDA_TRY(cudaMemcpyAsync(db.p, b, k * n * 32, cudaMemcpyHostToDevice, s));
    HP_TRY(ozaki_qd_gemm(da.as<double>(), db.as<double>(), dc.as<double>(), m, n, k, atb, s));
    HP_CUDA_TRY(cudaMemcpyAsync(c, dc.p, m * n * 32, cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    return consume_device_status(s);
  }
  const size_t Kp = round_up(k, GB_K);
  const size_t panels_wanted = m >= 2048 ? 16 : m >= 1024 ? 8 : 4;
  const size_t pr = round_up((m + panels_wanted - 1) / panels_wanted, GP_M);  // rows per A panel
  const size_t np = (m + pr - 1) / pr;
  const size_t pc = round_up((n + (n >= 1024 ? 1 : 0)) / (n >= 1024 ? 2 : 1), GP_N);  // columns per B panel
  const size_t nq = (n + pc - 1) / pc;
  const size_t Mpa = np * pr;
  if (pr / GB_M * (pc / GB_N) * (size_t)L > (size_t)INT32_MAX || 2 * Kp > (size_t)INT32_MAX) {
    set_error("ozaki f256: problem too large");
    return HP_ERR_INVALID_ARG;
  }
  DevBuf dA(m * k * 32, s), dB(k * n * 32, s), dC(m * n * 32, s);
  DevBuf exps((Mpa + nq * pc) * sizeof(int), s);
  DevBuf ares((size_t)L * Mpa * 2 * Kp, s), bres((size_t)L * nq * pc * 2 * Kp, s), gg((size_t)2 * L * pr * pc, s);
  if (!dA.p || !dB.p || !dC.p || !exps.p || !ares.p || !bres.p || !gg.p) {
    set_error("ozaki f256: workspace allocation failed");
    return HP_ERR_CUDA;
  }
  EventSet ev(1 + nq + np + np * nq);
  if (!ev.ok()) {
    set_error("ozaki f256: event creation failed");
    return HP_ERR_CUDA;
  }
  StreamsDrain drain{s, sin, sout};
  cudaEvent_t ready = ev.ev[0];
  cudaEvent_t* eB = ev.ev.data() + 1;
  cudaEvent_t* eA = eB + nq;
  cudaEvent_t* eC = eA + np;
  int* expA = exps.as<int>();
  int* expB = expA + Mpa;
  HP_CUDA_TRY(cudaEventRecord(ready, s));
  HP_CUDA_TRY(cudaStreamWaitEvent(sin, ready, 0));
  HP_CUDA_TRY(cudaStreamWaitEvent(sout, ready, 0));
  auto copy_b = [&](size_t j) -> int {
    const size_t j0 = j * pc, nj = std::min(pc, n - j0);
    HP_CUDA_TRY(cudaMemcpy2DAsync(dB.as<char>() + j0 * k * 32, nj * 32, reinterpret_cast<const char*>(b) + j0 * 32,
                                  n * 32, nj * 32, k, cudaMemcpyHostToDevice, sin));
    HP_CUDA_TRY(cudaEventRecord(eB[j], sin));
    return HP_OK;
  };
  auto copy_a = [&](size_t i) -> int {
    const size_t r0 = i * pr, mi = std::min(pr, m - r0);
    if (atb)
      HP_CUDA_TRY(cudaMemcpy2DAsync(dA.as<char>() + r0 * k * 32, mi * 32, reinterpret_cast<const char*>(a) + r0 * 32,
                                    m * 32, mi * 32, k, cudaMemcpyHostToDevice, sin));
    else
      HP_CUDA_TRY(cudaMemcpyAsync(dA.as<char>() + r0 * k * 32, reinterpret_cast<const char*>(a) + r0 * k * 32,
                                  mi * k * 32, cudaMemcpyHostToDevice, sin));
    HP_CUDA_TRY(cudaEventRecord(eA[i], sin));
    return HP_OK;
  };
  HP_TRY(copy_b(0));
  HP_TRY(copy_a(0));
  for (size_t j = 1; j < nq; j++) HP_TRY(copy_b(j));
  for (size_t i = 1; i < np; i++) HP_TRY(copy_a(i));
  uint32_t* status = device_status(s);
  if (!status) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  HP_CUDA_TRY(cudaMemsetAsync(exps.p, 0, (Mpa + nq * pc) * sizeof(int), s));  // maxima merge by atomicMax
  for (size_t i = 0; i < np; i++) {
    const size_t r0 = i * pr, mi = std::min(pr, m - r0), Mpi = round_up(mi, GP_M);
    const double4* A4 = dA.as<const double4>() + r0 * k;
    int8_t* aresi = ares.as<int8_t>() + (size_t)L * r0 * 2 * Kp;  // L planes of Mpi x 2 Kp
    HP_CUDA_TRY(cudaStreamWaitEvent(s, eA[i], 0));
    HP_TRY(launch_maxexp(A4, (const double4*)nullptr, mi, 0, k, atb, expA + r0, nullptr, s));
    int rc = launch_residues_tc_qd(atb, L, A4, mi, expA + r0, aresi, Mpi, nullptr, 0, nullptr, nullptr, 0, k, Kp,
                                   D->num_sms, status, s);
    if (rc != HP_OK) return rc == HP_ERR_UNSUPPORTED ? HP_ERR_CUDA : rc;  // device buffers are aligned
    for (size_t j = 0; j < nq; j++) {
      const size_t j0 = j * pc, nj = std::min(pc, n - j0);
      int8_t* bresj = bres.as<int8_t>() + (size_t)L * j0 * 2 * Kp;  // L planes of pc x 2 Kp
      if (i == 0) {
        const double4* B4 = dB.as<const double4>() + j0 * k;
        HP_CUDA_TRY(cudaStreamWaitEvent(s, eB[j], 0));
        HP_TRY(launch_maxexp((const double4*)nullptr, B4, 0, nj, k, false, nullptr, expB + j0, s));
        rc = launch_residues_tc_qd(false, L, nullptr, 0, nullptr, nullptr, 0, B4, nj, expB + j0, bresj, pc, k, Kp,
                                   D->num_sms, status, s);
        if (rc != HP_OK) return rc == HP_ERR_UNSUPPORTED ? HP_ERR_CUDA : rc;
      }
      uint8_t* g1 = gg.as<uint8_t>();
      uint8_t* g2 = g1 + (size_t)L * Mpi * pc;
      HP_TRY(ozaki_residue_gemm_pair(aresi, bresj, g1, L, Mpi, pc, Kp, s, true, true, 2 * Kp, 0, Kp));
      HP_TRY(ozaki_residue_gemm_pair(aresi, bresj, g2, L, Mpi, pc, 2 * Kp, s, false, true));
      double* Cij = dC.as<double>() + (r0 * n + j0) * 4;
      HP_TRY(launch_crt_tc_qd(g1, Mpi, pc, mi, nj, expA + r0, expB + j0, BETA_QD, L, reinterpret_cast<double4*>(Cij),
                              D->num_sms, status, s, n));
      cudaEvent_t e = eC[i * nq + j];
      HP_CUDA_TRY(cudaEventRecord(e, s));
      HP_CUDA_TRY(cudaStreamWaitEvent(sout, e, 0));
      HP_CUDA_TRY(cudaMemcpy2DAsync(reinterpret_cast<char*>(c) + (r0 * n + j0) * 32, n * 32, Cij, n * 32, nj * 32, mi,
                                    cudaMemcpyDeviceToHost, sout));
    }
  }
  HP_CUDA_TRY(cudaStreamSynchronize(sout));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return consume_device_status(s);
}


// ===========================================================================
// Cholesky with the trailing matrix kept in the residue domain.
//
// With D = diag(2^e_i) chosen so that (D S D)_ii lies in [2^(2B-2), 2^(2B)),
// B = 106, the scaled matrix A~ = round(D S D) is an integer matrix whose
// Schur complements stay below 2^(2B) in magnitude (for an SPD matrix
// |a_ij| <= sqrt(a_ii a_jj) and the diagonal only decreases). A~ is held as
// residues modulo L = 29 moduli (M > 2^(2B+3)). Per block column of width
// nb = 64:
//   1. CRT the panel (rows kb.., columns kb..kb+nb) back to f128 integers;
//   2. factor the nb x nb diagonal block in f128 (one CTA) and invert it;
//   3. L21 = A21 L11^-T in f128 and round L21 to integers (|L21| < 2^B);
//   4. subtract L21 L21^T from the trailing residues with the int8 tcgen05
//      GEMM (exact modular arithmetic: no rounding at all in the update).
// The factor returned is L = D^-1 L~, in f128. Errors: the f128 rounding of
// the panel values (2^-104 relative) and the rounding of L21 to B-bit
// integers, i.e. an f128-quality factor whose O(n^3) work ran on the tensor
// cores.
// ===========================================================================
namespace ozaki {

constexpr int BETA_CH = 106;
constexpr int CH_NB = 64;

using RnsErr = FactorErr;

__global__ void rns_scale_kernel(const dd* __restrict__ S, int64_t n, int beta, int* __restrict__ e,
                                 RnsErr* err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double d = S[i * n + i].hi;
  if (!(d > 0.0) || !isfinite(d)) {
    err->flag = 1;
    atomicMin(&err->pivot, (long long)i);
    e[i] = 0;
    return;
  }
  const int E = exp_field(d) - 1022;  // d = m 2^E, m in [0.5, 1)
  e[i] = (2 * beta - E) >> 1;         // floor((2B - E) / 2)
}

// Balanced base-2^22 digits of rint(v), |v| < 2^214 (exact).
__device__ __forceinline__ void int_digits10(double v, int32_t* d) {
  double a = fabs(rint(v));
  int32_t s = signbit(v) ? -1 : 1;
#pragma unroll
  for (int c = NDIG2 - 1; c >= 1; c--) {
    const double sc = scale_pow2(1.0, -22 * c), up = scale_pow2(1.0, 22 * c);
    double t = floor(__dmul_rn(a, sc));
    a = __dsub_rn(a, __dmul_rn(t, up));
    d[c] = s * (int32_t)t;
  }
  d[0] = s * (int32_t)a;
}

// Res[l][i][j] = round((D S D)_ij) mod m_l (unbalanced bytes) for the tiles
// that meet the lower triangle of n x n (the factorisation reads no other
// entry below row n). Block tile 64 rows x 32 columns, 8 columns per thread.
// EPT consecutive entries of a row per thread (tile 64 rows x 4 EPT
// columns); LC > 0: L == LC at compile time (moduli loop unrolled, each
// modulus' constants immediate operands). Every entry's digits and residues
// are the same for any EPT and LC.
template <int EPT, int LC>
__global__ void __launch_bounds__(256) rns_init_kernel(const dd* __restrict__ S, int64_t n, const int* __restrict__ e,
                                                       int L_, int64_t Rp, uint8_t* __restrict__ res) {
  const int L = LC > 0 ? LC : L_;
  const int64_t row0 = (int64_t)blockIdx.y * 64, col0 = (int64_t)blockIdx.x * (4 * EPT);
  if (row0 >= n || col0 >= n || col0 > row0 + 63) return;
  const int t = threadIdx.x;
  const int64_t i = (int64_t)blockIdx.y * 64 + t / 4;
  const int64_t j0 = col0 + EPT * (t % 4);
  int32_t dig[EPT][NDIG2];
#pragma unroll
  for (int q = 0; q < EPT; q++)
#pragma unroll
    for (int c = 0; c < NDIG2; c++) dig[q][c] = 0;
  if (i < n) {
#pragma unroll
    for (int q = 0; q < EPT; q++) {
      const int64_t j = j0 + q;
      if (j < n) {
        const dd v = S[i * n + j];
        const int sft = e[i] + e[j];
        int32_t dh[NDIG2], dl[NDIG2];
        int_digits10(scale_pow2(v.hi, sft), dh);
        int_digits10(scale_pow2(v.lo, sft), dl);
#pragma unroll
        for (int c = 0; c < NDIG2; c++) dig[q][c] = dh[c] + dl[c];
#pragma unroll
        for (int c = 0; c < NDIG2 - 1; c++) {
          int32_t carry = (dig[q][c] + (1 << 21)) >> 22;
          dig[q][c] -= carry << 22;
          dig[q][c + 1] += carry;
        }
      }
    }
  }
#pragma unroll(LC > 0 ? LC : 1)
  for (int l = 0; l < L; l++) {
    const uint32_t m = (uint32_t)c_tab.mod[l];
    uint32_t w0 = 0, w1 = 0;
#pragma unroll
    for (int q = 0; q < EPT; q++) {
      int32_t x1 = 0, x2 = 0;
#pragma unroll
      for (int c = 0; c < 5; c++) x1 += dig[q][c] * c_tab.pw[l][c];
#pragma unroll
      for (int c = 5; c < NDIG2; c++) x2 += dig[q][c] * c_tab.pw[l][c];
      uint32_t r = mod_reduce(x1, l) + mod_reduce(x2, l);
      if (r >= m) r -= m;
      if (q < 4)
        w0 |= r << (8 * q);
      else
        w1 |= r << (8 * (q - 4));
    }
    uint8_t* dst = res + (size_t)l * Rp * Rp + (size_t)i * Rp + j0;
    if constexpr (EPT == 8)
      *reinterpret_cast<uint2*>(dst) = make_uint2(w0, w1);
    else
      *reinterpret_cast<uint32_t*>(dst) = w0;
  }
}

// P[r][c] = CRT(Res[.][r0 + r][c0 + c]) as an f128 integer, r < R, c < C.
// LC > 0: L == LC at compile time, tables from c_crt (weights as immediate
// operands), moduli loop unrolled.
template <int NC, int LC = 0>
__global__ void __launch_bounds__(256) crt_block_kernel(const uint8_t* __restrict__ res, int64_t ld, int64_t plane,
                                                        int64_t r0, int64_t c0, int64_t R, int64_t C,
                                                        const CrtTable* __restrict__ tab, dd* __restrict__ P) {
  __shared__ double w_sm[LC > 0 ? 1 : MAXL][NC];
  __shared__ double mch_sm[NC];
  const int L = LC > 0 ? LC : tab->L;
  if constexpr (LC == 0) {
    for (int i = threadIdx.x; i < L * NC; i += blockDim.x) w_sm[i / NC][i % NC] = tab->w[i / NC][i % NC];
    if (threadIdx.x < NC) mch_sm[threadIdx.x] = tab->mchunk[threadIdx.x];
  }
  const double(*w_s)[NCMAX] = LC > 0 ? c_crt[LC > 0 ? LC - CRT_CONST_L0 : 0].w : nullptr;
  const double(*w_d)[NC] = w_sm;
  const double* mch_s = LC > 0 ? c_crt[LC > 0 ? LC - CRT_CONST_L0 : 0].mchunk : mch_sm;
  const double inv_m = LC > 0 ? c_crt[LC > 0 ? LC - CRT_CONST_L0 : 0].inv_m : tab->inv_m;
  sm100::griddep_launch_dependents();
  sm100::griddep_wait();  // the residues come from the preceding GEMM
  if constexpr (LC == 0) __syncthreads();
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= R * C) return;
  const int64_t r = idx / C, c = idx % C;
  const uint8_t* rp = res + (size_t)(r0 + r) * ld + c0 + c;
  double acc[NC + 1];
#pragma unroll
  for (int q = 0; q <= NC; q++) acc[q] = 0.0;
#pragma unroll(LC > 0 ? 8 : 1)
  for (int l0 = 0; l0 < L; l0 += 8) {
    uint32_t v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) v[u] = (l0 + u < L) ? (uint32_t)__ldg(rp + (size_t)(l0 + u) * plane) : 0u;
#pragma unroll
    for (int u = 0; u < 8; u++) {
      if (l0 + u >= L) break;
      const double x = byte_to_double(v[u]);
#pragma unroll
      for (int q = 0; q < NC; q++) acc[q] = __fma_rn(x, LC > 0 ? w_s[l0 + u][q] : w_d[l0 + u][q], acc[q]);
    }
  }
  bool neg;
  dd s = crt_finish<NC>(acc, mch_s, inv_m, &neg);
  P[idx] = neg ? dd_neg(s) : s;
}

// Factor the jb x jb block P[0..jb)[0..jb) (row stride jb, symmetric values)
// in f128: L~11 scaled back to Lout, and for the panel solve the unit lower
// factor L1 = L~11 diag(1 / l_jj) (row-major 64 x 64, zero on and above the
// diagonal) with rinv[j] = 1 / l_jj. The block is padded to 64 x 64 with the
// identity, so every step has the same shape. Columns go in pairs
// (2q, 2q + 1); iteration q (one barrier):
//   warp 31 (the critical path): pair q + 1 gets its last updates from
//     pair q (four independent chains per lane), then column 2q + 2 is
//     pivoted and scaled, applied to column 2q + 3 inside the warp, and
//     column 2q + 3 is pivoted and scaled; every lane forms each 1/sqrt from
//     the same value, so nothing needs broadcasting but the two l values.
//     The scaled columns replace their entries of the block in shared
//     memory (no other warp touches columns 2q + 2, 2q + 3 in iteration q).
//   the bulk warps (those on the three other schedulers, warp % 4 != 3):
//     pair q applied to every column k >= 2q + 4 (rows i >= k; a table
//     ordered by column makes these the first T slots).
//   the other warps of warp 31's scheduler stay idle, so that nothing
//     competes with the pivot chain for its scheduler's FP64 pipe.
// Lout, L1 and rinv are written by all warps after the last pair. Each
// entry receives its column updates in column order, as in a plain
// right-looking Cholesky; dd_fms_fast (f128-level accuracy, not the
// reference's bits).
constexpr int CI_THREADS = 1024;
constexpr int CI_BULK = CI_THREADS / 4 * 3;  // warps with warp % 4 != 3
__global__ void __launch_bounds__(CI_THREADS) chol_block_kernel(const dd* __restrict__ P, int jb, int64_t kb,
                                                                int64_t n, const int* __restrict__ e,
                                                                dd* __restrict__ Lout, dd* __restrict__ L1g,
                                                                dd* __restrict__ rinvg, RnsErr* err) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  dd* A = reinterpret_cast<dd*>(sm_raw);  // [64][65]; factored columns hold L~ below the diagonal
  __shared__ dd rinv[64], dpiv[64];       // 1 / l_jj and the pivot a_jj (l_jj = a_jj / l_jj)
  __shared__ uint16_t tab[2016];          // (i << 6) | k, column k = 63..1, rows i = k..63
  __shared__ int esh[64];
  __shared__ int fail;
  const int t = threadIdx.x, lane = t % 32, warp = t / 32;
  const bool critical = warp == CI_THREADS / 32 - 1;
  const bool bulk = warp % 4 != 3;
  const int bt = (warp / 4 * 3 + warp % 4) * 32 + lane;  // bulk thread index
  sm100::griddep_launch_dependents();
  sm100::griddep_wait();  // P comes from the preceding CRT
  if (err->flag) return;
  if (t < 64) esh[t] = t < jb ? e[kb + t] : 0;
  if (t == 0) fail = 0;
#pragma unroll 4
  for (int q = t; q < 64 * 64; q += CI_THREADS) {
    const int r = q / 64, c = q % 64;
    A[r * 65 + c] = (r < jb && c < jb) ? P[r * jb + c] : dd_from(r == c ? 1.0 : 0.0);
    if (c >= 1 && r >= c) tab[(63 - c) * (64 - c) / 2 + (r - c)] = (uint16_t)((r << 6) | c);
    if (c >= r) L1g[r * 64 + c] = dd{0.0, 0.0};  // L1 is stored strictly lower
  }
  __syncthreads();
  // Pivot p on warp 31, branch-free: every lane forms r = 1/sqrt(d) from
  // the same d; a failure is flagged once.
  auto pivot = [&](int p, dd d, dd& r) -> bool {
    if (!(d.hi > 0.0)) {
      if (lane == 0) {
        fail = 1;
        err->flag = 1;
        err->pivot = kb + p;
      }
      return false;
    }
    r = dd_rsqrt_fast(d);
    if (lane == 0) {
      rinv[p] = r;
      dpiv[p] = d;  // l_jj = d r is formed after the loop, off the pivot chain
    }
    return true;
  };
  // Factor the pair (c0, c0 + 1) on warp 31 from its updated entries a?0
  // (column c0) and a?1 (column c0 + 1) at rows c0 + lane and c0 + 32 + lane;
  // the scaled columns go to A's columns c0, c0 + 1 below the diagonal.
  auto factor_pair = [&](int c0, dd a00, dd a10, dd a01, dd a11) -> bool {
    const int c1 = c0 + 1, i0 = c0 + lane, i1 = c0 + 32 + lane;
    dd r0, r1;
    const dd d0 = {__shfl_sync(0xffffffffu, a00.hi, 0), __shfl_sync(0xffffffffu, a00.lo, 0)};
    if (!pivot(c0, d0, r0)) return false;
    const dd s00 = dd_mul(a00, r0), s10 = dd_mul(a10, r0);
    const dd l10 = {__shfl_sync(0xffffffffu, s00.hi, 1), __shfl_sync(0xffffffffu, s00.lo, 1)};  // l_{c1,c0}
    a01 = dd_fms_fast(a01, s00, l10);
    a11 = dd_fms_fast(a11, s10, l10);
    const dd d1 = {__shfl_sync(0xffffffffu, a01.hi, 1), __shfl_sync(0xffffffffu, a01.lo, 1)};
    if (!pivot(c1, d1, r1)) return false;
    const dd s01 = dd_mul(a01, r1), s11 = dd_mul(a11, r1);
    if (i0 < 64 && i0 > c0) A[i0 * 65 + c0] = s00;
    if (i1 < 64) A[i1 * 65 + c0] = s10;
    if (i0 < 64 && i0 > c1) A[i0 * 65 + c1] = s01;
    if (i1 < 64) A[i1 * 65 + c1] = s11;
    return true;
  };
  if (critical) {  // pair 0
    const int i0 = lane, i1 = 32 + lane;
    factor_pair(0, A[i0 * 65], A[i1 * 65], A[i0 * 65 + 1], A[i1 * 65 + 1]);
  }
  __syncthreads();
  for (int q = 0; q < 32; q++) {
    if (fail) return;
    const int ca = 2 * q, cb = ca + 1;  // pair q's columns (scaled L~ below the diagonal)
    if (critical) {
      if (q < 31) {
        // pair q + 1 (columns c0, c0 + 1): last updates from pair q. Indices
        // are clamped so the chains run unconditionally; stores are predicated.
        const int c0 = 2 * q + 2, c1 = c0 + 1;
        const int i0c = min(c0 + lane, 63), i1c = min(c0 + 32 + lane, 63);
        const dd la0 = A[c0 * 65 + ca], la1 = A[c1 * 65 + ca], lb0 = A[c0 * 65 + cb], lb1 = A[c1 * 65 + cb];
        const dd lai = A[i0c * 65 + ca], laj = A[i1c * 65 + ca], lbi = A[i0c * 65 + cb], lbj = A[i1c * 65 + cb];
        const dd a00 = dd_fms_fast(dd_fms_fast(A[i0c * 65 + c0], lai, la0), lbi, lb0);
        const dd a10 = dd_fms_fast(dd_fms_fast(A[i1c * 65 + c0], laj, la0), lbj, lb0);
        const dd a01 = dd_fms_fast(dd_fms_fast(A[i0c * 65 + c1], lai, la1), lbi, lb1);
        const dd a11 = dd_fms_fast(dd_fms_fast(A[i1c * 65 + c1], laj, la1), lbj, lb1);
        factor_pair(c0, a00, a10, a01, a11);
      }
    } else if (bulk) {
      const int m = 60 - 2 * q;  // columns >= 2q + 4: T = m (m + 1) / 2 slots
      const int Tn = m > 0 ? m * (m + 1) / 2 : 0;
      for (int u = bt; u < Tn; u += CI_BULK) {
        const int ent = tab[u], i = ent >> 6, kk = ent & 63;
        A[i * 65 + kk] =
            dd_fms_fast(dd_fms_fast(A[i * 65 + kk], A[i * 65 + ca], A[kk * 65 + ca]), A[i * 65 + cb], A[kk * 65 + cb]);
      }
    }
    __syncthreads();
  }
  // outputs of every column: L~ (scaled back) to Lout, L1 = L~ / l_jj, rinv
  for (int u = t; u < 64 * 64; u += CI_THREADS) {
    const int i = u / 64, j = u % 64;
    if (i < j) continue;
    const dd rj = rinv[j];
    const dd v = i == j ? dd_mul(dpiv[j], rj) : A[i * 65 + j];
    if (i > j) L1g[i * 64 + j] = dd_mul(v, rj);
    if (i < jb && j < jb) {
      const int sh = -esh[i];
      Lout[(kb + i) * n + kb + j] = dd_renorm(scale_pow2(v.hi, sh), scale_pow2(v.lo, sh));
    }
  }
  if (t < 64) rinvg[t] = rinv[t];
}

// L21 = P21 L~11^-T for the rows below the diagonal block. With
// L~11 = L1 D (L1 unit lower, D = diag(l_jj)), each row z of z L1^T = P21 is a
// forward substitution without divisions, z_c = p_c - sum_{k<c} z_k L1[c][k],
// and L21 = z D^-1, for panel rows r0 <= r < m. One warp per row; lane c owns
// columns c and c + 32, z_k
// is broadcast by shuffle as it becomes final; L1 sits in shared memory with
// zeros on and above the diagonal, so every update is unconditional.
// dd_fms_fast accumulation (f128 accuracy). Epilogue: each entry is rounded
// to an integer, written scaled back to Lout (rows t0.., columns kb..) and,
// as balanced bytes modulo every modulus, to the L~ residue planes.
// LC > 0: L == LC at compile time (the residue epilogue's moduli loop is
// unrolled with each modulus' constants as immediate operands).
template <int LC = 0>
__global__ void __launch_bounds__(256) panel_trsm_kernel(const dd* __restrict__ P21, const dd* __restrict__ L1g,
                                                         const dd* __restrict__ rinvg, int64_t r0, int64_t m, int jb,
                                                         int64_t t0,
                                                         int64_t kb, int64_t n, const int* __restrict__ e,
                                                         dd* __restrict__ Lout, int L, int8_t* __restrict__ lres,
                                                         int64_t ld, int64_t plane) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  dd(*L1s)[CH_NB + 1] = reinterpret_cast<dd(*)[CH_NB + 1]>(sm_raw);  // [CH_NB][CH_NB + 1]
  __shared__ dd rs[CH_NB];
  sm100::griddep_launch_dependents();
  sm100::griddep_wait();  // L1 and 1/l come from the preceding block factor
  for (int q = threadIdx.x; q < CH_NB * CH_NB; q += blockDim.x) L1s[q / CH_NB][q % CH_NB] = L1g[q];
  if (threadIdx.x < CH_NB) rs[threadIdx.x] = rinvg[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x % 32;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const int64_t nw = (int64_t)gridDim.x * blockDim.x / 32;
  for (int64_t r = r0 + w0; r < m; r += nw) {
    dd z0 = lane < jb ? P21[r * jb + lane] : dd{0.0, 0.0};
    dd z1 = lane + 32 < jb ? P21[r * jb + lane + 32] : dd{0.0, 0.0};
    const int kend = min(jb, 32);
    for (int k = 0; k < kend; k++) {  // columns k < 32: both halves still move
      const dd zk = {__shfl_sync(0xffffffffu, z0.hi, k), __shfl_sync(0xffffffffu, z0.lo, k)};
      z0 = dd_fms_fast(z0, zk, L1s[lane][k]);
      z1 = dd_fms_fast(z1, zk, L1s[lane + 32][k]);
    }
    for (int k = 32; k < jb; k++) {  // columns k >= 32: only the upper half moves
      const dd zk = {__shfl_sync(0xffffffffu, z1.hi, k - 32), __shfl_sync(0xffffffffu, z1.lo, k - 32)};
      z1 = dd_fms_fast(z1, zk, L1s[lane + 32][k]);
    }
    const int sh = -e[t0 + r];
    for (int h = 0; h < 2; h++) {
      const int c = lane + 32 * h;
      if (c >= jb) continue;
      const dd x = dd_mul(h ? z1 : z0, rs[c]);
      // L~21 rounded to an integer: scaled back into Lout, and its residues
      // into row t0 + r, column kb + c of the L~ residue planes
      const dd xr = dd_renorm(rint(x.hi), rint(x.lo));
      Lout[(t0 + r) * n + kb + c] = dd_renorm(scale_pow2(xr.hi, sh), scale_pow2(xr.lo, sh));
      int32_t D[NDIG];
      element_digits(make_double2(x.hi, x.lo), 0, D);
      int8_t* dst = lres + (t0 + r) * ld + kb + c;
      if constexpr (LC > 0) {
#pragma unroll
        for (int l = 0; l < LC; l++) dst[(size_t)l * plane] = (int8_t)balanced_byte(D, l, c_tab.mod[l]);
      } else {
        for (int l = 0; l < L; l++) dst[(size_t)l * plane] = (int8_t)balanced_byte(D, l, c_tab.mod[l]);
      }
    }
  }
}


}  // namespace ozaki


// res[l][r0 + i][c0 + j] -= sum_p A[l][i][p] B[l][j][p] (mod m_l) for
// i < R, j < CH_NB, p < K: A = R rows of L~ residues from arow, B = CH_NB
// rows from brow (rows KL bytes apart, planes plane_stride bytes apart). The
// maps cover rows_a / rows_b rows and the first kv bytes of each: the
// k-blocks past kv (K is kv rounded up to the 128-byte k-block) and the tile
// rows past the maps read zeros, so the residue planes need no zeroing. One
// launch of the 128 x 64 tile GEMM on at most max_ctas CTAs.
static int rns_panel_update(const uint8_t* arow, size_t rows_a, const uint8_t* brow, size_t rows_b, size_t KL,
                            size_t kv, size_t plane_stride, int L, size_t R, size_t K, uint8_t* res, size_t Np,
                            size_t r0, size_t c0, int max_ctas, cudaStream_t s, bool pdl = false) {
  using namespace ozaki;
  constexpr int BN = CH_NB;
  if (R == 0 || K == 0 || rows_a == 0 || rows_b == 0) return HP_OK;
  static bool attr_set[64] = {};
  int dev = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 64 && !attr_set[dev]) {
    HP_CUDA_TRY(cudaFuncSetAttribute(i8_gemm_mod_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     GemmCfg<BN>::SMEM));
    attr_set[dev] = true;
  }
  CUtensorMap mapA, mapB;
  HP_TRY(make_map(&mapA, arow, kv, rows_a, L, GB_M, plane_stride, KL));
  HP_TRY(make_map(&mapB, brow, kv, rows_b, L, BN, plane_stride, KL));
  uint32_t* status = device_status(s);
  if (!status) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  const int tiles_m = (int)((R + GB_M - 1) / GB_M);
  const int grid = std::max(1, std::min(L * tiles_m, max_ctas));
  const int nkb = (int)(K / GB_K), kb_chunk = MAX_K_CHUNK / GB_K;
  for (int k0 = 0; k0 < nkb; k0 += kb_chunk) {
    HP_CUDA_TRY(launch_k(pdl && k0 == 0, i8_gemm_mod_kernel<BN>, dim3(grid), dim3(256), GemmCfg<BN>::SMEM, s, mapA,
                         mapB, L, tiles_m, 1, k0, std::min(nkb, k0 + kb_chunk), 0, 2, res, (int64_t)Np,
                         (int64_t)(Np * Np), (int64_t)r0, (int64_t)c0, status));
  }
  return HP_OK;
}

// The two streams of the panel pipeline (one pair per device, created once):
// the diagonal path at the device's greatest priority, so that its blocks
// take SMs ahead of the other path's as they free up, and the other path at
// the least priority.
static int pipeline_streams(cudaStream_t* hi, cudaStream_t* lo) {
  static cudaStream_t streams[64][2] = {};
  static std::mutex mu;
  int dev = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("device ordinal %d out of range", dev);
    return HP_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!streams[dev][0]) {
    int least = 0, greatest = 0;
    HP_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    HP_CUDA_TRY(cudaStreamCreateWithPriority(&streams[dev][0], cudaStreamNonBlocking, greatest));
    HP_CUDA_TRY(cudaStreamCreateWithPriority(&streams[dev][1], cudaStreamNonBlocking, least));
  }
  *hi = streams[dev][0];
  *lo = streams[dev][1];
  return HP_OK;
}

// Events of one factorisation. The pipeline streams start after the
// caller's stream; on destruction both are joined back into it, so that
// stream-ordered frees of the workspace come after them.
struct PipelineEvents {
  cudaStream_t s, s1, s2;
  cudaEvent_t F, Td, Gd, Cr, E, start, join1, join2;
  bool ok = true;
  PipelineEvents(cudaStream_t caller, cudaStream_t hi, cudaStream_t lo) : s(caller), s1(hi), s2(lo) {
    for (cudaEvent_t* e : {&F, &Td, &Gd, &Cr, &E, &start, &join1, &join2})
      ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventRecord(start, s) == cudaSuccess && cudaStreamWaitEvent(s1, start, 0) == cudaSuccess &&
         cudaStreamWaitEvent(s2, start, 0) == cudaSuccess;
  }
  void join() {
    if (!ok) return;
    if (cudaEventRecord(join1, s1) == cudaSuccess) cudaStreamWaitEvent(s, join1, 0);
    if (cudaEventRecord(join2, s2) == cudaSuccess) cudaStreamWaitEvent(s, join2, 0);
  }
  ~PipelineEvents() {
    join();
    for (cudaEvent_t e : {F, Td, Gd, Cr, E, start, join1, join2}) cudaEventDestroy(e);
  }
};

int rns_cholesky(const double* S_, double* L_, size_t n, int64_t* pivot, cudaStream_t s, FactorErr* err_out) {
  using namespace ozaki;
  if (n == 0) return HP_OK;
  DevTables* D;
  HP_TRY(device_tables(&D));
  const HostTables& T = host_tables();
  int L = -1;
  for (int q = 1; q <= MAXL; q++)
    if (T.cum_log2[q] >= 2.0 * BETA_CH + 3.0) {
      L = q;
      break;
    }
  const int nc = T.crt[L].nc;
  const dd* S = reinterpret_cast<const dd*>(S_);
  dd* Lout = reinterpret_cast<dd*>(L_);
  const size_t Np = round_up(n, GB_N) + GB_N;  // residue planes of A~ (room for tile overhang)
  const size_t KL = round_up(n, GB_K);   // L~ residue planes: row length (bytes)
  const size_t RL = round_up(n, GB_M) + GB_M;  // and rows
  const size_t nb = CH_NB;
  DevBuf ebuf(n * sizeof(int), s), res((size_t)L * Np * Np, s), lres((size_t)L * RL * KL, s),
      Pb(2 * n * nb * 16, s), L1b(2 * nb * nb * 16, s), RIb(2 * nb * 16, s), err(sizeof(RnsErr), s);
  if (!ebuf.p || !res.p || !lres.p || !Pb.p || !L1b.p || !RIb.p || !err.p) {
    set_error("rns_cholesky: workspace allocation failed");
    return HP_ERR_CUDA;
  }
  RnsErr h0{0, 0, (long long)0x7fffffffffffffffll};
  HP_CUDA_TRY(cudaMemcpyAsync(err.p, &h0, sizeof(h0), cudaMemcpyHostToDevice, s));
  // No zeroing: rns_init writes every residue tile the panels read (rows
  // past n feed only output rows past n), and the L~ planes are read
  // through maps that end at the written columns and rows.
  cudaStream_t s_caller = s, s2 = nullptr;
  HP_TRY(pipeline_streams(&s, &s2));
  PipelineEvents ev(s_caller, s, s2);  // declared after the buffers: joins both streams before they are freed
  if (!ev.ok) {
    set_error("rns_cholesky: event creation failed");
    return HP_ERR_CUDA;
  }
  rns_scale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(S, n, BETA_CH, ebuf.as<int>(), err.as<RnsErr>());
  HP_LAUNCH_CHECK();
  {
    // 4 entries per thread; the moduli counts the factor uses (28-30) unrolled
    dim3 g((unsigned)(Np / 16), (unsigned)(Np / 64));
    auto kern = L == 28 ? rns_init_kernel<4, 28> : L == 29 ? rns_init_kernel<4, 29>
                : L == 30 ? rns_init_kernel<4, 30> : rns_init_kernel<4, 0>;
    kern<<<g, 256, 0, s>>>(S, n, ebuf.as<int>(), L, Np, res.as<uint8_t>());
    HP_LAUNCH_CHECK();
  }
  const size_t blk_smem = 64 * 65 * 16, trsm_smem = CH_NB * (CH_NB + 1) * 16;
  HP_CUDA_TRY(cudaFuncSetAttribute(chol_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)blk_smem));
  HP_CUDA_TRY(cudaFuncSetAttribute(panel_trsm_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem));
  HP_CUDA_TRY(cudaFuncSetAttribute(panel_trsm_kernel<28>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem));
  HP_CUDA_TRY(cudaFuncSetAttribute(panel_trsm_kernel<29>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem));
  int8_t* lres8 = reinterpret_cast<int8_t*>(lres.as<uint8_t>());
  const size_t plane_l = RL * KL;
  const int gemm_ctas = std::max(1, D->num_sms - 8);  // leave SMs for the diagonal path
  auto crt = [&](size_t r0, size_t rows, size_t kb, int jb, dd* out, cudaStream_t st, bool pdl) -> int {
    if (rows == 0) return HP_OK;
#define HP_CRTB(NC)                                                                                               \
  case NC:                                                                                                        \
    HP_CUDA_TRY(launch_k(pdl, crt_block_kernel<NC>, dim3((unsigned)((rows * jb + 255) / 256)), dim3(256), 0, st, \
                         (const uint8_t*)res.as<uint8_t>(), (int64_t)Np, (int64_t)(Np * Np), (int64_t)r0,        \
                         (int64_t)kb, (int64_t)rows, (int64_t)jb, (const CrtTable*)(D->crt + L), out));          \
    break;
#define HP_CRTB_LC(NCV, LCV)                                                                                      \
  if (nc == NCV && L == LCV) {                                                                                    \
    HP_CUDA_TRY(launch_k(pdl, crt_block_kernel<NCV, LCV>, dim3((unsigned)((rows * jb + 255) / 256)), dim3(256), 0, \
                         st, (const uint8_t*)res.as<uint8_t>(), (int64_t)Np, (int64_t)(Np * Np), (int64_t)r0,      \
                         (int64_t)kb, (int64_t)rows, (int64_t)jb, (const CrtTable*)(D->crt + L), out));           \
    return HP_OK;                                                                                                 \
  }
    HP_CRTB_LC(6, 28) HP_CRTB_LC(6, 29) HP_CRTB_LC(6, 30) HP_CRTB_LC(7, 28) HP_CRTB_LC(7, 29) HP_CRTB_LC(7, 30)
#undef HP_CRTB_LC
    switch (nc) {
      HP_CRTB(5) HP_CRTB(6) HP_CRTB(7)
      default:
        set_error("rns_cholesky: unsupported chunk count %d", nc);
        return HP_ERR_UNSUPPORTED;
    }
#undef HP_CRTB
    return HP_OK;
  };
  auto trsm = [&](int par, size_t kb, int jb, size_t r0, size_t m, cudaStream_t st, bool pdl) -> int {
    if (r0 >= m) return HP_OK;
    const unsigned blocks = (unsigned)std::min<size_t>((m - r0 + 7) / 8, (size_t)D->num_sms * 3);
    auto kern = L == 28 ? panel_trsm_kernel<28> : L == 29 ? panel_trsm_kernel<29> : panel_trsm_kernel<0>;
    HP_CUDA_TRY(launch_k(pdl, kern, dim3(blocks), dim3(256), trsm_smem, st,
                         (const dd*)(Pb.as<dd>() + (size_t)par * n * nb + (size_t)jb * jb),
                         (const dd*)(L1b.as<dd>() + (size_t)par * nb * nb), (const dd*)(RIb.as<dd>() + par * nb),
                         (int64_t)r0, (int64_t)m, jb, (int64_t)(kb + jb), (int64_t)kb, (int64_t)n,
                         (const int*)ebuf.as<int>(), Lout, L, lres8, (int64_t)KL, (int64_t)plane_l));
    return HP_OK;
  };
  // Left-looking, with a look-ahead pipeline. Panel q (block column kb)
  // receives all earlier updates, A~[kb.., kb..kb+nb) -= L~[kb.., 0..kb)
  // L~[kb..kb+nb, 0..kb)^T, as residue GEMMs (N = nb) over the stored residue
  // planes of L~. Residues make the update order free: every GEMM subtracts
  // its products modulo m, so the panel's update is split by K into
  //   early: columns [0, kb - nb) (panels q - 2 and before), all rows, on s2,
  //          enqueued one panel ahead so that it runs while panel q - 1 is
  //          being factored;
  //   late:  columns [kb - nb, kb) (panel q - 1, one k-block), on s for the
  //          first 128 rows (the diagonal path) and on s2 for the others.
  // Stream s (greatest priority) carries the diagonal path: late GEMM, CRT
  // of the diagonal block, factor, and the first 128 rows of the panel
  // solve (which the next late GEMM reads); stream s2 carries the rest of
  // the rows' late GEMM, CRT and solve, and the next panel's early GEMM.
  // Two GEMMs touching the same residues are always ordered by a stream or
  // an event. Panel buffers (P, L1, 1/l) alternate by panel parity; the
  // maps of every GEMM end at the columns that hold panels, so the partial
  // 128-byte k-blocks read zeros. The integers are those of the
  // right-looking order; only the schedule differs.
  const size_t npanel = (n + nb - 1) / nb;
  for (size_t kb = 0, p = 0; kb < n; kb += nb, p++) {
    const int jb = (int)std::min(nb, n - kb);
    const size_t R = n - kb, m = R - jb;
    const int par = (int)(p & 1);
    dd* Pp = Pb.as<dd>() + (size_t)par * n * nb;
    const size_t Rd = std::min<size_t>(R, GB_M);  // rows of the diagonal path's GEMM
    if (kb == 0) {
      HP_TRY(crt(0, R, 0, jb, Pp, s, false));
    } else {
      // late update of the diagonal path: panel q - 1's columns (its solve
      // rows kb..kb+128 came from this stream); after the early update of
      // the same rows (event E, recorded on s2 after it)
      if (p >= 2) HP_CUDA_TRY(cudaStreamWaitEvent(s, ev.E, 0));
      const uint8_t* lrow = lres.as<uint8_t>() + kb * KL;
      HP_TRY(rns_panel_update(lrow + (kb - nb), R, lrow + (kb - nb), R, KL, nb, plane_l, L, Rd, GB_K,
                              res.as<uint8_t>(), Np, kb, kb, gemm_ctas, s, true));
      HP_CUDA_TRY(cudaEventRecord(ev.Gd, s));
      HP_TRY(crt(kb, (size_t)jb, kb, jb, Pp, s, true));
      // s2: late update of the other rows (after the previous panel's solve
      // rows on s), then their CRT
      HP_CUDA_TRY(cudaStreamWaitEvent(s2, ev.Td, 0));
      if (R > Rd) {
        const uint8_t* arow = lres.as<uint8_t>() + (kb + Rd) * KL;
        HP_TRY(rns_panel_update(arow + (kb - nb), R - Rd, lrow + (kb - nb), R, KL, nb, plane_l, L, R - Rd, GB_K,
                                res.as<uint8_t>(), Np, kb + Rd, kb, gemm_ctas, s2));
      }
      HP_CUDA_TRY(cudaStreamWaitEvent(s2, ev.Gd, 0));
      HP_TRY(crt(kb + jb, m, kb, jb, Pp + (size_t)jb * jb, s2, false));
      HP_CUDA_TRY(cudaEventRecord(ev.Cr, s2));
    }
    // s2: early update of panel q + 1 (columns [0, kb), every panel up to
    // q - 1, all of whose rows are solved by now in s2's order or behind
    // the event Td it waited for), while panel q is factored
    if (p + 1 < npanel && kb > 0) {
      const size_t kn = kb + nb, Rn = n - kn;
      const uint8_t* nrow = lres.as<uint8_t>() + kn * KL;
      HP_TRY(rns_panel_update(nrow, Rn, nrow, Rn, KL, kb, plane_l, L, Rn, round_up(kb, GB_K), res.as<uint8_t>(),
                              Np, kn, kn, gemm_ctas, s2));
      HP_CUDA_TRY(cudaEventRecord(ev.E, s2));
    }
    HP_CUDA_TRY(launch_k(true, chol_block_kernel, dim3(1), dim3(CI_THREADS), blk_smem, s, (const dd*)Pp, jb,
                         (int64_t)kb, (int64_t)n, (const int*)ebuf.as<int>(), Lout,
                         L1b.as<dd>() + (size_t)par * nb * nb, RIb.as<dd>() + par * nb, err.as<RnsErr>()));
    HP_CUDA_TRY(cudaEventRecord(ev.F, s));
    if (m == 0) break;
    const size_t md = std::min<size_t>(m, GB_M);  // panel-solve rows on the diagonal path
    if (kb > 0) HP_CUDA_TRY(cudaStreamWaitEvent(s, ev.Cr, 0));
    HP_TRY(trsm(par, kb, jb, 0, md, s, true));
    HP_CUDA_TRY(cudaEventRecord(ev.Td, s));
    HP_CUDA_TRY(cudaStreamWaitEvent(s2, ev.F, 0));
    HP_TRY(trsm(par, kb, jb, md, m, s2, false));
  }
  ev.join();  // both pipeline streams finish before the caller's stream goes on
  s = s_caller;
  if (err_out) {  // the caller reads the outcome later, with its own next readback
    HP_CUDA_TRY(cudaMemcpyAsync(err_out, err.p, sizeof(RnsErr), cudaMemcpyDeviceToDevice, s));
    return HP_OK;
  }
  RnsErr h;
  HP_CUDA_TRY(cudaMemcpyAsync(&h, err.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (h.flag) {
    if (pivot) *pivot = h.pivot;
    set_error("Cholesky failed at pivot %lld", (long long)h.pivot);
    return HP_ERR_NOT_SPD;
  }
  return HP_OK;
}

}  // namespace hp

// ===========================================================================
// Allocation-free f128 Ozaki GEMM (hp_f128_gemm_noalloc_dev).
// Some callers cannot let a library allocate device memory in the middle of
// a call: a host that hands all device memory to its own pool at start-up,
// a latency-bound loop where cudaMalloc / cudaFree (which may synchronise
// the whole device) would stall its other streams, or an embedding whose
// device memory belongs to a foreign allocator. For them this entry point
// keeps its entire workspace in one file-scope device array of
// NOALLOC_SCRATCH_BYTES bytes and calls no allocating routine. Every call on
// a device shares that one array, so calls that overlap in time (two host
// threads, or two streams) race on it: the caller must order them. The
// first call on each device does the set-up (symbol addresses, table
// upload, kernel attribute) and blocks the host while it does, so that
// first call should come before any stream capture. Each call returns once
// its stream has run it: it reads the call's status word back, so that a
// bounded wait in the tensor-core kernel that gave up is returned as
// HP_ERR_TIMEOUT by this call rather than lost.
// ===========================================================================
namespace hp {
namespace ozaki {
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)64 << 20;  // 64 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];
static __device__ __align__(16) CrtTable g_noalloc_crt[MAXL + 1];
static __device__ __align__(16) uint32_t g_noalloc_status[4];

struct NoAllocDev {
  bool ready = false;
  unsigned char* scratch = nullptr;
  CrtTable* crt = nullptr;
  uint32_t* status = nullptr;
  int num_sms = 0;
};
static NoAllocDev g_noalloc[64];

// Once per device, with that device current.
static int noalloc_setup(NoAllocDev** out) {
  int d = 0;
  HP_CUDA_TRY(cudaGetDevice(&d));
  if (d < 0 || d >= 64) {
    set_error("device ordinal %d out of range", d);
    return HP_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_dev_mu);
  NoAllocDev& N = g_noalloc[d];
  if (!N.ready) {
    const HostTables& T = host_tables();
    // the modulus table is uploaded by whichever Ozaki path runs first
    if (!g_dev[d].ready) {
      HP_CUDA_TRY(cudaMemcpyToSymbol(c_tab, &T.mt, sizeof(ModTable)));
      HP_CUDA_TRY(cudaMemcpyToSymbol(c_crt_tc, T.crt_tc, sizeof(CrtTcTable) * CRT_CONST_N));
    }
    HP_CUDA_TRY(cudaMemcpyToSymbol(g_noalloc_crt, T.crt.data(), sizeof(CrtTable) * (MAXL + 1)));
    HP_CUDA_TRY(cudaGetSymbolAddress((void**)&N.scratch, g_noalloc_scratch));
    HP_CUDA_TRY(cudaGetSymbolAddress((void**)&N.crt, g_noalloc_crt));
    HP_CUDA_TRY(cudaGetSymbolAddress((void**)&N.status, g_noalloc_status));
    HP_CUDA_TRY(cudaDeviceGetAttribute(&N.num_sms, cudaDevAttrMultiProcessorCount, d));
    HP_CUDA_TRY(cudaFuncSetAttribute(i8_gemm_mod_kernel<GB_N>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
    N.ready = true;
  }
  *out = &N;
  return HP_OK;
}

// Byte offset of the next 256-byte aligned region of `bytes` bytes.
static size_t carve(size_t* off, size_t bytes) {
  const size_t o = *off;
  *off = round_up(o + bytes, 256);
  return o;
}

}  // namespace ozaki

// Same four phases as ozaki_dd_gemm (C = A B, row-major f128), with the
// exponent vectors, residue planes and product residues carved from the
// static scratch instead of allocated.
static int ozaki_dd_gemm_noalloc(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                                 cudaStream_t s) {
  using namespace ozaki;
  NoAllocDev* N;
  HP_TRY(noalloc_setup(&N));
  if (m == 0 || n == 0) return HP_OK;
  if (k == 0) {
    HP_CUDA_TRY(cudaMemsetAsync(c, 0, m * n * 16, s));
    return HP_OK;
  }
  const int beta = BETA_DD;
  const int L = ozaki_moduli_for(k, beta);
  if (L < 0) {
    set_error("ozaki: k = %zu needs more moduli than the table holds", k);
    return HP_ERR_UNSUPPORTED;
  }
  size_t need = SIZE_MAX, Mp = 0, Np = 0, Kp = 0, o_ea = 0, o_eb = 0, o_a = 0, o_b = 0, o_c = 0;
  if (m <= NOALLOC_SCRATCH_BYTES && n <= NOALLOC_SCRATCH_BYTES && k <= NOALLOC_SCRATCH_BYTES) {
    Mp = round_up(m, GB_M);
    Np = round_up(n, GB_N);
    Kp = round_up(k, GB_K);
    size_t off = 0;
    o_ea = carve(&off, Mp * sizeof(int));
    o_eb = carve(&off, Np * sizeof(int));
    o_a = carve(&off, (size_t)L * Mp * Kp);
    o_b = carve(&off, (size_t)L * Np * Kp);
    o_c = carve(&off, (size_t)L * Mp * Np);
    need = off;
  }
  if (need > NOALLOC_SCRATCH_BYTES) {
    set_error("hp_f128_gemm_noalloc_dev: %zu x %zu x %zu needs %s%zu bytes of scratch, the static scratch holds %zu",
              m, n, k, need == SIZE_MAX ? "more than " : "", need == SIZE_MAX ? NOALLOC_SCRATCH_BYTES : need,
              NOALLOC_SCRATCH_BYTES);
    return HP_ERR_INVALID_ARG;
  }
  int* expA = reinterpret_cast<int*>(N->scratch + o_ea);
  int* expB = reinterpret_cast<int*>(N->scratch + o_eb);
  int8_t* ares = reinterpret_cast<int8_t*>(N->scratch + o_a);
  int8_t* bres = reinterpret_cast<int8_t*>(N->scratch + o_b);
  uint8_t* cres = N->scratch + o_c;
  // what must start at zero: the exponent maxima (atomicMax) and the status
  // word; residue and product planes are fully overwritten
  HP_CUDA_TRY(cudaMemsetAsync(expA, 0, Mp * sizeof(int), s));
  HP_CUDA_TRY(cudaMemsetAsync(expB, 0, Np * sizeof(int), s));
  HP_CUDA_TRY(cudaMemsetAsync(N->status, 0, sizeof(uint32_t), s));
  const double2* A2 = reinterpret_cast<const double2*>(a);
  const double2* B2 = reinterpret_cast<const double2*>(b);
  HP_TRY(launch_maxexp(A2, B2, m, n, k, false, expA, expB, s));
  {
    const unsigned tay = (unsigned)(Mp / RT_R);
    dim3 g((unsigned)(Kp / RT_P), tay + (unsigned)(Np / RT_R));
    residue_ab_kernel<true, 8, false><<<g, 256, 0, s>>>(A2, m, expA, ares, (int64_t)(Mp * Kp), tay, B2, n, expB, bres,
                                              (int64_t)(Np * Kp), k, beta, L, (int64_t)Kp);
    HP_LAUNCH_CHECK();
  }
  {
    CUtensorMap mapA, mapB;
    HP_TRY(make_map(&mapA, ares, Kp, Mp, L, GB_M));
    HP_TRY(make_map(&mapB, bres, Kp, Np, L, GB_N));
    const int tiles_m = (int)(Mp / GB_M), tiles_n = (int)(Np / GB_N);
    const int grid = std::min(L * tiles_m * tiles_n, N->num_sms);
    const int nkb = (int)(Kp / GB_K), kb_chunk = MAX_K_CHUNK / GB_K;
    for (int c0 = 0; c0 < nkb; c0 += kb_chunk) {
      i8_gemm_mod_kernel<GB_N><<<grid, 256, GEMM_SMEM, s>>>(mapA, mapB, L, tiles_m, tiles_n, c0, std::min(nkb, c0 + kb_chunk),
                                                       0, c0 > 0 ? 1 : 0, cres, (int64_t)Np, (int64_t)(Mp * Np), 0, 0,
                                                       N->status);
      HP_LAUNCH_CHECK();
    }
  }
  if (L >= CRT_CONST_L0 && L < CRT_CONST_L0 + CRT_CONST_N)
    HP_TRY(launch_crt_tc(cres, Mp, Np, m, n, expA, expB, beta, L, reinterpret_cast<double2*>(c), N->num_sms,
                         N->status, s, false));
  else
    HP_TRY(launch_crt_dd(cres, Mp, Np, m, n, expA, expB, beta, N->crt + L, host_tables().crt[L].nc,
                         reinterpret_cast<double2*>(c), s));
  // The status word lives in the static array as well; it is read back here,
  // before the next call clears it, so a wait that gave up is reported by
  // the call it happened in.
  uint32_t st = 0;
  HP_CUDA_TRY(cudaMemcpyAsync(&st, N->status, sizeof(st), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (st & DEV_STATUS_TIMEOUT) {
    set_error("hp_f128_gemm_noalloc_dev: a bounded device-side wait gave up (status 0x%x)", st);
    return HP_ERR_TIMEOUT;
  }
  return HP_OK;
}

}  // namespace hp

extern "C" int hp_f128_gemm_noalloc_dev(const double* a, const double* b, double* c, size_t m, size_t n, size_t k,
                                        void* stream) {
  using namespace hp;
  size_t t, ba, bb, bc;
  if (mul_overflows(m, k, &t) || mul_overflows(t, 16, &ba) || mul_overflows(k, n, &t) || mul_overflows(t, 16, &bb) ||
      mul_overflows(m, n, &t) || mul_overflows(t, 16, &bc)) {
    set_error("matrix size overflows size_t");
    return HP_ERR_INVALID_ARG;
  }
  if ((ba && !a) || (bb && !b) || (bc && !c)) {
    set_error("null pointer with non-zero size");
    return HP_ERR_INVALID_ARG;
  }
  if (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c) % 16) {
    set_error("device pointers must be 16-byte aligned");
    return HP_ERR_INVALID_ARG;
  }
  return ozaki_dd_gemm_noalloc(a, b, c, m, n, k, (cudaStream_t)stream);
}
