// Batched uneven overlap SPD solves and batched Jacobi eigensolves.
//
// batched_spd_kernel: one persistent launch for a whole batch. CTAs (512
// threads) pull system indices from a global counter; the host orders the
// queue largest-n first so the long systems start early. Per system, inside
// one CTA, with its working matrices in a per-CTA global slot (L2-resident):
//   1. assemble S (f128) from the basis with overlap_norm_pair (the same
//      f128 evaluation as hp_overlap_norm_dd, bit-identical);
//   2. right-looking f128 Cholesky (crates/quad/src/linalg.rs:42-96 algebra,
//      pivots by 1/sqrt in f128, updates with the 16-operation dd_fms_fast),
//      pivot <= 0 -> status NOT_SPD;
//   3. x = L^-T L^-1 b, then refinement x += L^-T L^-1 (b - S x) with the
//      residual from error-free products and a 3-level TwoSum cascade
//      (~2^-159), until max|dx| <= tol max|x| (crates/solver/src/lib.rs
//      :75-125 with an f256-grade residual).
// Only __syncthreads inside a CTA and one atomicAdd for the queue: no wait
// can spin.
//
// batched_jacobi_kernel: one CTA per matrix (n <= 128), cyclic Jacobi in
// the parallel (round-robin tournament) ordering: each round applies n/2
// disjoint rotations at once, n-1 rounds per sweep. Rotation formulas, skip
// rule (|a_pq| < 1e-60), stopping rule (off-norm < 1e-30 at the start of a
// sweep) and the row-eigenvector output follow linalg.rs:299-362; the
// rotation order differs (parallel instead of sequential) and the rotations
// are evaluated with the chosen-path f128 helpers (reciprocal, 1/sqrt,
// fused plane rotation), so results agree with the reference to f128
// rounding, not bit-for-bit.
#include <algorithm>
#include <mutex>
#include <vector>

#include "hp_arith.cuh"
#include "hp_overlap.cuh"
#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {

namespace {

constexpr int SPD_PANEL = 8;  // columns per panel of the batched Cholesky

template <int NT>
__device__ double block_max(double v, double* red) {
  v = fmax(v, __shfl_xor_sync(0xffffffffu, v, 16));
  v = fmax(v, __shfl_xor_sync(0xffffffffu, v, 8));
  v = fmax(v, __shfl_xor_sync(0xffffffffu, v, 4));
  v = fmax(v, __shfl_xor_sync(0xffffffffu, v, 2));
  v = fmax(v, __shfl_xor_sync(0xffffffffu, v, 1));
  __syncthreads();
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = v;
  __syncthreads();
  double m = 0.0;
  for (int w = 0; w < NT / 32; w++) m = fmax(m, red[w]);
  __syncthreads();
  return m;
}

// In-CTA triangular solves with L (row-major n x n; the factor below the
// diagonal, its mirror above it, so column j is read along row j) and
// rinv[j] = 1 / l_jj, v in place; v and rinv in shared memory. Each step's
// first entry of L is loaded before the barrier that publishes v_j.
template <int NT>
__device__ void cta_trsv(const dd* L, const dd* rinv, dd* v, int n, bool upper_t, dd* bc) {
  for (int s = 0; s < n; s++) {
    const int j = upper_t ? n - 1 - s : s;
    const int i0 = upper_t ? threadIdx.x : j + 1 + threadIdx.x, i1 = upper_t ? j : n;
    const dd l0 = i0 < i1 ? L[(size_t)j * n + i0] : dd{0.0, 0.0};
    if (threadIdx.x == 0) {
      v[j] = dd_mul(v[j], rinv[j]);
      *bc = v[j];
    }
    __syncthreads();
    const dd vj = *bc;
    if (i0 < i1) v[i0] = dd_fms_fast(v[i0], l0, vj);
    for (int i = i0 + NT; i < i1; i += NT) v[i] = dd_fms_fast(v[i], L[(size_t)j * n + i], vj);
    __syncthreads();
  }
}

struct Casc3 {
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  __device__ __forceinline__ void add(double t) {
    double a, e1, e2;
    two_sum(s1, t, a, e1);
    s1 = a;
    two_sum(s2, e1, a, e2);
    s2 = a;
    s3 = __dadd_rn(s3, e2);
  }
};

template <int NT>
__global__ void __launch_bounds__(NT) batched_spd_kernel(int count, const int* __restrict__ order,
                                                         const int64_t* __restrict__ off,
                                                         const double* __restrict__ centers,
                                                         const double* __restrict__ alpha, const dd* __restrict__ b,
                                                         dd* __restrict__ x_out, int* __restrict__ status,
                                                         int* __restrict__ iters, int* queue, dd* __restrict__ work,
                                                         int64_t slot_elems, double tol, int max_iter) {
  // shared memory per system: the Cholesky panel (rows jb..n-1 x SPD_PANEL
  // columns), then x, r and 1 / l_jj (n entries each)
  extern __shared__ __align__(16) unsigned char sm_raw[];
  dd* P = reinterpret_cast<dd*>(sm_raw);
  __shared__ int sys_sh;
  __shared__ dd bc;
  __shared__ dd head[SPD_PANEL];  // scaled entries of the pivot's column at the panel's rows
  __shared__ double red[NT / 32];
  __shared__ int fail;
  dd* S = work + (size_t)blockIdx.x * 2 * slot_elems;
  dd* L = S + slot_elems;
  while (true) {
    if (threadIdx.x == 0) {
      int q = atomicAdd(queue, 1);
      sys_sh = q < count ? order[q] : -1;
      fail = 0;
    }
    __syncthreads();
    const int sys = sys_sh;
    if (sys < 0) break;
    const int64_t o = off[sys];
    const int n = (int)(off[sys + 1] - o);
    const double* cen = centers + 3 * o;
    const double* al = alpha + o;
    dd* xg = x_out + o;
    dd* x = P + (size_t)n * SPD_PANEL;
    dd* r = x + n;
    dd* rd = r + n;
    // 1. assemble S (lower triangle evaluated, mirrored), copy to L
    for (int p = threadIdx.x; p < n * (n + 1) / 2; p += NT) {
      int i = (int)((sqrtf(8.0f * (float)p + 1.0f) - 1.0f) * 0.5f);
      while (i * (i + 1) / 2 > p) i--;
      while ((i + 1) * (i + 2) / 2 <= p) i++;
      const int j = p - i * (i + 1) / 2;
      const dd v = overlap_norm_pair(al[i], cen + 3 * i, al[j], cen + 3 * j);
      S[(size_t)i * n + j] = v;
      S[(size_t)j * n + i] = v;
      L[(size_t)i * n + j] = v;
    }
    __syncthreads();
    // 2. right-looking Cholesky in panels of SPD_PANEL columns: the panel
    //    (its rows jb..n-1) is factored in shared memory, then the trailing
    //    matrix takes the panel's columns in one pass per entry. Every entry
    //    receives its column updates one at a time in column order with the
    //    same operands as the column-by-column form, so the factor is the same.
    for (int jb = 0; jb < n && !fail; jb += SPD_PANEL) {
      const int kw = min(SPD_PANEL, n - jb), rows = n - jb;
      for (int q = threadIdx.x; q < rows * kw; q += NT) {
        const int r = q / kw, c = q % kw;
        if (r >= c) P[r * SPD_PANEL + c] = L[(size_t)(jb + r) * n + jb + c];
      }
      __syncthreads();
      for (int c = 0; c < kw; c++) {
        if (threadIdx.x == 0) {
          const dd d = P[c * SPD_PANEL + c];
          if (!(d.hi > 0.0)) {
            fail = 1;
          } else {
            const dd rs = dd_rsqrt_fast(d);
            P[c * SPD_PANEL + c] = dd_mul(d, rs);
            rd[jb + c] = rs;
            bc = rs;
            for (int c2 = c + 1; c2 < kw; c2++) head[c2] = dd_mul(P[c2 * SPD_PANEL + c], rs);  // l_{c2, c}
          }
        }
        __syncthreads();
        if (fail) break;
        const dd rs = bc;
        for (int r = c + 1 + threadIdx.x; r < rows; r += NT) {
          const dd lrc = dd_mul(P[r * SPD_PANEL + c], rs);
          P[r * SPD_PANEL + c] = lrc;
          for (int c2 = c + 1; c2 < kw && c2 <= r; c2++)
            P[r * SPD_PANEL + c2] = dd_fms_fast(P[r * SPD_PANEL + c2], lrc, head[c2]);
        }
        __syncthreads();
      }
      if (fail) break;
      for (int q = threadIdx.x; q < rows * kw; q += NT) {  // the factored panel back to L, and its mirror
        const int r = q / kw, c = q % kw;
        if (r >= c) L[(size_t)(jb + r) * n + jb + c] = P[r * SPD_PANEL + c];
        if (r > c) L[(size_t)(jb + c) * n + jb + r] = P[r * SPD_PANEL + c];
      }
      {  // trailing update: one warp per row, lanes along k <= i
        const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
        for (int i = jb + kw + warp; i < n; i += NT / 32) {
          const dd* pi = P + (i - jb) * SPD_PANEL;
          for (int k = jb + kw + lane; k <= i; k += 32) {
            const dd* pk = P + (k - jb) * SPD_PANEL;
            dd a = L[(size_t)i * n + k];
            for (int c = 0; c < kw; c++) a = dd_fms_fast(a, pi[c], pk[c]);
            L[(size_t)i * n + k] = a;
          }
        }
      }
      __syncthreads();
    }
    if (fail) {
      if (threadIdx.x == 0) {
        status[sys] = HP_ERR_NOT_SPD;
        iters[sys] = 0;
      }
      __syncthreads();
      continue;
    }
    // 3. solve and refine
    for (int i = threadIdx.x; i < n; i += NT) x[i] = b[o + i];
    __syncthreads();
    cta_trsv<NT>(L, rd, x, n, false, &bc);
    cta_trsv<NT>(L, rd, x, n, true, &bc);
    int it = 0, conv = 0;
    for (it = 1; it <= max_iter; it++) {
      const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
      for (int row = warp; row < n; row += NT / 32) {
        Casc3 c;
        if (lane == 0) {
          c.add(-b[o + row].hi);
          c.add(-b[o + row].lo);
        }
        for (int j = lane; j < n; j += 32) {
          const dd sv = S[(size_t)row * n + j], xv = x[j];
          double pp, e;
          two_prod(sv.hi, xv.hi, pp, e);
          c.add(pp);
          c.add(e);
          two_prod(sv.hi, xv.lo, pp, e);
          c.add(pp);
          c.add(e);
          two_prod(sv.lo, xv.hi, pp, e);
          c.add(pp);
          c.add(e);
          c.add(__dmul_rn(sv.lo, xv.lo));
        }
        for (int w = 16; w; w >>= 1) {
          const double t1 = __shfl_down_sync(0xffffffffu, c.s1, w);
          const double t2 = __shfl_down_sync(0xffffffffu, c.s2, w);
          const double t3 = __shfl_down_sync(0xffffffffu, c.s3, w);
          if (lane < w) {
            c.add(t1);
            c.add(t2);
            c.add(t3);
          }
        }
        if (lane == 0) {
          double h, l;
          two_sum(c.s1, c.s2, h, l);
          r[row] = dd_neg(dd_renorm(h, __dadd_rn(l, c.s3)));
        }
      }
      __syncthreads();
      cta_trsv<NT>(L, rd, r, n, false, &bc);
      cta_trsv<NT>(L, rd, r, n, true, &bc);
      double md = 0.0, mx = 0.0;
      for (int i = threadIdx.x; i < n; i += NT) {
        x[i] = dd_add(x[i], r[i]);
        md = fmax(md, fabs(r[i].hi));
        mx = fmax(mx, fabs(x[i].hi));
      }
      md = block_max<NT>(md, red);
      mx = block_max<NT>(mx, red);
      if (md <= tol * mx) {
        conv = 1;
        break;
      }
    }
    for (int i = threadIdx.x; i < n; i += NT) xg[i] = x[i];
    if (threadIdx.x == 0) {
      status[sys] = conv ? HP_OK : HP_ERR_NO_CONVERGE;
      iters[sys] = conv ? it : max_iter;
    }
    __syncthreads();
  }
}

// Round-robin tournament over nn (even) players: in round r, slot k pairs
// with slot nn-1-k; slot 0 is fixed and the others rotate.
__device__ __forceinline__ int rr_player(int slot, int round, int nn) {
  if (slot == 0) return 0;
  return 1 + (slot - 1 + round) % (nn - 1);
}

// Jacobi on A (row-major n x n f128, symmetric: its lower triangle is read)
// with the working matrix in shared memory as a packed lower triangle
// (n (n + 1) / 2 entries, 132 KB at n = 128) and V transposed in the per-CTA
// slot of global memory (Vt[j][r] = V[r][j], so a column rotation of V is a
// coalesced row update). A round has two barriers: the n/2 rotations
// (linalg.rs:326-336), then every 2 x 2 block of A, rows of pair k1 by
// columns of pair k2 (k1 <= k2), updated by one thread -- the column
// rotation of pair k2 and then the row rotation of pair k1, the order of
// A J followed by J^T (A J) -- with the diagonal blocks set by the
// reference's formulas (linalg.rs:337-340), and V's columns rotated
// (linalg.rs:342-357). The rotations of off-diagonal entries and of V use
// the fused dd_rot_fast (f128 accuracy, not the reference's operation order).
__device__ __forceinline__ int packed_index(int i, int j) {  // lower triangle, row-major
  return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}
// CTA b takes matrix order[b] (b itself without an order) and the V slot b;
// JT threads per CTA.
template <int JT>
__global__ void __launch_bounds__(JT) batched_jacobi_kernel(const int64_t* __restrict__ n_off,
                                                            const int64_t* __restrict__ mat_off,
                                                            const dd* __restrict__ Ain, dd* __restrict__ evals,
                                                            dd* __restrict__ evecs, int* __restrict__ sweeps_out,
                                                            int* __restrict__ status, dd* __restrict__ work,
                                                            int64_t slot_elems, int max_sweeps,
                                                            const int* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  dd* Ap = reinterpret_cast<dd*>(sm_raw);  // packed lower triangle of A
  __shared__ dd cs[64][2];
  __shared__ dd old[64][3];  // a_pp, a_qq, a_pq before the round
  __shared__ dd tt[64];
  __shared__ int prs[64][3];  // p, q, rotated?
  __shared__ dd red[JT / 32];
  __shared__ int stop;
  // a launch that follows this one on the stream works on other matrices:
  // let it start on SMs this one leaves free
  asm volatile("griddepcontrol.launch_dependents;");
  const int sys = order ? order[blockIdx.x] : (int)blockIdx.x;
  const int n = (int)(n_off[sys + 1] - n_off[sys]);
  const dd* Asrc = Ain + mat_off[sys];
  dd* Vt = work + (size_t)blockIdx.x * slot_elems;
  for (int p = threadIdx.x; p < n * n; p += JT) {
    const int i = p / n, j = p % n;
    if (i >= j) Ap[packed_index(i, j)] = Asrc[p];
    Vt[p] = dd_from(i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  const int nn = n + (n & 1), half = nn / 2;
  const int nblocks = half * (half + 1) / 2;
  int sweep = 0, converged = 0;
  for (sweep = 0; sweep < max_sweeps; sweep++) {
    // off-diagonal norm (linalg.rs:307-315): the entries above the diagonal
    dd acc = dd{0.0, 0.0};
    for (int p = threadIdx.x; p < n * n; p += JT)
      if (p % n > p / n) {
        const dd v = Ap[packed_index(p / n, p % n)];
        acc = dd_add(acc, dd_mul(v, v));
      }
    for (int w = 16; w; w >>= 1) {
      dd t;
      t.hi = __shfl_xor_sync(0xffffffffu, acc.hi, w);
      t.lo = __shfl_xor_sync(0xffffffffu, acc.lo, w);
      acc = dd_add(acc, t);
    }
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      dd tot = dd{0.0, 0.0};
      for (int w = 0; w < JT / 32; w++) tot = dd_add(tot, red[w]);
      stop = dd_lt(dd_sqrt(tot), dd_from(1e-30)) ? 1 : 0;
    }
    __syncthreads();
    if (stop) {
      converged = 1;
      break;
    }
    for (int round = 0; round < nn - 1; round++) {
      if (threadIdx.x < half) {
        const int k = threadIdx.x;
        int p = rr_player(k, round, nn), q = rr_player(nn - 1 - k, round, nn);
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        dd c = dd_from(1.0), sr = dd_from(0.0), t = dd_from(0.0);
        int rot = 0;
        if (q < n) {
          const dd apq = Ap[packed_index(q, p)];
          if (!dd_lt(dd_abs(apq), dd_from(1e-60))) {  // linalg.rs:326-335
            // the reference's formulas with the chosen-path reciprocal and
            // 1/sqrt (f128 accuracy; the round's pivot chain is shorter)
            const dd app = Ap[packed_index(p, p)], aqq = Ap[packed_index(q, q)];
            const dd tau = dd_mul(dd_sub(aqq, app), dd_recip_fast(dd_mul(dd_from(2.0), apq)));
            const dd y = dd_add(dd_from(1.0), dd_mul(tau, tau));
            const dd tden = dd_add(dd_abs(tau), dd_mul(y, dd_rsqrt_fast(y)));  // |tau| + sqrt(1 + tau^2)
            t = dd_recip_fast(tden);
            if (tau.hi < 0.0) t = dd_neg(t);
            c = dd_rsqrt_fast(dd_add(dd_from(1.0), dd_mul(t, t)));
            sr = dd_mul(t, c);
            old[k][0] = app;
            old[k][1] = aqq;
            old[k][2] = apq;
            rot = 1;
          }
        }
        prs[k][0] = p;
        prs[k][1] = q;
        prs[k][2] = rot;
        cs[k][0] = c;
        cs[k][1] = sr;
        tt[k] = t;
      }
      __syncthreads();
      // 2 x 2 blocks of A: rows of pair k1, columns of pair k2
      for (int b = threadIdx.x; b < nblocks; b += JT) {
        int k2 = (int)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
        while (k2 * (k2 + 1) / 2 > b) k2--;
        while ((k2 + 1) * (k2 + 2) / 2 <= b) k2++;
        const int k1 = b - k2 * (k2 + 1) / 2;
        const int r1 = prs[k1][2], r2 = prs[k2][2];
        if (k1 == k2) {
          if (r1) {  // linalg.rs:337-340
            const int p = prs[k1][0], q = prs[k1][1];
            Ap[packed_index(p, p)] = dd_sub(old[k1][0], dd_mul(tt[k1], old[k1][2]));
            Ap[packed_index(q, q)] = dd_add(old[k1][1], dd_mul(tt[k1], old[k1][2]));
            Ap[packed_index(q, p)] = dd{0.0, 0.0};
          }
          continue;
        }
        if (!r1 && !r2) continue;
        const int rows[2] = {prs[k1][0], prs[k1][1]}, cols[2] = {prs[k2][0], prs[k2][1]};
        dd x[2][2];
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
          for (int v = 0; v < 2; v++)
            x[u][v] = rows[u] < n && cols[v] < n ? Ap[packed_index(rows[u], cols[v])] : dd{0.0, 0.0};
        if (r2) {  // A J: columns p2, q2
          const dd c = cs[k2][0], sr = cs[k2][1];
#pragma unroll
          for (int u = 0; u < 2; u++) dd_rot_fast(c, sr, x[u][0], x[u][1], x[u][0], x[u][1]);
        }
        if (r1) {  // J^T (A J): rows p1, q1
          const dd c = cs[k1][0], sr = cs[k1][1];
#pragma unroll
          for (int v = 0; v < 2; v++) dd_rot_fast(c, sr, x[0][v], x[1][v], x[0][v], x[1][v]);
        }
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
          for (int v = 0; v < 2; v++)
            if (rows[u] < n && cols[v] < n) Ap[packed_index(rows[u], cols[v])] = x[u][v];
      }
      // columns p, q of V (rows p, q of Vt)
      for (int e = threadIdx.x; e < half * n; e += JT) {
        const int k = e / n, row = e % n;
        if (!prs[k][2]) continue;
        const int p = prs[k][0], q = prs[k][1];
        const dd c = cs[k][0], sr = cs[k][1];
        dd vp, vq;
        dd_rot_fast(c, sr, Vt[(size_t)p * n + row], Vt[(size_t)q * n + row], vp, vq);
        Vt[(size_t)p * n + row] = vp;
        Vt[(size_t)q * n + row] = vq;
      }
      __syncthreads();
    }
  }
  dd* ev = evals + n_off[sys];
  dd* vo = evecs + mat_off[sys];
  for (int i = threadIdx.x; i < n; i += JT) ev[i] = Ap[packed_index(i, i)];
  for (int p = threadIdx.x; p < n * n; p += JT) vo[p] = Vt[p];  // rows = eigenvectors
  if (threadIdx.x == 0) {
    sweeps_out[sys] = sweep;
    status[sys] = converged ? HP_OK : HP_ERR_NO_CONVERGE;
  }
}

// Packed overlap matrices for a batch: S_s at S + mat_off[s] (n_s x n_s).
__global__ void batched_assemble_kernel(const int64_t* __restrict__ off, const double* __restrict__ centers,
                                        const double* __restrict__ alpha, const int64_t* __restrict__ mat_off,
                                        dd* __restrict__ S) {
  const int sys = blockIdx.x;
  const int64_t o = off[sys];
  const int n = (int)(off[sys + 1] - o);
  dd* out = S + mat_off[sys];
  for (int p = threadIdx.x; p < n * n; p += blockDim.x) {
    const int i = p / n, j = p % n;
    out[p] = overlap_norm_pair(alpha[o + i], centers + 3 * (o + i), alpha[o + j], centers + 3 * (o + j));
  }
}

}  // namespace

// Launch configurations of the persistent solver: threads per CTA and CTAs
// per SM (grid = SMs x ctas_per_sm). Every candidate computes the same bits
// (each entry's operation sequence is independent of the CTA size and
// count: warp-per-row updates and residual cascades, in-CTA solves with the
// same j order, order-free max reductions), so the choice is free.
// Dynamic shared memory of the persistent kernel: the Cholesky panel of the
// largest system (its rows x SPD_PANEL columns) and its x, r and 1 / l_jj.
size_t batched_spd_smem(int nmax) { return (size_t)std::max(nmax, 1) * (SPD_PANEL + 3) * 16; }
constexpr size_t SPD_SMEM_MAX = 200 * 1024;  // n <= 1163
// Raises the kernels' dynamic shared-memory limit when a batch needs more
// than any earlier one on this device (never inside a stream capture: the
// graph path calls this before it captures).
int batched_spd_prepare(int nmax) {
  static std::mutex mu;
  static size_t set_for[64] = {};
  const size_t smem = batched_spd_smem(nmax);
  if (smem > SPD_SMEM_MAX) {
    set_error("batched: systems up to n = %zu supported (got %d)", SPD_SMEM_MAX / ((SPD_PANEL + 3) * 16), nmax);
    return HP_ERR_UNSUPPORTED;
  }
  int dev = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 64 && set_for[dev] >= smem) return HP_OK;
  HP_CUDA_TRY(cudaFuncSetAttribute(batched_spd_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  HP_CUDA_TRY(cudaFuncSetAttribute(batched_spd_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  HP_CUDA_TRY(cudaFuncSetAttribute(batched_spd_kernel<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (dev < 64) set_for[dev] = smem;
  return HP_OK;
}

std::vector<BatchedConfig> batched_spd_candidates(int nmax) {
  std::vector<BatchedConfig> out;
  if (batched_spd_prepare(nmax) != HP_OK) return out;
  const size_t smem = batched_spd_smem(nmax);
  const int threads[3] = {256, 512, 1024};
  for (int t : threads) {
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    if (t == 256) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batched_spd_kernel<256>, 256, smem);
    if (t == 512) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batched_spd_kernel<512>, 512, smem);
    if (t == 1024) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batched_spd_kernel<1024>, 1024, smem);
    if (e != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    for (int c = 1; c <= std::min(nb, 4); c++) out.push_back(BatchedConfig{t, c});
  }
  return out;
}
int batched_spd_grid(const BatchedConfig& cfg) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms * std::max(1, cfg.ctas_per_sm);
}
size_t batched_spd_work_bytes(int grid, int nmax) {
  const int64_t slot = (int64_t)nmax * nmax + 2 * (int64_t)nmax;  // S, then L + r
  return (size_t)grid * 2 * slot * 16;
}

// Queue reset + persistent launch on caller-provided workspace (no
// allocation: safe inside stream capture).
int batched_spd_launch(int count, const int* order, const int64_t* off, const double* centers, const double* alpha,
                       const double* b, double* x, int* status, int* iters, int nmax, double tol, int max_iter,
                       void* work, int* queue, const BatchedConfig& cfg, cudaStream_t s) {
  const int64_t slot = (int64_t)nmax * nmax + 2 * (int64_t)nmax;
  const int grid = batched_spd_grid(cfg);
  HP_TRY(batched_spd_prepare(nmax));
  const size_t smem = batched_spd_smem(nmax);
  HP_CUDA_TRY(cudaMemsetAsync(queue, 0, sizeof(int), s));
#define HP_BATCHED_LAUNCH(NT)                                                                                      \
  batched_spd_kernel<NT><<<grid, NT, smem, s>>>(count, order, off, centers, alpha, reinterpret_cast<const dd*>(b), \
                                                reinterpret_cast<dd*>(x), status, iters, queue,                    \
                                                reinterpret_cast<dd*>(work), slot, tol, max_iter)
  switch (cfg.threads) {
    case 256: HP_BATCHED_LAUNCH(256); break;
    case 512: HP_BATCHED_LAUNCH(512); break;
    case 1024: HP_BATCHED_LAUNCH(1024); break;
    default:
      set_error("batched: unsupported CTA size %d", cfg.threads);
      return HP_ERR_INVALID_ARG;
  }
#undef HP_BATCHED_LAUNCH
  HP_LAUNCH_CHECK();
  return HP_OK;
}

int batched_spd(int count, const int* order, const int64_t* off, const double* centers, const double* alpha,
                const double* b, double* x, int* status, int* iters, int nmax, double tol, int max_iter,
                cudaStream_t s, const BatchedConfig& cfg) {
  const int grid = batched_spd_grid(cfg);
  DevBuf work(batched_spd_work_bytes(grid, nmax), s), queue(sizeof(int), s);
  if (!work.p || !queue.p) {
    set_error("batched: workspace allocation failed");
    return HP_ERR_CUDA;
  }
  return batched_spd_launch(count, order, off, centers, alpha, b, x, status, iters, nmax, tol, max_iter, work.p,
                            queue.as<int>(), cfg, s);
}

int batched_jacobi(int count, const int64_t* n_off, const int64_t* mat_off, const double* A, double* evals,
                   double* evecs, int* sweeps, int* status, int nmax, int max_sweeps, cudaStream_t s,
                   const int* order, int count_big, int nmax_small) {
  if (count == 0) return HP_OK;
  if (nmax > 128) {
    set_error("batched jacobi: n <= 128 supported (got %d)", nmax);
    return HP_ERR_UNSUPPORTED;
  }
  if (!order) count_big = count;
  const int64_t slot = (int64_t)nmax * nmax;  // V^T of each matrix
  DevBuf work((size_t)count * slot * 16, s);
  if (!work.p) return HP_ERR_CUDA;
  // the packed lower triangle of each launch's largest matrix
  auto smem_for = [](int m) { return m * (m + 1) / 2 * 16; };
  // the large matrices (one CTA per SM by shared memory) with 1024 threads,
  // the small ones (two CTAs per SM) with 512
  HP_CUDA_TRY(cudaFuncSetAttribute(batched_jacobi_kernel<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   smem_for(nmax)));
  HP_CUDA_TRY(cudaFuncSetAttribute(batched_jacobi_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   smem_for(nmax)));
  auto launch = [&](int first, int cnt, int m, bool pdl) -> cudaError_t {
    const bool big = m > JACOBI_SMALL_N;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cnt);
    cfg.blockDim = dim3(big ? 1024 : 512);
    cfg.dynamicSmemBytes = smem_for(m);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? at : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, big ? batched_jacobi_kernel<1024> : batched_jacobi_kernel<512>, n_off, mat_off,
                              reinterpret_cast<const dd*>(A), reinterpret_cast<dd*>(evals), reinterpret_cast<dd*>(evecs),
                              sweeps, status, work.as<dd>() + (size_t)first * slot, slot, max_sweeps,
                              order ? order + first : order);
  };
  // the large matrices (one CTA per SM by shared memory), then the small
  // ones, which start on the SMs the large ones' last wave leaves free
  if (count_big > 0) HP_CUDA_TRY(launch(0, count_big, nmax, false));
  if (count_big < count) HP_CUDA_TRY(launch(count_big, count - count_big, nmax_small, count_big > 0));
  return HP_OK;
}

int batched_assemble(int count, const int64_t* off, const double* centers, const double* alpha,
                     const int64_t* mat_off, double* S, cudaStream_t s) {
  if (count == 0) return HP_OK;
  batched_assemble_kernel<<<count, 256, 0, s>>>(off, centers, alpha, mat_off, reinterpret_cast<dd*>(S));
  HP_LAUNCH_CHECK();
  return HP_OK;
}

}  // namespace hp
