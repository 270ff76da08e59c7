// Normalised s-Gaussian pair overlap in f128, shared by the assembly
// kernels (overlap.cu, batched.cu, adjoint.cu):
//   S = (4ab/(a+b)^2)^{3/4} exp(-ab/(a+b) |R-R'|^2)
// evaluated with the reference's f128 operations only (crates/quad/src/
// dd.rs:61-121: sqrt, division and its Taylor exp), so every kernel that
// calls it produces the same bits as the CPU evaluation.
#pragma once
#include "hp_arith.cuh"

namespace hp {

// Exponents below -700 give exactly 0: dd.rs:119 builds 2^k by bit
// manipulation, which is only valid for k >= -1022, and the true value is
// below 1e-304.
__device__ __forceinline__ dd overlap_norm_pair(double a_, const double* ca, double b_, const double* cb) {
  dd a = dd_from(a_), b = dd_from(b_);
  dd sum = dd_add(a, b);
  dd prod = dd_mul(a, b);
  dd ratio = dd_div(dd_mul(dd_from(4.0), prod), dd_mul(sum, sum));
  dd sq = dd_sqrt(ratio);
  dd pref = dd_mul(sq, dd_sqrt(sq));
  dd mu = dd_div(prod, sum);
  dd dx = dd_sub(dd_from(ca[0]), dd_from(cb[0]));
  dd dy = dd_sub(dd_from(ca[1]), dd_from(cb[1]));
  dd dz = dd_sub(dd_from(ca[2]), dd_from(cb[2]));
  dd r2 = dd_add(dd_add(dd_mul(dx, dx), dd_mul(dy, dy)), dd_mul(dz, dz));
  dd arg = dd_neg(dd_mul(mu, r2));
  if (arg.hi < -700.0) return dd{0.0, 0.0};
  return dd_mul(pref, dd_exp(arg));
}

}  // namespace hp
