// The damped closed-form inverse of a point block (src/kernels.jl:14-67), shared by the kernels of libblsgpu.
#pragma once
#include <cuda_runtime.h>

namespace bls {

// --- phase 1: damped inverse of each eliminated block (src/kernels.jl:14-67, src/schur_reduction.jl:127-147) ---
// The closed forms are evaluated with explicitly rounded operations (no FMA contraction), as the reference's Julia
// arithmetic is, so that the pivot tests take the reference's decisions.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ bool inv_sym_closed(int de, const double* H, const double* damp, double* inv) {
  const double tol = 4504.0 * 2.220446049250313e-16;   // singular_tol(Float64) = 4504 * eps(Float64)
  if (de == 1) {
    double h11 = add(H[0], mul(1.0, damp[0]));
    if (!(h11 > 0.0) || !isfinite(h11)) return false;
    inv[0] = __drcp_rn(h11);
    return true;
  }
  if (de == 2) {
    double H11 = add(H[0], damp[0]), H22 = add(H[3], damp[1]), H12 = H[2];
    double det = sub(mul(H11, H22), mul(H12, H12));
    if (!(H11 > 0.0) || !(det > mul(tol, mul(H11, H22))) || !isfinite(det)) return false;
    double id = __drcp_rn(det);
    inv[0] = mul(H22, id); inv[1] = mul(-H12, id); inv[2] = mul(-H12, id); inv[3] = mul(H11, id);
    return true;
  }
  // de == 3, H column-major: H[i + 3j]
  double H11 = add(H[0], damp[0]), H22 = add(H[4], damp[1]), H33 = add(H[8], damp[2]);
  double H12 = H[3], H13 = H[6], H23 = H[7];
  double c11 = sub(mul(H22, H33), mul(H23, H23));
  double c12 = sub(mul(H13, H23), mul(H12, H33));
  double c13 = sub(mul(H12, H23), mul(H13, H22));
  double c22 = sub(mul(H11, H33), mul(H13, H13));
  double c23 = sub(mul(H12, H13), mul(H11, H23));
  double c33 = sub(mul(H11, H22), mul(H12, H12));
  double det = add(add(mul(H11, c11), mul(H12, c12)), mul(H13, c13));
  if (!(H11 > 0.0) || !(c33 > mul(tol, mul(H11, H22))) || !(det > mul(tol, mul(c33, H33))) || !isfinite(det)) return false;
  double id = __drcp_rn(det);
  inv[0] = mul(c11, id); inv[1] = mul(c12, id); inv[2] = mul(c13, id);
  inv[3] = mul(c12, id); inv[4] = mul(c22, id); inv[5] = mul(c23, id);
  inv[6] = mul(c13, id); inv[7] = mul(c23, id); inv[8] = mul(c33, id);
  return true;
}


}  // namespace bls
