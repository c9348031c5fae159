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


// Blocks of 4 to 16 (src/kernels.jl:69-85 up to 8, src/schur_reduction.jl:164-225 above; in FP64 the two agree):
// upper Cholesky U of the damped block Hd = H + diag(damp), every pivot squared over its damped diagonal entry above
// singular_tol, inverse U^-1 U^-T (restated from the mathematics: the reference calls StaticArrays and LAPACK here, so
// this path agrees with it to rounding, not bit for bit). H column-major d x d.
__device__ __forceinline__ bool inv_sym_chol(int d, const double* H, const double* damp, double* inv) {
  const double tol = 4504.0 * 2.220446049250313e-16;
  double U[256], Ui[256];
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) U[i + d * j] = i <= j ? H[i + d * j] + (i == j ? damp[i] : 0.0) : 0.0;
  double hd[16];
  for (int i = 0; i < d; ++i) hd[i] = U[i + d * i];
  for (int j = 0; j < d; ++j) {
    double s = U[j + d * j];
    for (int k = 0; k < j; ++k) s -= U[k + d * j] * U[k + d * j];
    if (!(s > 0.0) || !isfinite(s)) return false;
    const double ujj = sqrt(s);
    U[j + d * j] = ujj;
    for (int i = j + 1; i < d; ++i) {
      double t = U[j + d * i];
      for (int k = 0; k < j; ++k) t -= U[k + d * j] * U[k + d * i];
      U[j + d * i] = t / ujj;
    }
  }
  for (int i = 0; i < d; ++i) {
    const double ratio = (U[i + d * i] * U[i + d * i]) / hd[i];
    if (!(isfinite(ratio) && ratio > tol)) return false;
  }
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) Ui[i + d * j] = 0.0;
  for (int j = 0; j < d; ++j) {
    Ui[j + d * j] = 1.0 / U[j + d * j];
    for (int i = j - 1; i >= 0; --i) {
      double s = 0.0;
      for (int k = i + 1; k <= j; ++k) s += U[i + d * k] * Ui[k + d * j];
      Ui[i + d * j] = -s / U[i + d * i];
    }
  }
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) {
      double s = 0.0;
      for (int k = i > j ? i : j; k < d; ++k) s += Ui[i + d * k] * Ui[j + d * k];
      inv[i + d * j] = s;
    }
  return true;
}

}  // namespace bls
