// The conditioning scale of the eliminated systems on sm_100a (src/conditioning.jl:24-87): per variable the power of two
// nearest, on a log scale, to 1 / (1e-12 + sqrt|d_j + lambda sc_j|), computed at the first solve of a fill and
// recomputed, for every variable, when some variable's |d_j + lambda sc_j| s_j^2 has left [2^-16, 2^16] and its own
// scale would change (prepare_scale!). Each scale is formed with IEEE double division, square root, frexp and ldexp, as
// the reference forms it, so the scales are bit-identical to the reference's.
#include <cmath>

#include "common.cuh"

namespace bls {

constexpr double COND_EPS = 1e-12;                       // CONDITIONING_EPS
constexpr double COND_BOUND = 65536.0;                   // RESCALE_BOUND = 2^16
constexpr double COND_SQRT_HALF = 0.70710678118654752440;  // sqrt(0.5), the double nearest

// conditioning_scale (src/conditioning.jl:29-36)
__device__ __forceinline__ double conditioning_scale(double d, double fmin) {
  const double dd = fabs(d);
  if (!isfinite(dd)) return 1.0;
  int e = 0;
  const double f = frexp(1.0 / (COND_EPS + sqrt(dd)), &e);
  const double s = f >= COND_SQRT_HALF ? ldexp(1.0, e) : ldexp(1.0, e - 1);
  return s > fmin ? s : fmin;
}

// the drift test of prepare_scale! (:69-77): set *flag when some variable has drifted out of the bound
__global__ void k_scale_drift(int64_t n, const double* __restrict__ d, double lambda, const double* __restrict__ sc,
                              const double* __restrict__ s, double fmin, int* __restrict__ flag) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double dj = d[j] + lambda * sc[j];
  const double v = fabs(dj) * (s[j] * s[j]);
  if (!(1.0 / COND_BOUND <= v && v <= COND_BOUND) && conditioning_scale(dj, fmin) != s[j]) atomicOr(flag, 1);
}

// s_j for every variable, when the scale is stale or has drifted
__global__ void k_scale_set(int64_t n, const double* __restrict__ d, double lambda, const double* __restrict__ sc, double* __restrict__ s,
                            double fmin, const int* __restrict__ flag, int stale) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n || !(stale || *flag)) return;
  s[j] = conditioning_scale(d[j] + lambda * sc[j], fmin);
}

}  // namespace bls

using namespace bls;

extern "C" int bls_prepare_scale(bls_ctx* ctx, int dtype, int64_t n, const double* d, double lambda, const double* sc, double* s, int stale,
                                 int* recomputed) {
  try {
    if (!ctx || n < 0 || (n > 0 && (!d || !sc || !s))) throw Error(BLS_EINVAL, "null argument");
    if (dtype != BLS_F64 && dtype != BLS_F32) throw Error(BLS_EINVAL, "unknown dtype");
    const double fmin = dtype == BLS_F64 ? 2.2250738585072014e-308 : 1.1754943508222875e-38;   // floatmin(T)
    if (!(lambda != lambda) && !(lambda > 0.0)) lambda = 0.0;   // max(lambda, 0.0), which keeps a NaN
    cudaStream_t st = ctx->stream;
    if (!ctx->flag) BLS_CUDA(cudaMalloc(&ctx->flag, sizeof(int)));
    BLS_CUDA(cudaMemsetAsync(ctx->flag, 0, sizeof(int), st));
    if (n > 0) {
      if (!stale) k_scale_drift<<<grid_for(n, 256), 256, 0, st>>>(n, d, lambda, sc, s, fmin, ctx->flag);
      k_scale_set<<<grid_for(n, 256), 256, 0, st>>>(n, d, lambda, sc, s, fmin, ctx->flag, stale);
    }
    BLS_CUDA(cudaGetLastError());
    if (recomputed) {
      int h = 0;
      BLS_CUDA(cudaMemcpyAsync(&h, ctx->flag, sizeof(int), cudaMemcpyDeviceToHost, st));
      BLS_CUDA(cudaStreamSynchronize(st));
      *recomputed = stale ? 1 : h;
    }
    return BLS_OK;
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  }
}
