// Dense Cholesky factorisation and solve of the reduced system on sm_100a: the reduced solve that follows
// reduce_schur_dense! when S is small enough to hold dense (the reference hands its dense S to DampedLinearSolve's
// Cholesky, src/schur_linear_systems.jl:312-320). S is read from its upper triangle in its storage type (FP64 or the
// mixed form's FP32), mirrored into an FP64 working matrix owned by the solver, and factored in place as S = L L' by a
// right-looking blocked Cholesky with 32 x 32 tiles: per tile column, the diagonal tile in one CTA's shared memory,
// the tiles below it by a triangular solve, then the trailing lower triangle updated tile by tile. A pivot that is not
// positive (or not finite) stops the factorisation; its column is reported, 1-based. The solve runs the two triangular
// substitutions by 32-column tiles in one CTA.
#include <algorithm>
#include <cmath>
#include <memory>

#include "common.cuh"

namespace bls {

constexpr int DNB = 32;   // tile size

struct DenseSolver {
  bls_ctx* ctx = nullptr;
  int64_t n = 0;
  DevBuf W;        // n x n FP64, column-major; L in its lower triangle after a successful factorisation
  DevBuf status;   // [0]: first failing column (0-based) or -1
  bool factored = false;
};

// W = S mirrored from its upper triangle, in FP64
template <class T>
__global__ void k_dense_load(int64_t n, const T* __restrict__ S, double* __restrict__ W, long long* __restrict__ status) {
  if (blockIdx.x == 0 && threadIdx.x == 0) status[0] = -1;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n * n; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q % n, j = q / n;
    W[q] = (double)(i <= j ? S[i + n * j] : S[j + n * i]);
  }
}

// The diagonal tile [k0, k0 + nb) in one CTA of 32 x 32 threads: unblocked Cholesky in shared memory, lower triangle
// written back. A non-positive or non-finite pivot records its column and leaves W as it is.
__global__ void __launch_bounds__(DNB * DNB) k_potrf_tile(int64_t n, double* __restrict__ W, int64_t k0, int nb,
                                                          long long* __restrict__ status) {
  __shared__ double a[DNB][DNB + 1];
  __shared__ int bad;
  if (status[0] >= 0) return;   // uniform across the CTA
  const int tx = threadIdx.x, ty = threadIdx.y;   // a[ty][tx] = W[k0 + ty, k0 + tx]
  if (tx < nb && ty < nb) a[ty][tx] = W[(k0 + ty) + n * (k0 + tx)];
  if (tx == 0 && ty == 0) bad = 0;
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    const double d = a[j][j];
    if (!(d > 0.0) || !isfinite(d)) {
      if (tx == 0 && ty == 0) {
        bad = 1;
        status[0] = k0 + j;
      }
      return;   // every thread reads the same d: the whole CTA returns here
    }
    const double ljj = sqrt(d);
    __syncthreads();
    if (ty > j && tx == 0) a[ty][j] /= ljj;
    if (ty == j && tx == 0) a[j][j] = ljj;
    __syncthreads();
    if (ty > j && tx > j && tx <= ty && ty < nb) a[ty][tx] -= a[ty][j] * a[tx][j];
    __syncthreads();
  }
  if (tx < nb && ty < nb && tx <= ty) W[(k0 + ty) + n * (k0 + tx)] = a[ty][tx];
}

// The tiles below the diagonal tile: rows [k0 + nb, n) of columns [k0, k0 + nb) solved against L_kk' (X L_kk' = A),
// one warp per 32 rows, a lane per row, columns in order
__global__ void __launch_bounds__(DNB) k_trsm_panel(int64_t n, double* __restrict__ W, int64_t k0, int nb, const long long* __restrict__ status) {
  __shared__ double L[DNB][DNB + 1];
  __shared__ double x[DNB][DNB + 1];
  if (status[0] >= 0) return;
  const int lane = threadIdx.x;
  for (int c = 0; c < nb; ++c)
    if (lane < nb) L[lane][c] = W[(k0 + lane) + n * (k0 + c)];
  const int64_t r = k0 + nb + (int64_t)blockIdx.x * DNB + lane;
  __syncwarp();
  if (r < n) {
    for (int c = 0; c < nb; ++c) {
      double v = W[r + n * (k0 + c)];
      for (int cp = 0; cp < c; ++cp) v -= x[lane][cp] * L[c][cp];
      x[lane][c] = v / L[c][c];
    }
    for (int c = 0; c < nb; ++c) W[r + n * (k0 + c)] = x[lane][c];
  }
}

// The trailing lower triangle: W[i, j] -= sum_c L[i, c] L[j, c] over the panel's columns c, for i >= j >= k0 + nb.
// One CTA of 32 x 32 threads per 32 x 32 output tile of the lower triangle (tiles listed by their index in it).
__global__ void __launch_bounds__(DNB * DNB) k_syrk_tiles(int64_t n, double* __restrict__ W, int64_t k0, int nb, int64_t nt,
                                                          const long long* __restrict__ status) {
  __shared__ double Pi[DNB][DNB + 1], Pj[DNB][DNB + 1];
  if (status[0] >= 0) return;
  // tile (ti, tj), tj <= ti, of the trailing triangle of nt tiles
  const int64_t t = blockIdx.x;
  int64_t ti = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
  while (ti * (ti + 1) / 2 > t) --ti;
  const int64_t tj = t - ti * (ti + 1) / 2;
  const int64_t base = k0 + nb;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t i = base + ti * DNB + ty, j = base + tj * DNB + ty;
  Pi[ty][tx] = (i < n && tx < nb) ? W[i + n * (k0 + tx)] : 0.0;
  Pj[ty][tx] = (j < n && tx < nb) ? W[j + n * (k0 + tx)] : 0.0;
  __syncthreads();
  const int64_t oi = base + ti * DNB + ty, oj = base + tj * DNB + tx;
  if (oi < n && oj < n && oj <= oi) {
    double s = 0.0;
    for (int c = 0; c < nb; ++c) s += Pi[ty][c] * Pj[tx][c];
    W[oi + n * oj] -= s;
  }
  (void)nt;
}

// x = (L L')^-1 g in one CTA, by 32-column tiles: each diagonal tile is solved by one warp (a lane per row, the pivot
// broadcast by shuffle), then every thread updates the rows the tile feeds (forward: the rows below, reading the
// tile's columns of L down a column; backward: the rows above, reading each row's 32 contiguous entries of the tile's
// rows of L). The right-hand side lives in shared memory.
__global__ void __launch_bounds__(1024) k_chol_solve(int64_t n, const double* __restrict__ W, const double* __restrict__ g,
                                                     double* __restrict__ x) {
  extern __shared__ double y[];
  __shared__ double t[DNB][DNB + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int64_t i = tid; i < n; i += blockDim.x) y[i] = g[i];
  __syncthreads();
  // forward: L y = g
  for (int64_t k0 = 0; k0 < n; k0 += DNB) {
    const int nb = (int)(n - k0 < DNB ? n - k0 : DNB);
    for (int q = tid; q < nb * nb; q += blockDim.x) t[q % nb][q / nb] = W[(k0 + q % nb) + n * (k0 + q / nb)];
    __syncthreads();
    if (warp == 0) {
      double yr = lane < nb ? y[k0 + lane] : 0.0;
      for (int c = 0; c < nb; ++c) {
        const double yc = __shfl_sync(0xffffffffu, yr, c) / t[c][c];
        if (lane == c) yr = yc;
        else if (lane > c && lane < nb) yr -= t[lane][c] * yc;
      }
      if (lane < nb) y[k0 + lane] = yr;
    }
    __syncthreads();
    for (int64_t i = k0 + nb + tid; i < n; i += blockDim.x) {
      double s = 0.0;
      for (int c = 0; c < nb; ++c) s += W[i + n * (k0 + c)] * y[k0 + c];
      y[i] -= s;
    }
    __syncthreads();
  }
  // backward: L' x = y
  for (int64_t k0 = ((n - 1) / DNB) * DNB; k0 >= 0; k0 -= DNB) {
    const int nb = (int)(n - k0 < DNB ? n - k0 : DNB);
    for (int q = tid; q < nb * nb; q += blockDim.x) t[q % nb][q / nb] = W[(k0 + q % nb) + n * (k0 + q / nb)];
    __syncthreads();
    if (warp == 0) {
      double yr = lane < nb ? y[k0 + lane] : 0.0;
      for (int c = nb - 1; c >= 0; --c) {
        const double xc = __shfl_sync(0xffffffffu, yr, c) / t[c][c];
        if (lane == c) yr = xc;
        else if (lane < c) yr -= t[c][lane] * xc;
      }
      if (lane < nb) y[k0 + lane] = yr;
    }
    __syncthreads();
    for (int64_t i = tid; i < k0; i += blockDim.x) {
      double s = 0.0;
      for (int c = 0; c < nb; ++c) s += W[(k0 + c) + n * i] * y[k0 + c];
      y[i] -= s;
    }
    __syncthreads();
  }
  for (int64_t i = tid; i < n; i += blockDim.x) x[i] = y[i];
}

template <class T>
static int factor(DenseSolver* D, const T* S, int64_t* failed_column) {
  if (!S) throw Error(BLS_EINVAL, "S is NULL");
  cudaStream_t s = D->ctx->stream;
  const int64_t n = D->n;
  double* W = D->W.as<double>();
  long long* st = D->status.as<long long>();
  k_dense_load<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((n * n + 255) / 256, 148 * 8)), 256, 0, s>>>(n, S, W, st);
  for (int64_t k0 = 0; k0 < n; k0 += DNB) {
    const int nb = (int)std::min<int64_t>(DNB, n - k0);
    k_potrf_tile<<<1, dim3(DNB, DNB), 0, s>>>(n, W, k0, nb, st);
    const int64_t rest = n - k0 - nb;
    if (rest > 0) {
      k_trsm_panel<<<(unsigned)((rest + DNB - 1) / DNB), DNB, 0, s>>>(n, W, k0, nb, st);
      const int64_t nt = (rest + DNB - 1) / DNB;
      k_syrk_tiles<<<(unsigned)(nt * (nt + 1) / 2), dim3(DNB, DNB), 0, s>>>(n, W, k0, nb, nt, st);
    }
  }
  BLS_CUDA(cudaGetLastError());
  long long h = -1;
  BLS_CUDA(cudaMemcpyAsync(&h, st, sizeof(long long), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  D->factored = h < 0;
  if (failed_column) *failed_column = h < 0 ? 0 : h + 1;
  return h < 0 ? BLS_OK : BLS_NOT_PD;
}

}  // namespace bls

using namespace bls;

struct bls_dense_solver : DenseSolver {};

#define DENSE_GUARD(...)                      \
  try {                                       \
    __VA_ARGS__                               \
  } catch (const bls::Error& e) {             \
    bls::set_error(e.what());                 \
    return e.code;                            \
  } catch (const std::bad_alloc&) {           \
    bls::set_error("out of host memory");     \
    return BLS_ENOMEM;                        \
  }

extern "C" {

int bls_dense_solver_create(bls_ctx* ctx, int64_t n, bls_dense_solver** out) {
  DENSE_GUARD({
    if (!ctx || !out) throw Error(BLS_EINVAL, "null argument");
    if (n < 1 || n > 16384) throw Error(BLS_EUNSUPPORTED, "dense reduced systems of 1 to 16384 variables are supported");
    std::unique_ptr<bls_dense_solver> D(new bls_dense_solver());
    D->ctx = ctx;
    D->n = n;
    D->W.alloc(sizeof(double) * (size_t)(n * n));
    D->status.alloc(sizeof(long long));
    *out = D.release();
    return BLS_OK;
  })
}

int bls_dense_solver_destroy(bls_dense_solver* D) {
  delete D;
  return BLS_OK;
}

int bls_dense_cholesky(bls_dense_solver* D, int dtype, const void* S, int64_t* failed_column) {
  DENSE_GUARD({
    if (!D) throw Error(BLS_EINVAL, "solver is NULL");
    if (dtype == BLS_F64) return factor<double>(D, (const double*)S, failed_column);
    if (dtype == BLS_F32) return factor<float>(D, (const float*)S, failed_column);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_dense_cholesky_solve(bls_dense_solver* D, const double* g, double* x) {
  DENSE_GUARD({
    if (!D || !g || !x) throw Error(BLS_EINVAL, "null argument");
    if (!D->factored) throw Error(BLS_EINVAL, "the solver holds no factorisation (bls_dense_cholesky first, and it must succeed)");
    const size_t smem = sizeof(double) * (size_t)D->n;
    // The static tile counts against the 48 KB default too, so opt in whenever the sum passes it.
    const size_t tile = sizeof(double) * DNB * (DNB + 1);
    if (smem + tile > 48 * 1024) BLS_CUDA(cudaFuncSetAttribute(k_chol_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_chol_solve<<<1, 1024, smem, D->ctx->stream>>>(D->n, D->W.as<double>(), g, x);
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

}  // extern "C"
