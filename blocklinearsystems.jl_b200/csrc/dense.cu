// Dense Cholesky factorisation and solve of the reduced system on sm_100a: the reduced solve that follows
// reduce_schur_dense! when S is small enough to hold dense (the reference hands its dense S to DampedLinearSolve's
// Cholesky, src/schur_linear_systems.jl:312-320). S is read from its upper triangle in its storage type (FP64 or the
// mixed form's FP32), mirrored into an FP64 working matrix owned by the solver, and factored in place as S = L L' by a
// right-looking blocked Cholesky with 64-column panels: per panel, one launch factors the diagonal tile (in every
// CTA's shared memory) and solves the rows below it, then the trailing lower triangle is updated in 64 x 64 tiles. A
// pivot that is not positive (or not finite) stops the factorisation; its column is reported, 1-based. The solve runs
// the two triangular substitutions as one launch per 64-row tile: all CTAs apply the last solved tile to the rows it
// feeds, and CTA 0, whose rows are the next diagonal tile, then solves that tile.
#include <algorithm>
#include <cmath>
#include <memory>

#include "common.cuh"

namespace bls {

constexpr int NB = 64;   // panel width and tile size
constexpr int kFusedPanelTiles = 32;   // panels with at most this many 64-row tiles below run as one launch

struct DenseSolver {
  bls_ctx* ctx = nullptr;
  int64_t n = 0;
  DevBuf W;        // n x n FP64, column-major; L in its lower triangle after a successful factorisation
  DevBuf dinv;     // n FP64: 1 / L[j, j], written by the factorisation
  DevBuf status;   // [0]: first failing column (0-based) or -1
  bool factored = false;
  // The next panel's diagonal tile and triangular solve run on a high-priority stream while the rest of the trailing
  // update runs on the caller's stream (created at the first factorisation).
  cudaStream_t panel_stream = nullptr;
  cudaEvent_t ev_join = nullptr, ev_panel = nullptr;
  int panel_priority = 0;
  // Everything after the load of S (the launches depend on n only) as one CUDA graph, captured at the first
  // factorisation; the panel kernels carry the high priority as a launch attribute, so the graph keeps it.
  cudaGraphExec_t factor_graph = nullptr;
  // The solve's launches (two per 64-row tile) as one CUDA graph on the solver's own right-hand side y, captured at
  // the first solve: g is copied into y, the graph replayed, y copied out to x.
  DevBuf y;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t solve_graph = nullptr;
  ~DenseSolver() {
    if (solve_graph) cudaGraphExecDestroy(solve_graph);
    if (factor_graph) cudaGraphExecDestroy(factor_graph);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_panel) cudaEventDestroy(ev_panel);
    if (panel_stream) cudaStreamDestroy(panel_stream);
  }
};

// W = S mirrored from its upper triangle, in FP64, plus lambda s_r[j] on the diagonal when s_r is given
template <class T>
__global__ void k_dense_load(int64_t n, const T* __restrict__ S, double* __restrict__ W, double lambda, const double* __restrict__ s_r,
                             long long* __restrict__ status) {
  if (blockIdx.x == 0 && threadIdx.x == 0) status[0] = -1;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n * n; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q % n, j = q / n;
    double v = (double)(i <= j ? S[i + n * j] : S[j + n * i]);
    if (s_r && i == j) v += lambda * s_r[j];
    W[q] = v;
  }
}

// The lower triangle of the diagonal tile [d0, d0 + dnb) of L into t by 256 threads, all 16 loads of a thread in flight
// (zeros elsewhere)
__device__ __forceinline__ void load_tile(double (*t)[NB + 1], const double* __restrict__ W, int64_t n, int64_t d0, int dnb,
                                          int tid) {
  double v[NB * NB / 256];
#pragma unroll
  for (int k = 0; k < NB * NB / 256; ++k) {
    const int e = tid + 256 * k, rr = e & 63, cc = e >> 6;
    v[k] = (rr < dnb && cc <= rr) ? W[(d0 + rr) + n * (d0 + cc)] : 0.0;
  }
#pragma unroll
  for (int k = 0; k < NB * NB / 256; ++k) {
    const int e = tid + 256 * k;
    t[e & 63][e >> 6] = v[k];
  }
}

// An asynchronous 8-byte global -> shared copy (cp.async); `bytes` 0 writes a zero and reads nothing.
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The diagonal tile T (lower triangle of its first nb rows and columns, in shared memory) factored in place by
// 256 threads, by 16-column sub-panels: warp 0 factors a sub-panel's rows (lane i holds rows c0 + i and c0 + 32 + i
// of its 16 columns in registers) with no barrier: per column the pivot comes from its lane by shuffle,
// L[j, j] = pivot * rsqrt(pivot), and each later column's entry of L is shuffled from its lane to update the rows
// below; then all threads subtract the sub-panel's rank-16 product from the rest of the tile. 1 / L[j, j] goes to dv.
// Returns (to every thread) the first column whose pivot is not positive or not finite, or -1.
__device__ int factor_tile(double (*T)[NB + 1], double* dv, int nb, int* failed) {
  const int tid = threadIdx.x, lane = tid & 31;
  for (int c0 = 0; c0 < nb; c0 += 16) {
    const int w = nb - c0 < 16 ? nb - c0 : 16;
    if (tid < 32) {
      const int r0 = c0 + lane, r1 = c0 + 32 + lane;
      double a0[16], a1[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        a0[k] = r0 < NB ? T[r0][c0 + k] : 0.0;
        a1[k] = r1 < NB ? T[r1][c0 + k] : 0.0;
      }
      int bad = -1;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        if (j < w && bad < 0) {   // uniform (no break, so the loop unrolls and a0, a1 stay in registers)
          const double d = __shfl_sync(0xffffffffu, a0[j], j);
          if (!(d > 0.0) || !isfinite(d)) {   // uniform
            bad = c0 + j;
          } else {
            const double inv = rsqrt(d);
            const double l0 = (lane == j ? d : a0[j]) * inv, l1 = a1[j] * inv;
            if (lane >= j) a0[j] = l0;
            a1[j] = l1;
            if (lane == j) dv[c0 + j] = inv;
#pragma unroll
            for (int k = j + 1; k < 16; ++k) {
              const double lk = __shfl_sync(0xffffffffu, l0, k);
              if (lane >= k) a0[k] -= l0 * lk;
              a1[k] -= l1 * lk;
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (r0 < NB && k <= lane) T[r0][c0 + k] = a0[k];
        if (r1 < NB) T[r1][c0 + k] = a1[k];
      }
      if (lane == 0) *failed = bad;
    }
    __syncthreads();
    if (*failed >= 0) return *failed;   // uniform
    // the rest of the tile's lower triangle: T[i, k] -= sum over the sub-panel's columns of L[i, c] L[k, c]
    const int base = c0 + 16, m = nb > base ? nb - base : 0;
    for (int e = tid; e < m * m; e += 256) {
      const int i = base + e / m, k = base + e % m;
      if (k > i) continue;
      double s0 = 0.0, s1 = 0.0;
#pragma unroll
      for (int c = 0; c < 16; c += 2) {
        s0 = fma(T[i][c0 + c], T[k][c0 + c], s0);
        s1 = fma(T[i][c0 + c + 1], T[k][c0 + c + 1], s1);
      }
      T[i][k] -= s0 + s1;
    }
    __syncthreads();
  }
  return -1;
}

// One row of the panel below the tile solved against L_kk' (x L_kk' = a): x holds the row's 64 entries; L[c2, c] is
// read from the factored tile as a broadcast.
__device__ __forceinline__ void solve_row(double (&x)[NB], const double (*T)[NB + 1], const double* dv) {
#pragma unroll
  for (int c = 0; c < NB; ++c) {
    x[c] *= dv[c];
#pragma unroll
    for (int c2 = c + 1; c2 < NB; ++c2) x[c2] -= x[c] * T[c2][c];
  }
}

// The diagonal tile [k0, k0 + nb) alone, in one CTA (followed by k_trsm_panel when many rows lie below it). A
// non-positive or non-finite pivot records its column and W is not written. 1 / L[j, j] goes to dinv.
__global__ void __launch_bounds__(256, 1) k_potrf_tile(int64_t n, double* __restrict__ W, double* __restrict__ dinv, int64_t k0,
                                                       int nb, long long* __restrict__ status) {
  __shared__ double T[NB][NB + 1];
  __shared__ double dv[NB];
  __shared__ int failed;
  if (status[0] >= 0) return;   // uniform across the CTA
  const int tid = threadIdx.x;
  load_tile(T, W, n, k0, nb, tid);
  if (tid == 0) failed = -1;
  __syncthreads();
  const int bad = factor_tile(T, dv, nb, &failed);
  if (bad >= 0) {
    if (tid == 0) status[0] = k0 + bad;
    return;
  }
#pragma unroll
  for (int k = 0; k < NB * NB / 256; ++k) {
    const int e = tid + 256 * k, rr = e & 63, cc = e >> 6;
    if (rr < nb && cc <= rr) W[(k0 + rr) + n * (k0 + cc)] = T[rr][cc];
  }
  if (tid < nb) dinv[k0 + tid] = dv[tid];
}

// The panel below the diagonal tile factored by k_potrf_tile: rows [k0 + NB, n) of columns [k0, k0 + NB), a thread
// per row with its 64 entries in registers, the tile in shared memory.
__global__ void __launch_bounds__(NB) k_trsm_panel(int64_t n, double* __restrict__ W, const double* __restrict__ dinv_g,
                                                   int64_t k0, const long long* __restrict__ status) {
  __shared__ double T[NB][NB + 1];
  __shared__ double dv[NB];
  if (status[0] >= 0) return;
  const int t = threadIdx.x;
  const int64_t r = k0 + NB + (int64_t)blockIdx.x * NB + t;
  // the row's 64 entries and the tile (16 columns at a time), every load of a batch in flight
  double x[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) x[c] = r < n ? W[r + n * (k0 + c)] : 0.0;
#pragma unroll
  for (int c0 = 0; c0 < NB; c0 += 16) {
    double v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = W[(k0 + t) + n * (k0 + c0 + c)];
#pragma unroll
    for (int c = 0; c < 16; ++c) T[t][c0 + c] = v[c];
  }
  dv[t] = dinv_g[k0 + t];
  __syncthreads();
  if (r >= n) return;
  solve_row(x, T, dv);
#pragma unroll
  for (int c = 0; c < NB; ++c) W[r + n * (k0 + c)] = x[c];
}

// shared memory of k_panel: the diagonal tile, the CTA's 64 panel rows, 1 / L[j, j]
constexpr int PANEL_SMEM = (2 * NB * (NB + 1) + NB) * (int)sizeof(double);

// One panel [k0, k0 + nb) in one launch of max(1, ceil(rows below / 64)) CTAs of 256 threads, for panels with few
// rows below: every CTA factors the diagonal tile in its own shared memory (the same operations on the same values,
// so every copy is identical; CTA 0 writes it and 1 / L[j, j] back) while its 64 rows below the tile arrive by
// cp.async, then a thread per row solves it. A non-positive or non-finite pivot is seen by every CTA: CTA 0 records
// its column and nothing is written.
__global__ void __launch_bounds__(256, 1) k_panel(int64_t n, double* __restrict__ W, double* __restrict__ dinv, int64_t k0,
                                                  int nb, long long* __restrict__ status) {
  extern __shared__ __align__(16) double panel_smem[];
  double (*T)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(panel_smem);
  double (*X)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(panel_smem + NB * (NB + 1));
  double* dv = panel_smem + 2 * NB * (NB + 1);
  __shared__ int failed;
  if (status[0] >= 0) return;   // uniform across the grid
  const int tid = threadIdx.x;
  const int64_t row0 = k0 + nb + (int64_t)blockIdx.x * NB;   // this CTA's rows below the tile
#pragma unroll
  for (int k = 0; k < NB * NB / 256; ++k) {
    const int e = tid + 256 * k, r = e & 63, c = e >> 6;
    const bool v = row0 + r < n;
    cp_async8(&X[r][c], v ? W + (row0 + r) + n * (k0 + c) : W, v ? 8 : 0);
  }
  cp_async_commit();
  load_tile(T, W, n, k0, nb, tid);
  if (tid == 0) failed = -1;
  __syncthreads();
  const int bad = factor_tile(T, dv, nb, &failed);
  if (bad >= 0) {
    cp_async_wait<0>();
    if (blockIdx.x == 0 && tid == 0) status[0] = k0 + bad;
    return;
  }
  if (blockIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NB * NB / 256; ++k) {
      const int e = tid + 256 * k, rr = e & 63, cc = e >> 6;
      if (rr < nb && cc <= rr) W[(k0 + rr) + n * (k0 + cc)] = T[rr][cc];
    }
    if (tid < nb) dinv[k0 + tid] = dv[tid];
  }
  cp_async_wait<0>();
  __syncthreads();
  const int64_t r = row0 + tid;
  if (tid >= NB || r >= n) return;   // rows below the tile exist only when nb == NB
  double x[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) x[c] = X[tid][c];
  solve_row(x, T, dv);
#pragma unroll
  for (int c = 0; c < NB; ++c) W[r + n * (k0 + c)] = x[c];
}

constexpr int SYRK_KC = 16, SYRK_STAGES = 3;
constexpr int SYRK_SMEM = SYRK_STAGES * 2 * SYRK_KC * NB * (int)sizeof(double);   // a ring of 16-column chunks of both panels

// The trailing lower triangle: W[i, j] -= sum_c L[i, c] L[j, c] over the panel's 64 columns, for i >= j >= k0 + NB,
// in two launches: `rest` == 0 the first tile column (the next panel), `rest` == 1 the tile columns after it.
// One CTA of 256 threads per 64 x 64 output tile of the lower triangle (tiles listed by their index in it). The two
// row panels pass through a three-stage ring of 16-column chunks in shared memory, copied asynchronously (cp.async,
// rows past n zero-filled) two chunks ahead of the products (48 KB and at most 64 registers a thread, so four CTAs fit
// an SM), and the output tile is fetched the same way into the two free stages during the last chunk. Each thread
// accumulates a 4 x 4 block (rows 2 tx + {0, 1, 32, 33}, columns 2 ty + {0, 1, 32, 33}) from 16-byte shared loads with
// FP64 fused multiply-adds (the FP64 tensor-core form, mma.sync m8n8k4 fragments per warp, measured 1.3x slower here).
__global__ void __launch_bounds__(256, 4) k_syrk_tiles(int64_t n, double* __restrict__ W, int64_t k0, int rest,
                                                       const long long* __restrict__ status) {
  constexpr int KC = SYRK_KC, NCH = NB / KC;
  extern __shared__ __align__(16) double syrk_smem[];
  auto Pi = [&](int stage) { return reinterpret_cast<double (*)[NB]>(syrk_smem + stage * 2 * KC * NB); };
  auto Pj = [&](int stage) { return reinterpret_cast<double (*)[NB]>(syrk_smem + stage * 2 * KC * NB + KC * NB); };
  if (status[0] >= 0) return;
  const int64_t t = blockIdx.x;
  int64_t ti = t, tj = 0;
  if (rest) {
    ti = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    while (ti * (ti + 1) / 2 > t) --ti;
    tj = t - ti * (ti + 1) / 2 + 1;
    ti += 1;
  }
  const int64_t bi = k0 + NB + ti * NB, bj = k0 + NB + tj * NB;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  auto issue = [&](int ch) {
    double (*A)[NB] = Pi(ch % SYRK_STAGES);
    double (*B)[NB] = Pj(ch % SYRK_STAGES);
#pragma unroll
    for (int k = 0; k < KC * NB / 256; ++k) {
      const int e = tid + 256 * k, c = e >> 6, r = e & 63;
      const int64_t col = n * (k0 + KC * ch + c);
      const bool vi = bi + r < n, vj = bj + r < n;
      cp_async8(&A[c][r], vi ? W + bi + r + col : W, vi ? 8 : 0);
      cp_async8(&B[c][r], vj ? W + bj + r + col : W, vj ? 8 : 0);
    }
    cp_async_commit();
  };
  issue(0);
  issue(1);
  double acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = 0.0;
  static_assert(NCH == 4 && SYRK_STAGES == 3, "the output tile is prefetched into stages 1 and 2 during the last chunk");
  double (*O)[NB] = reinterpret_cast<double (*)[NB]>(syrk_smem + 2 * KC * NB);   // stages 1 and 2: 64 x 64, O[col][row]
  for (int ch = 0; ch < NCH; ++ch) {
    if (ch + 2 < NCH) issue(ch + 2);   // into the stage chunk ch - 1 used: every thread passed the barrier after it
    else cp_async_commit();           // an empty group keeps the count of groups in flight uniform
    cp_async_wait<2>();
    __syncthreads();
    if (ch == NCH - 1) {
      // stages 1 and 2 are free (chunks 1 and 2 are done): fetch the output tile for the read-modify-write while the
      // last chunk's products run
#pragma unroll
      for (int k = 0; k < NB * NB / 256; ++k) {
        const int e = tid + 256 * k, col = e >> 6, row = e & 63;
        const bool v = bi + row < n && bj + col < n;
        cp_async8(&O[col][row], v ? W + (bi + row) + n * (bj + col) : W, v ? 8 : 0);
      }
      cp_async_commit();
    }
    double (*A)[NB] = Pi(ch % SYRK_STAGES);
    double (*B)[NB] = Pj(ch % SYRK_STAGES);
#pragma unroll 4
    for (int c = 0; c < KC; ++c) {
      const double2 a0 = *reinterpret_cast<const double2*>(&A[c][2 * tx]);
      const double2 a1 = *reinterpret_cast<const double2*>(&A[c][32 + 2 * tx]);
      const double2 b0 = *reinterpret_cast<const double2*>(&B[c][2 * ty]);
      const double2 b1 = *reinterpret_cast<const double2*>(&B[c][32 + 2 * ty]);
      const double ra[4] = {a0.x, a0.y, a1.x, a1.y}, rb[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = fma(ra[p], rb[q], acc[p][q]);
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  __syncthreads();
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int ri = 2 * tx + (p & 1) + 32 * (p >> 1), cj = 2 * ty + (q & 1) + 32 * (q >> 1);
      const int64_t oi = bi + ri, oj = bj + cj;
      if (oi < n && oj <= oi) W[oi + n * oj] = O[cj][ri] - acc[p][q];
    }
}

// The diagonal tile [d0, d0 + dnb) of L into t for one warp's substitution, by 256 threads (all 16 loads of a thread
// in flight), pre-scaled so that a column step is one shuffle and one fused multiply-add: forward (rows_scaled = 0),
// t[r][c] = L[r][c] / L[c][c] for r > c; backward (rows_scaled = 1), t[r][c] = L[r][c] / L[r][r] for r > c; zero on and
// above the diagonal and outside the tile.
__device__ __forceinline__ void load_scaled_tile(double (*t)[NB + 1], const double* __restrict__ W, const double* __restrict__ dinv,
                                                 int64_t n, int64_t d0, int dnb, int rows_scaled, int tid) {
  double v[NB * NB / 256];
#pragma unroll
  for (int k = 0; k < NB * NB / 256; ++k) {
    const int e = tid + 256 * k, rr = e & 63, cc = e >> 6;
    v[k] = (rr < dnb && cc < rr) ? W[(d0 + rr) + n * (d0 + cc)] * dinv[d0 + (rows_scaled ? rr : cc)] : 0.0;
  }
#pragma unroll
  for (int k = 0; k < NB * NB / 256; ++k) {
    const int e = tid + 256 * k;
    t[e & 63][e >> 6] = v[k];
  }
}

// The forward substitution of one diagonal tile [d0, d0 + dnb) by one warp, t from load_scaled_tile (forward): lanes
// own rows lane and lane + 32 and start from ys (shared); per column the finished row value is shuffled from its lane
// and every lane subtracts its scaled entry times it, so the column chain is a shuffle and a fused multiply-add; the
// rows are multiplied by 1 / L[r][r] (dlo, dhi) once at the end and written to y.
__device__ __forceinline__ void tile_forward(const double (*t)[NB + 1], double dlo, double dhi, const double* ys,
                                             double* __restrict__ y, int64_t d0, int dnb, int lane) {
  double y0 = ys[lane], y1 = ys[lane + 32];
#pragma unroll 8
  for (int c = 0; c < 32; ++c) {
    const double yc = __shfl_sync(0xffffffffu, y0, c);
    y0 = fma(-t[lane][c], yc, y0);
    y1 = fma(-t[lane + 32][c], yc, y1);
  }
#pragma unroll 8
  for (int c = 32; c < NB; ++c) {
    const double yc = __shfl_sync(0xffffffffu, y1, c - 32);
    y1 = fma(-t[lane + 32][c], yc, y1);
  }
  if (lane < dnb) y[d0 + lane] = y0 * dlo;
  if (lane + 32 < dnb) y[d0 + 32 + lane] = y1 * dhi;
}

// The backward substitution (L' x = y) of one diagonal tile [d0, d0 + dnb), t from load_scaled_tile (backward), as
// tile_forward from the last column to the first.
__device__ __forceinline__ void tile_backward(const double (*t)[NB + 1], double dlo, double dhi, const double* ys,
                                              double* __restrict__ y, int64_t d0, int dnb, int lane) {
  double y0 = ys[lane], y1 = ys[lane + 32];
#pragma unroll 8
  for (int c = NB - 1; c >= 32; --c) {
    const double yc = __shfl_sync(0xffffffffu, y1, c - 32);
    y1 = fma(-t[c][lane + 32], yc, y1);
    y0 = fma(-t[c][lane], yc, y0);
  }
#pragma unroll 8
  for (int c = 31; c >= 0; --c) {
    const double yc = __shfl_sync(0xffffffffu, y0, c);
    y0 = fma(-t[c][lane], yc, y0);
  }
  if (lane < dnb) y[d0 + lane] = y0 * dlo;
  if (lane + 32 < dnb) y[d0 + 32 + lane] = y1 * dhi;
}

// One forward step of L y = g, y in place: rows [d0, n) take the update from the solved tile [d0 - NB, d0) (when
// `update`), CTA b the 64 rows from d0 + 64 b, four threads per row over 16 columns each; then CTA 0, whose rows are
// the next diagonal tile [d0, d0 + dnb), solves it. Every global load of the step is issued before the first barrier,
// and CTA 0 keeps its updated rows in shared memory, so the step costs one round trip to memory plus the tile's chain.
__global__ void __launch_bounds__(256) k_fwd_step(int64_t n, const double* __restrict__ W, const double* __restrict__ dinv,
                                                  double* __restrict__ y, int64_t d0, int dnb, int update) {
  __shared__ double t[NB][NB + 1];
  __shared__ double yk[NB];
  __shared__ double part[4][NB];
  __shared__ double ys[NB];
  const int tid = threadIdx.x, r = tid & 63, q = tid >> 6;
  const int64_t i = d0 + (int64_t)blockIdx.x * NB + r, k0 = d0 - NB;
  double w[16];
  double yi = 0.0, dlo = 0.0, dhi = 0.0;
  if (update) {
    if (i < n) {
#pragma unroll
      for (int c = 0; c < 16; ++c) w[c] = W[i + n * (k0 + 16 * q + c)];
    }
    if (tid < NB) yk[tid] = y[k0 + tid];
  }
  if (q == 0 && i < n) yi = y[i];
  if (blockIdx.x == 0) {
    load_scaled_tile(t, W, dinv, n, d0, dnb, 0, tid);
    if (tid < 32) {
      if (tid < dnb) dlo = dinv[d0 + tid];
      if (tid + 32 < dnb) dhi = dinv[d0 + 32 + tid];
    }
  }
  __syncthreads();
  if (update) {
    double s = 0.0;
    if (i < n) {
#pragma unroll
      for (int c = 0; c < 16; ++c) s = fma(w[c], yk[16 * q + c], s);
    }
    part[q][r] = s;
    __syncthreads();
    if (q == 0) yi -= (part[0][r] + part[1][r]) + (part[2][r] + part[3][r]);
  }
  if (blockIdx.x != 0) {
    if (update && q == 0 && i < n) y[i] = yi;
    return;
  }
  if (q == 0) ys[r] = yi;
  __syncthreads();
  if (tid < 32) tile_forward(t, dlo, dhi, ys, y, d0, dnb, tid);
}

// One backward step of L' x = y, in place: rows [0, k0) take the update from the solved tile [k0, k0 + unb), CTA b
// the 64 rows below k0 - 64 b, a warp per row reading that row's entries of the tile's rows of L (64 contiguous
// values of one column of W); then CTA 0, whose rows are the tile [k0 - NB, k0), solves it. Loads are issued before
// the first barrier and CTA 0's rows stay in shared memory, as in the forward step.
__global__ void __launch_bounds__(256) k_bwd_step(int64_t n, const double* __restrict__ W, const double* __restrict__ dinv,
                                                  double* __restrict__ y, int64_t k0, int unb) {
  __shared__ double t[NB][NB + 1];
  __shared__ double xk[NB];
  __shared__ double ys[NB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t row0 = k0 - NB * (int64_t)(blockIdx.x + 1);   // this CTA's rows [row0, row0 + 64)
  double w0[8], w1[8];
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const double* colj = W + n * (row0 + warp * 8 + m) + k0;
    w0[m] = lane < unb ? colj[lane] : 0.0;
    w1[m] = lane + 32 < unb ? colj[lane + 32] : 0.0;
  }
  if (tid < NB) xk[tid] = tid < unb ? y[k0 + tid] : 0.0;
  const double yold = lane < 8 ? y[row0 + warp * 8 + lane] : 0.0;
  double dlo = 0.0, dhi = 0.0;
  if (blockIdx.x == 0) {
    load_scaled_tile(t, W, dinv, n, row0, NB, 1, tid);
    if (tid < 32) {
      dlo = dinv[row0 + tid];
      dhi = dinv[row0 + 32 + tid];
    }
  }
  __syncthreads();
  const double x0 = xk[lane], x1 = xk[lane + 32];
  double s[8];
#pragma unroll
  for (int m = 0; m < 8; ++m) s[m] = w0[m] * x0 + w1[m] * x1;
#pragma unroll
  for (int m = 0; m < 8; ++m) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[m] += __shfl_xor_sync(0xffffffffu, s[m], o);
  }
  double v = s[0];
#pragma unroll
  for (int m = 1; m < 8; ++m)
    if (lane == m) v = s[m];
  if (blockIdx.x != 0) {
    if (lane < 8) y[row0 + warp * 8 + lane] = yold - v;
    return;
  }
  if (lane < 8) ys[warp * 8 + lane] = yold - v;
  __syncthreads();
  if (tid < 32) tile_backward(t, dlo, dhi, ys, y, row0, NB, tid);
}

// The last diagonal tile [d0, n) of the backward pass (the only one that may be short), solved by one warp.
__global__ void __launch_bounds__(32) k_bwd_last(int64_t n, const double* __restrict__ W, const double* __restrict__ dinv,
                                                 double* __restrict__ y, int64_t d0) {
  __shared__ double t[NB][NB + 1];
  __shared__ double ys[NB];
  const int lane = threadIdx.x, dnb = (int)(n - d0);
  for (int e = lane; e < NB * NB; e += 32) {
    const int rr = e & 63, cc = e >> 6;
    t[rr][cc] = (rr < dnb && cc < rr) ? W[(d0 + rr) + n * (d0 + cc)] * dinv[d0 + rr] : 0.0;
  }
  ys[lane] = lane < dnb ? y[d0 + lane] : 0.0;
  ys[lane + 32] = lane + 32 < dnb ? y[d0 + 32 + lane] : 0.0;
  const double dlo = lane < dnb ? dinv[d0 + lane] : 0.0, dhi = lane + 32 < dnb ? dinv[d0 + 32 + lane] : 0.0;
  __syncwarp();
  tile_backward(t, dlo, dhi, ys, y, d0, dnb, lane);
}

// x = (L L')^-1 x in place: the forward steps, then the backward steps, on stream s
static void launch_solve(cudaStream_t s, int64_t n, const double* W, const double* dv, double* x) {
  // forward: tile [0, NB) first, then each step updates the rows below the tile it just solved and solves the next
  k_fwd_step<<<1, 256, 0, s>>>(n, W, dv, x, 0, (int)std::min<int64_t>(NB, n), 0);
  for (int64_t d0 = NB; d0 < n; d0 += NB)
    k_fwd_step<<<(unsigned)((n - d0 + NB - 1) / NB), 256, 0, s>>>(n, W, dv, x, d0, (int)std::min<int64_t>(NB, n - d0), 1);
  // backward: the last (possibly short) tile first, then upward
  const int64_t kl = ((n - 1) / NB) * NB;
  k_bwd_last<<<1, 32, 0, s>>>(n, W, dv, x, kl);
  for (int64_t k0 = kl; k0 > 0; k0 -= NB)
    k_bwd_step<<<(unsigned)(k0 / NB), 256, 0, s>>>(n, W, dv, x, k0, (int)std::min<int64_t>(NB, n - k0));
}

// Launches kernel on stream st with the given priority (a launch attribute, so that a captured graph keeps it).
template <class... Args>
static void launch_prio(void (*kernel)(Args...), unsigned grid, unsigned block, size_t smem, cudaStream_t st, int prio,
                        Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributePriority;
  attr[0].val.priority = prio;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BLS_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
}

// The factorisation after the load of S into W: panels on the panel stream p, trailing updates on s, joined on s.
static void launch_factor_body(DenseSolver* D, cudaStream_t s, cudaStream_t p) {
  const int64_t n = D->n;
  double* W = D->W.as<double>();
  double* dv = D->dinv.as<double>();
  long long* st = D->status.as<long long>();
  const int prio = D->panel_priority;
  BLS_CUDA(cudaEventRecord(D->ev_join, s));
  BLS_CUDA(cudaStreamWaitEvent(p, D->ev_join, 0));
  // panel k: its diagonal tile and the rows below it, on the panel stream. With few rows below, one launch in which
  // every CTA factors the tile itself (a launch less on the panel chain); with many, the tile in one CTA and then the
  // rows (the redundant factorisations would take SMs from the trailing update running beside them).
  auto panel = [&](int64_t k0) {
    const int nb = (int)std::min<int64_t>(NB, n - k0);
    const int64_t below = (n - k0 - nb + NB - 1) / NB;
    if (below <= kFusedPanelTiles) {
      launch_prio(k_panel, (unsigned)std::max<int64_t>(1, below), 256, PANEL_SMEM, p, prio, n, W, dv, k0, nb, st);
    } else {
      launch_prio(k_potrf_tile, 1, 256, 0, p, prio, n, W, dv, k0, nb, st);
      launch_prio(k_trsm_panel, (unsigned)below, NB, 0, p, prio, n, W, (const double*)dv, k0, (const long long*)st);
    }
    BLS_CUDA(cudaEventRecord(D->ev_panel, p));
  };
  panel(0);
  // Lookahead by one panel: the trailing update of panel k updates the next panel's tile column first; the next panel
  // is factored on the panel stream while the caller's stream updates the tile columns after it.
  for (int64_t k0 = 0; n - k0 > NB; k0 += NB) {
    const int64_t nt = (n - k0 - NB + NB - 1) / NB;
    BLS_CUDA(cudaStreamWaitEvent(s, D->ev_panel, 0));
    k_syrk_tiles<<<(unsigned)nt, 256, SYRK_SMEM, s>>>(n, W, k0, 0, st);
    BLS_CUDA(cudaEventRecord(D->ev_join, s));
    BLS_CUDA(cudaStreamWaitEvent(p, D->ev_join, 0));
    panel(k0 + NB);
    if (nt > 1) k_syrk_tiles<<<(unsigned)((nt - 1) * nt / 2), 256, SYRK_SMEM, s>>>(n, W, k0, 1, st);
  }
  BLS_CUDA(cudaStreamWaitEvent(s, D->ev_panel, 0));
}

template <class T>
static int factor(DenseSolver* D, const T* S, double lambda, const double* s_r, int64_t* failed_column) {
  if (!S) throw Error(BLS_EINVAL, "S is NULL");
  cudaStream_t s = D->ctx->stream;
  const int64_t n = D->n;
  double* W = D->W.as<double>();
  long long* st = D->status.as<long long>();
  if (!D->panel_stream) {
    int lo = 0, hi = 0;
    BLS_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    D->panel_priority = hi;
    BLS_CUDA(cudaStreamCreateWithPriority(&D->panel_stream, cudaStreamNonBlocking, hi));
    BLS_CUDA(cudaEventCreateWithFlags(&D->ev_join, cudaEventDisableTiming));
    BLS_CUDA(cudaEventCreateWithFlags(&D->ev_panel, cudaEventDisableTiming));
    BLS_CUDA(cudaFuncSetAttribute(k_syrk_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, SYRK_SMEM));
    BLS_CUDA(cudaFuncSetAttribute(k_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, PANEL_SMEM));
  }
  k_dense_load<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((n * n + 255) / 256, 148 * 8)), 256, 0, s>>>(n, S, W, lambda, s_r, st);
  if (!D->factor_graph) {
    if (!D->cap_stream) BLS_CUDA(cudaStreamCreateWithFlags(&D->cap_stream, cudaStreamNonBlocking));
    BLS_CUDA(cudaStreamBeginCapture(D->cap_stream, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t gr = nullptr;
    try {
      launch_factor_body(D, D->cap_stream, D->panel_stream);
    } catch (...) {
      cudaStreamEndCapture(D->cap_stream, &gr);
      if (gr) cudaGraphDestroy(gr);
      throw;
    }
    BLS_CUDA(cudaStreamEndCapture(D->cap_stream, &gr));
    const cudaError_t e = cudaGraphInstantiate(&D->factor_graph, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) {
      D->factor_graph = nullptr;
      throw Error(BLS_ECUDA, std::string("instantiating the factorisation: ") + cudaGetErrorString(e));
    }
  }
  BLS_CUDA(cudaGraphLaunch(D->factor_graph, s));
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
    D->dinv.alloc(sizeof(double) * (size_t)n);
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
    if (dtype == BLS_F64) return factor<double>(D, (const double*)S, 0.0, nullptr, failed_column);
    if (dtype == BLS_F32) return factor<float>(D, (const float*)S, 0.0, nullptr, failed_column);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_dense_cholesky_shifted(bls_dense_solver* D, int dtype, const void* S, double lambda, const double* s_r, int64_t* failed_column) {
  DENSE_GUARD({
    if (!D || !s_r) throw Error(BLS_EINVAL, "null argument");
    if (!(std::isfinite(lambda) && lambda >= 0))
      throw Error(BLS_EINVAL, "lambda must be finite and non-negative, got " + std::to_string(lambda));
    if (dtype == BLS_F64) return factor<double>(D, (const double*)S, lambda, s_r, failed_column);
    if (dtype == BLS_F32) return factor<float>(D, (const float*)S, lambda, s_r, failed_column);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_dense_cholesky_solve(bls_dense_solver* D, const double* g, double* x) {
  DENSE_GUARD({
    if (!D || !g || !x) throw Error(BLS_EINVAL, "null argument");
    if (!D->factored) throw Error(BLS_EINVAL, "the solver holds no factorisation (bls_dense_cholesky first, and it must succeed)");
    const int64_t n = D->n;
    const double* W = D->W.as<double>();
    const double* dv = D->dinv.as<double>();
    cudaStream_t s = D->ctx->stream;
    if (!D->solve_graph) {
      D->y.alloc(sizeof(double) * (size_t)n);
      if (!D->cap_stream) BLS_CUDA(cudaStreamCreateWithFlags(&D->cap_stream, cudaStreamNonBlocking));
      BLS_CUDA(cudaStreamBeginCapture(D->cap_stream, cudaStreamCaptureModeThreadLocal));
      launch_solve(D->cap_stream, n, W, dv, D->y.as<double>());
      cudaGraph_t gr = nullptr;
      const cudaError_t e1 = cudaGetLastError();
      const cudaError_t e2 = cudaStreamEndCapture(D->cap_stream, &gr);
      if (e1 != cudaSuccess || e2 != cudaSuccess) {
        if (gr) cudaGraphDestroy(gr);
        throw Error(BLS_ECUDA, std::string("capturing the solve: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
      }
      const cudaError_t e3 = cudaGraphInstantiate(&D->solve_graph, gr, 0);
      cudaGraphDestroy(gr);
      if (e3 != cudaSuccess) {
        D->solve_graph = nullptr;
        throw Error(BLS_ECUDA, std::string("instantiating the solve: ") + cudaGetErrorString(e3));
      }
    }
    double* y = D->y.as<double>();
    BLS_CUDA(cudaMemcpyAsync(y, g, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    BLS_CUDA(cudaGraphLaunch(D->solve_graph, s));
    BLS_CUDA(cudaMemcpyAsync(x, y, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

}  // extern "C"
