// Block-Jacobi and preconditioned conjugate gradients on the reduced camera system S x = g, on sm_100a.
//
// Reference: factor_diagonal_blocks! / solve_diagonal_blocks! (src/diagonal_blocks.jl:6-61), the block-Jacobi
// preconditioner of the LSMR path (ext/KrylovExt.jl:97-132). PCG itself has no counterpart in the reference: it is the
// iterative reduced solve on the Schur complement that the sparse reduction feeds (src/schur_linear_systems.jl:362-406
// solves the same system with CHOLMOD / LDLFactorizations).
//
// S is the reduction's output: the upper block triangle of the symmetric reduced matrix in the CSC layout of
// build_schur_pattern (column r2 of blocks (r1 <= r2), column stride col_heights[r2]; diagonal blocks stored full with
// only their upper triangle meaningful). When every retained block has 6 columns, y = S x reads each stored entry once,
// one warp per block column (k_spmv_cols): B p_r2 is scattered into the rows r1 with FP64 atomics and B' p_r1 summed
// for the column; otherwise it reads each stored block twice, as B for block row r1 and as B' for block row r2, from a
// per-row list built once per pattern (one warp per block row gathers its row: no atomics, deterministic). Vectors,
// scalars and products are FP64 whatever S's storage type.
//
// One PCG iteration is three kernels (four with the column product): (1) q = S p with the partial sums of p'q (the
// column form takes a separate p'q pass); (2) alpha = (r'z)/(p'q), x += alpha p, r -= alpha q, z = M^-1 r (block
// solves) with the partial sums of r'z and r'r; (3) beta, p = z + beta p, and the convergence test. Per-iteration scalars live in device slots, so a run of iterations can be replayed as one CUDA
// graph; after convergence the remaining kernels of the run return at once. The converged x is checked by an explicit
// FP64 residual g - S x; if the recursive residual drifted above the tolerance, PCG restarts from x (iterative
// refinement).
#include <algorithm>
#include <cmath>
#include <climits>
#include <memory>
#include <vector>

#include "pcg_plan.hpp"

namespace bls {

// ---------------------------------------------------------------------------------------------------------------
// Block-Jacobi: factor_diagonal_blocks! and solve_diagonal_blocks! (src/diagonal_blocks.jl:6-61)
// ---------------------------------------------------------------------------------------------------------------

// One thread per block: the Cholesky factor L of the d x d block in place in its lower triangle, in the reference's
// operation order. A block that is not positive definite (or not finite) records its index (lowest wins).
template <class T>
__global__ void k_factor_blocks(int64_t nb, const int32_t* __restrict__ dims, const int64_t* __restrict__ doff, T* __restrict__ D,
                                long long* __restrict__ failed) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int d = dims[b];
  T* A = D + doff[b];
  for (int j = 0; j < d; ++j) {
    T s = A[j * d + j];
    for (int k = 0; k < j; ++k) {
      const T l = A[k * d + j];
      s -= l * l;
    }
    if (!(s > T(0) && isfinite((double)s))) {
      atomicMin(failed, (long long)b);
      return;
    }
    const T ljj = sqrt(s);
    A[j * d + j] = ljj;
    for (int i = j + 1; i < d; ++i) {
      T t = A[j * d + i];
      for (int k = 0; k < j; ++k) t -= A[k * d + i] * A[k * d + j];
      A[j * d + i] = t / ljj;
    }
  }
}

// y = (L L')^-1 x per block, with D factored as above (y may alias x)
template <class T>
__device__ __forceinline__ void block_solve(double* y, const T* __restrict__ L, int d, const double* x) {
  double v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i)
    if (i < d) v[i] = x[i];
  for (int j = 0; j < d; ++j) {
    const double yj = v[j] / (double)L[j * d + j];
    v[j] = yj;
    for (int i = j + 1; i < d; ++i) v[i] -= (double)L[j * d + i] * yj;
  }
  for (int j = d - 1; j >= 0; --j) {
    double t = v[j];
    for (int i = j + 1; i < d; ++i) t -= (double)L[j * d + i] * v[i];
    v[j] = t / (double)L[j * d + j];
  }
#pragma unroll
  for (int i = 0; i < 16; ++i)
    if (i < d) y[i] = v[i];
}

template <class T>
__global__ void k_solve_blocks(int64_t nb, const int32_t* __restrict__ dims, const int64_t* __restrict__ doff, const int64_t* __restrict__ voff,
                               const T* __restrict__ D, const double* __restrict__ x, double* __restrict__ y) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= nb) return;
  block_solve<T>(y + voff[b], D + doff[b], dims[b], x + voff[b]);
}

// ---------------------------------------------------------------------------------------------------------------
// y = S x (or y = g - S x) from the upper block storage, one warp per block row
// ---------------------------------------------------------------------------------------------------------------
template <class T, bool RESIDUAL, bool DOT>
__global__ void __launch_bounds__(256) k_spmv(int64_t nrb, const int64_t* __restrict__ row_ptr, const RowEntry* __restrict__ rows,
                                              const int32_t* __restrict__ dims, const int32_t* __restrict__ boff, const T* __restrict__ S,
                                              const double* __restrict__ x, const double* __restrict__ g, double* __restrict__ y,
                                              double* __restrict__ dot_out, const int* __restrict__ done) {
  if (done && *done) return;
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  double part = 0.0;
  if (r < nrb) {
    const int dr = dims[r];
    double acc[16];
#pragma unroll
    for (int a = 0; a < 16; ++a) acc[a] = 0.0;
    for (int64_t e = row_ptr[r] + lane; e < row_ptr[r + 1]; e += 32) {
      const RowEntry en = rows[e];
      const T* B = S + en.base;
      const double* xv = x + en.xo;
      if (en.mode == 0) {            // S[r, c] = B (dr x dother): acc[a] += B[a, w] x[w]
        for (int w = 0; w < en.dother; ++w) {
          const double xw = xv[w];
          const T* col = B + (int64_t)w * en.stride;
#pragma unroll
          for (int a = 0; a < 16; ++a)
            if (a < dr) acc[a] += (double)col[a] * xw;
        }
      } else if (en.mode == 1) {     // S[r, c] = B' (B is dother x dr): acc[w] += B[a, w] x[a]
#pragma unroll
        for (int w = 0; w < 16; ++w) {
          if (w < dr) {
            const T* col = B + (int64_t)w * en.stride;
            double s = 0.0;
            for (int a = 0; a < en.dother; ++a) s += (double)col[a] * xv[a];
            acc[w] += s;
          }
        }
      } else {                       // diagonal block: upper triangle, mirrored
#pragma unroll
        for (int a = 0; a < 16; ++a) {
          if (a < dr) {
            double s = 0.0;
            for (int w = 0; w < dr; ++w) {
              const int lo = a < w ? a : w, hi = a < w ? w : a;
              s += (double)B[lo + (int64_t)hi * en.stride] * xv[w];
            }
            acc[a] += s;
          }
        }
      }
    }
#pragma unroll
    for (int a = 0; a < 16; ++a) {
      if (a < dr) {
        double v = acc[a];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        acc[a] = v;
      }
    }
    if (lane < dr) {
      double v = 0.0;
#pragma unroll
      for (int a = 0; a < 16; ++a)
        if (a == lane) v = acc[a];
      const int64_t i = boff[r] + lane;
      if (RESIDUAL) v = g[i] - v;
      y[i] = v;
      if (DOT) part = x[i] * v;
    }
  }
  if (DOT) {
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0 && part != 0.0) atomicAdd(dot_out, part);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// PCG iteration kernels (thread per block row)
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Start: r = g - S x (already in r), z = M^-1 r, p = z, rz and rr into slot 0
// z = M^-1 r for one block: the block-Jacobi solve with the factored D, or the dense block Bp (d x d, column-major)
__device__ __forceinline__ void precondition(double* z, const double* __restrict__ D, const double* __restrict__ Bp, int d, const double* r) {
  if (Bp) {
    double v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = 0.0;
    for (int j = 0; j < d; ++j) {
      const double rj = r[j];
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (i < d) v[i] += Bp[j * d + i] * rj;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (i < d) z[i] = v[i];
  } else {
    block_solve<double>(z, D, d, r);
  }
}

__global__ void k_pcg_start(int64_t nrb, const int32_t* __restrict__ dims, const int32_t* __restrict__ boff, const int64_t* __restrict__ doff,
                            const double* __restrict__ D, const double* __restrict__ Bp, const double* __restrict__ r, double* __restrict__ z,
                            double* __restrict__ p, double* __restrict__ q, double* __restrict__ slot0) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double rz = 0.0, rr = 0.0;
  if (b < nrb) {
    const int d = dims[b];
    const int64_t o = boff[b];
    precondition(z + o, D + doff[b], Bp ? Bp + doff[b] : nullptr, d, r + o);
    for (int i = 0; i < d; ++i) {
      q[o + i] = 0.0;
      p[o + i] = z[o + i];
      rz += r[o + i] * z[o + i];
      rr += r[o + i] * r[o + i];
    }
  }
  rz = warp_sum_d(rz);
  rr = warp_sum_d(rr);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(slot0 + PS_RZ, rz);
    atomicAdd(slot0 + PS_RRN, rr);
  }
}

// q += S p by block columns, for patterns whose retained blocks all have 6 columns: one warp per block column r2,
// lanes over (block, row) of five blocks at a time, each stored entry read once. A block (r1, r2) adds B p_r2 to q_r1
// (one FP64 atomic per row) and B' p_r1 to q_r2 (summed over the column's blocks in registers, one atomic per column
// entry at the end); the diagonal block uses its upper triangle both ways. q must be zero on entry (k_pcg_update and
// k_pcg_start clear it); after convergence within a replayed run the kernel returns at once.
template <class T>
__global__ void __launch_bounds__(256) k_spmv_cols(int64_t nrb, const int64_t* __restrict__ c_ptr, const int64_t* __restrict__ c_base,
                                                   const int32_t* __restrict__ c_xo, const int32_t* __restrict__ c_stride,
                                                   const T* __restrict__ S, const double* __restrict__ p, double* __restrict__ q,
                                                   const int* __restrict__ done) {
  if (done && *done) return;
  const int64_t r2 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r2 >= nrb) return;
  const int64_t j0 = 6 * r2;
  const int64_t stride = c_stride[r2];
  double pj[6];
#pragma unroll
  for (int w = 0; w < 6; ++w) pj[w] = p[j0 + w];
  double t[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const int sub = lane / 6, a = lane - 6 * sub;
  const int64_t kb = c_ptr[r2], ke = c_ptr[r2 + 1];
  // the next run's block offsets are loaded while the current run is computed (one dependent load less per run; a
  // two-deep pipeline that also preloads the entries measured slower: 80 registers against 64)
  int64_t base_n = 0;
  int xo_n = 0;
  if (lane < 30 && kb + sub < ke) {
    base_n = c_base[kb + sub];
    xo_n = c_xo[kb + sub];
  }
  for (int64_t k0 = kb; k0 < ke; k0 += 5) {
    const int64_t k = k0 + sub;
    const int64_t base = base_n;
    const int i0 = xo_n;
    if (lane < 30 && k + 5 < ke) {
      base_n = c_base[k + 5];
      xo_n = c_xo[k + 5];
    }
    if (lane < 30 && k < ke) {
      const T* B = S + base + a;
      const bool diag = i0 == j0;
      double sv[6];
#pragma unroll
      for (int w = 0; w < 6; ++w) sv[w] = (double)B[w * stride];
      const double pi = p[i0 + a];
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < 6; ++w) {
        if (!diag || w >= a) v += sv[w] * pj[w];
        if (!diag || w > a) t[w] += sv[w] * pi;
      }
      atomicAdd(q + i0 + a, v);
    }
  }
#pragma unroll
  for (int w = 0; w < 6; ++w)
    for (int o = 16; o > 0; o >>= 1) t[w] += __shfl_xor_sync(0xffffffffu, t[w], o);
  if (lane < 6) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < 6; ++w)
      if (w == lane) v = t[w];
    atomicAdd(q + j0 + lane, v);
  }
}

// y = g - y (the residual from a product accumulated in y)
__global__ void k_from_g(int64_t n, const double* __restrict__ g, double* __restrict__ y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = g[i] - y[i];
}

// p'q into the iteration's slot (after k_spmv_cols)
__global__ void k_dot_pq(int64_t n, const double* __restrict__ p, const double* __restrict__ q, double* __restrict__ out,
                         const int* __restrict__ done) {
  if (*done) return;
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) s += p[i] * q[i];
  s = warp_sum_d(s);
  if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(out, s);
}

// (2) alpha = rz / pq; x += alpha p; r -= alpha q; z = M^-1 r; rz_next, rr_next
__global__ void k_pcg_update(int64_t nrb, const int32_t* __restrict__ dims, const int32_t* __restrict__ boff, const int64_t* __restrict__ doff,
                             const double* __restrict__ D, const double* __restrict__ Bp, double* __restrict__ x, double* __restrict__ r,
                             double* __restrict__ z,
                             const double* __restrict__ p, double* __restrict__ q, double* __restrict__ slot,
                             const int* __restrict__ done, int clear_q) {
  if (*done) return;
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const double alpha = slot[PS_RZ] / slot[PS_PQ];
  double rz = 0.0, rr = 0.0;
  if (b < nrb) {
    const int d = dims[b];
    const int64_t o = boff[b];
    for (int i = 0; i < d; ++i) {
      x[o + i] += alpha * p[o + i];
      r[o + i] -= alpha * q[o + i];
      if (clear_q) q[o + i] = 0.0;   // the next q = S p accumulates into zeros
    }
    precondition(z + o, D + doff[b], Bp ? Bp + doff[b] : nullptr, d, r + o);
    for (int i = 0; i < d; ++i) {
      rz += r[o + i] * z[o + i];
      rr += r[o + i] * r[o + i];
    }
  }
  rz = warp_sum_d(rz);
  rr = warp_sum_d(rr);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(slot + PS_RZN, rz);
    atomicAdd(slot + PS_RRN, rr);
  }
}

// (3) convergence test on rr_next; beta = rz_next / rz; p = z + beta p; the next slot's rz. flags: [0] done,
// [1] iterations; tol2 = (tol * |g|)^2 read from scal's last entry.
__global__ void k_pcg_direction(int64_t nr, const double* __restrict__ z, double* __restrict__ p, double* __restrict__ slot,
                                double* __restrict__ next, const double* __restrict__ tol2, int* __restrict__ flags) {
  if (flags[0]) return;
  const double rrn = slot[PS_RRN];
  const bool conv = !(rrn > *tol2);   // also stops on NaN
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (conv) {
    if (i == 0) {
      flags[0] = 1;
      flags[1] += 1;
    }
    return;
  }
  const double beta = slot[PS_RZN] / slot[PS_RZ];
  if (i < nr) p[i] = z[i] + beta * p[i];
  if (i == 0) {
    next[PS_RZ] = slot[PS_RZN];
    flags[1] += 1;
  }
}

// Before a run of K iterations: zero the accumulators of slots 0..K and move the carried rz of slot K into slot 0
__global__ void k_pcg_slots(double* __restrict__ scal, int K) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double carry = scal[K * PS_W + PS_RZ];
  for (int i = 0; i < (K + 1) * PS_W; ++i) scal[i] = 0.0;
  scal[PS_RZ] = carry;
}

// Full diagonal blocks of S (upper triangle mirrored), one thread per entry
template <class T>
__global__ void k_extract_diag(int64_t nrb, int dmax, const int32_t* __restrict__ dims, const int64_t* __restrict__ dbase,
                               const int32_t* __restrict__ dstride, const int64_t* __restrict__ doff, const T* __restrict__ S,
                               double* __restrict__ D) {
  const int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t b = id / (dmax * dmax);
  if (b >= nrb) return;
  const int e = (int)(id - b * dmax * dmax), d = dims[b];
  const int w = e / dmax, a = e - w * dmax;
  if (w >= d || a >= d) return;
  const int lo = a < w ? a : w, hi = a < w ? w : a;
  D[doff[b] + w * d + a] = (double)S[dbase[b] + lo + (int64_t)hi * dstride[b]];
}

__global__ void k_dot_self(int64_t n, const double* __restrict__ v, double* __restrict__ out) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) s += v[i] * v[i];
  s = warp_sum_d(s);
  if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(out, s);
}

__global__ void k_zero_d(double* __restrict__ p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = 0.0;
}

// Refined solve helpers: y += lambda * sc .* x (the damping of the reset system), r = g - y, x += d
__global__ void k_add_damping(int64_t n, double* __restrict__ y, double lambda, const double* __restrict__ sc, const double* __restrict__ x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] += lambda * sc[i] * x[i];
}
__global__ void k_residual(int64_t n, double* __restrict__ r, const double* __restrict__ g, const double* __restrict__ y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) r[i] = g[i] - y[i];
}
__global__ void k_add(int64_t n, double* __restrict__ x, const double* __restrict__ d) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) x[i] += d[i];
}

// ---------------------------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------------------------
static PCGPlan* pcg_plan_create(bls_ctx* ctx, int64_t nrb, const int64_t* r_dims, const int64_t* bcolptr, const int64_t* browval,
                                const int64_t* brow_off, const int64_t* col_h, const int64_t* Scolptr) {
  if (nrb < 1 || !r_dims || !bcolptr || !browval || !brow_off || !col_h || !Scolptr) throw Error(BLS_EINVAL, "a PCG plan needs the block pattern");
  std::unique_ptr<PCGPlan> P(new PCGPlan());
  P->ctx = ctx;
  cudaStream_t s = ctx->stream;
  P->nrb = nrb;
  std::vector<int32_t> dims(nrb), boff(nrb);
  std::vector<int64_t> doff(nrb + 1, 0), voff(nrb);
  int64_t nr = 0;
  for (int64_t r = 0; r < nrb; ++r) {
    if (r_dims[r] < 1 || r_dims[r] > 16) throw Error(BLS_EUNSUPPORTED, "retained block sizes above 16 are not supported on the device");
    dims[r] = (int32_t)r_dims[r];
    boff[r] = (int32_t)nr;
    voff[r] = nr;
    nr += r_dims[r];
    doff[r + 1] = doff[r] + r_dims[r] * r_dims[r];
    P->max_d = std::max<int>(P->max_d, dims[r]);
  }
  P->nr = nr;
  P->nnz = Scolptr[nr];
  P->ndiag = doff[nrb];
  std::vector<std::vector<RowEntry>> rows(nrb);
  std::vector<int64_t> dbase(nrb, -1);
  std::vector<int32_t> dstride(nrb, 0);
  for (int64_t r2 = 0; r2 < nrb; ++r2) {
    for (int64_t w = 0; w < dims[r2]; ++w)
      if (Scolptr[boff[r2] + w + 1] - Scolptr[boff[r2] + w] != col_h[r2]) throw Error(BLS_EINVAL, "S_colptr does not match col_heights");
    for (int64_t k = bcolptr[r2]; k < bcolptr[r2 + 1]; ++k) {
      const int64_t r1 = browval[k];
      if (r1 < 0 || r1 > r2 || brow_off[k] < 0 || brow_off[k] + dims[r1] > col_h[r2]) throw Error(BLS_EINVAL, "malformed block pattern");
      RowEntry e{};
      e.base = Scolptr[boff[r2]] + brow_off[k];
      e.stride = (int32_t)col_h[r2];
      if (r1 == r2) {
        e.xo = boff[r2];
        e.dother = (int16_t)dims[r2];
        e.mode = 2;
        rows[r2].push_back(e);
        dbase[r2] = e.base;
        dstride[r2] = e.stride;
      } else {
        e.xo = boff[r2];
        e.dother = (int16_t)dims[r2];
        e.mode = 0;
        rows[r1].push_back(e);
        e.xo = boff[r1];
        e.dother = (int16_t)dims[r1];
        e.mode = 1;
        rows[r2].push_back(e);
      }
    }
  }
  for (int64_t r = 0; r < nrb; ++r)
    if (dbase[r] < 0) throw Error(BLS_EINVAL, "the pattern has no diagonal block " + std::to_string(r + 1));
  std::vector<int64_t> rptr(nrb + 1, 0);
  std::vector<RowEntry> flat;
  for (int64_t r = 0; r < nrb; ++r) {
    flat.insert(flat.end(), rows[r].begin(), rows[r].end());
    rptr[r + 1] = (int64_t)flat.size();
  }
  upload(P->row_ptr, rptr, s);
  upload(P->rows, flat, s);
  if (P->max_d == 6) {
    bool all6 = true;
    for (int64_t r = 0; r < nrb && all6; ++r) all6 = dims[r] == 6;
    if (all6 && bcolptr[nrb] < INT32_MAX) {
      std::vector<int64_t> cptr(bcolptr, bcolptr + nrb + 1), cbase(bcolptr[nrb]);
      std::vector<int32_t> cxo(bcolptr[nrb]), cstr(nrb);
      for (int64_t r2 = 0; r2 < nrb; ++r2) {
        cstr[r2] = (int32_t)col_h[r2];
        for (int64_t k = bcolptr[r2]; k < bcolptr[r2 + 1]; ++k) {
          cbase[k] = Scolptr[boff[r2]] + brow_off[k];
          cxo[k] = boff[browval[k]];
        }
      }
      upload(P->c_ptr, cptr, s);
      upload(P->c_base, cbase, s);
      upload(P->c_xo, cxo, s);
      upload(P->c_stride, cstr, s);
      P->cols6 = true;
    }
  }
  upload(P->r_dims, dims, s);
  upload(P->boff, boff, s);
  upload(P->doff, doff, s);
  upload(P->diag_base, dbase, s);
  upload(P->diag_stride, dstride, s);
  P->D.alloc(sizeof(double) * (size_t)P->ndiag);
  P->r.alloc(sizeof(double) * nr);
  P->z.alloc(sizeof(double) * nr);
  P->p.alloc(sizeof(double) * nr);
  P->q.alloc(sizeof(double) * nr);
  P->scal.alloc(sizeof(double) * ((P->K + 1) * PS_W + 8));
  P->flags.alloc(sizeof(int) * 4 + sizeof(long long) * 2);
  BLS_CUDA(cudaMallocHost(&P->host, sizeof(double) * 8));
  BLS_CUDA(cudaStreamSynchronize(s));
  return P.release();
}

template <class T>
static void spmv(PCGPlan* P, const T* S, const double* x, const double* g, double* y, bool residual, cudaStream_t s) {
  const unsigned grid = (unsigned)grid_for(P->nrb * 32, 256);
  if (P->cols6) {   // y = 0; y += S x by block columns; r = g - y
    BLS_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * P->nr, s));
    k_spmv_cols<T><<<grid, 256, 0, s>>>(P->nrb, P->c_ptr.as<int64_t>(), P->c_base.as<int64_t>(), P->c_xo.as<int32_t>(), P->c_stride.as<int32_t>(),
                                        S, x, y, nullptr);
    P->launches += 1;
    if (residual) {
      k_from_g<<<std::max(1, grid_for(P->nr, 256)), 256, 0, s>>>(P->nr, g, y);
      P->launches += 1;
    }
    return;
  }
  if (residual)
    k_spmv<T, true, false><<<grid, 256, 0, s>>>(P->nrb, P->row_ptr.as<int64_t>(), P->rows.as<RowEntry>(), P->r_dims.as<int32_t>(),
                                                P->boff.as<int32_t>(), S, x, g, y, nullptr, nullptr);
  else
    k_spmv<T, false, false><<<grid, 256, 0, s>>>(P->nrb, P->row_ptr.as<int64_t>(), P->rows.as<RowEntry>(), P->r_dims.as<int32_t>(),
                                                 P->boff.as<int32_t>(), S, x, nullptr, y, nullptr, nullptr);
  P->launches += 1;
}

template <class T>
static void extract_diag(PCGPlan* P, const T* S, double* D, cudaStream_t s) {
  const int64_t n = P->nrb * P->max_d * P->max_d;
  k_extract_diag<T><<<grid_for(n, 256), 256, 0, s>>>(P->nrb, P->max_d, P->r_dims.as<int32_t>(), P->diag_base.as<int64_t>(),
                                                     P->diag_stride.as<int32_t>(), P->doff.as<int64_t>(), S, D);
  P->launches += 1;
}

static int64_t factor_D(PCGPlan* P, cudaStream_t s) { return pcg_factor_blocks(P, P->D.as<double>(), s); }

// The kernels of one PCG iteration on slot j
template <class T>
static void iteration(PCGPlan* P, const T* S, double* x, int j, cudaStream_t s) {
  double* slot = P->scal.as<double>() + j * PS_W;
  int* flags = P->flags.as<int>();
  const unsigned gsp = (unsigned)grid_for(P->nrb * 32, 256), gb = (unsigned)grid_for(P->nrb, 128), gv = (unsigned)grid_for(P->nr, 256);
  if (P->cols6) {
    k_spmv_cols<T><<<gsp, 256, 0, s>>>(P->nrb, P->c_ptr.as<int64_t>(), P->c_base.as<int64_t>(), P->c_xo.as<int32_t>(), P->c_stride.as<int32_t>(),
                                       S, P->p.as<double>(), P->q.as<double>(), flags);
    k_dot_pq<<<std::max(1, std::min(grid_for(P->nr, 256), 296)), 256, 0, s>>>(P->nr, P->p.as<double>(), P->q.as<double>(), slot + PS_PQ, flags);
    P->launches += 1;
  } else {
    k_spmv<T, false, true><<<gsp, 256, 0, s>>>(P->nrb, P->row_ptr.as<int64_t>(), P->rows.as<RowEntry>(), P->r_dims.as<int32_t>(),
                                               P->boff.as<int32_t>(), S, P->p.as<double>(), nullptr, P->q.as<double>(), slot + PS_PQ, flags);
  }
  k_pcg_update<<<gb, 128, 0, s>>>(P->nrb, P->r_dims.as<int32_t>(), P->boff.as<int32_t>(), P->doff.as<int64_t>(), P->D.as<double>(), P->precond, x,
                                  P->r.as<double>(), P->z.as<double>(), P->p.as<double>(), P->q.as<double>(), slot, flags, P->cols6 ? 1 : 0);
  k_pcg_direction<<<gv, 256, 0, s>>>(P->nr, P->z.as<double>(), P->p.as<double>(), slot, slot + PS_W,
                                     P->scal.as<double>() + (P->K + 1) * PS_W, flags);
  P->launches += 3;
}

// A run of n <= K iterations on slots 0..n; the carried rz enters from slot K (where the start kernel and every full run
// leave it). Only the last run of a solve may be shorter than K.
template <class T>
static void run_block(PCGPlan* P, const T* S, double* x, int n, cudaStream_t s) {
  k_pcg_slots<<<1, 32, 0, s>>>(P->scal.as<double>(), P->K);
  P->launches += 1;
  for (int j = 0; j < n; ++j) iteration<T>(P, S, x, j, s);
}

// PCG to ||g - S x|| <= tol ||g|| (FP64), block-Jacobi preconditioner in P->D (factored). Returns BLS_OK,
// BLS_NOT_CONVERGED (maxit reached) or BLS_NOT_PD (a diagonal block of S is not positive definite).
template <class T>
static int pcg_solve(PCGPlan* P, const T* S, const double* g, double* x, double tol, int64_t maxit, bool use_graph, int64_t* iters_out,
                     double* rel_out, int64_t* failed_block) {
  if (!(tol > 0) || maxit < 0) throw Error(BLS_EINVAL, "tol must be positive and maxit non-negative");
  cudaStream_t s = P->ctx->stream;
  int* flags = P->flags.as<int>();
  double* scal = P->scal.as<double>();
  double* tol2 = scal + (P->K + 1) * PS_W;
  double* gg = tol2 + 1;
  double* tr = tol2 + 2;
  // block-Jacobi: D = the diagonal blocks of S, factored
  extract_diag<T>(P, S, P->D.as<double>(), s);
  const int64_t fb = factor_D(P, s);
  if (fb >= 0) {
    if (failed_block) *failed_block = fb + 1;
    return BLS_NOT_PD;
  }
  // |g|^2 and the tolerance
  k_zero_d<<<1, 32, 0, s>>>(gg, 2);
  k_dot_self<<<std::max(1, std::min(grid_for(P->nr, 256), 296)), 256, 0, s>>>(P->nr, g, gg);
  P->launches += 2;
  BLS_CUDA(cudaMemcpyAsync(P->host, gg, sizeof(double), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  const double gnorm2 = P->host[0];
  if (gnorm2 == 0.0) {
    k_zero_d<<<grid_for(P->nr, 256), 256, 0, s>>>(x, P->nr);
    *iters_out = 0;
    *rel_out = 0.0;
    return BLS_OK;
  }
  const double t2 = tol * tol * gnorm2;
  int64_t iters = 0;
  double rel = INFINITY;
  for (int restart = 0; restart < 4; ++restart) {
    // r = g - S x; z = M^-1 r; p = z; rz into the carry slot; the tolerance
    spmv<T>(P, S, x, g, P->r.as<double>(), true, s);
    k_zero_d<<<1, 256, 0, s>>>(scal, (P->K + 1) * PS_W);
    BLS_CUDA(cudaMemcpyAsync(tol2, &t2, sizeof(double), cudaMemcpyHostToDevice, s));
    BLS_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(int), s));
    k_pcg_start<<<grid_for(P->nrb, 128), 128, 0, s>>>(P->nrb, P->r_dims.as<int32_t>(), P->boff.as<int32_t>(), P->doff.as<int64_t>(),
                                                      P->D.as<double>(), P->precond, P->r.as<double>(), P->z.as<double>(),
                                                      P->p.as<double>(), P->q.as<double>(), scal + P->K * PS_W);
    P->launches += 2;
    BLS_CUDA(cudaMemcpyAsync(P->host, scal + P->K * PS_W + PS_RRN, sizeof(double), cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaStreamSynchronize(s));
    if (!(P->host[0] > t2)) {
      rel = std::sqrt(P->host[0] / gnorm2);
      break;
    }
    int64_t done_here = 0;
    while (iters + done_here < maxit) {
      const int64_t left = maxit - iters - done_here;
      if (use_graph && left >= P->K) {
        if (!P->graph || P->graph_S != (const void*)S || P->graph_dtype != (int)sizeof(T) || P->graph_x != x || P->graph_precond != P->precond) {
          if (P->graph) {
            cudaGraphExecDestroy(P->graph);
            P->graph = nullptr;
          }
          cudaGraph_t gr;
          BLS_CUDA(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeThreadLocal));
          run_block<T>(P, S, x, P->K, P->cap_stream);
          BLS_CUDA(cudaStreamEndCapture(P->cap_stream, &gr));
          BLS_CUDA(cudaGraphInstantiate(&P->graph, gr, 0));
          cudaGraphDestroy(gr);
          P->graph_S = S;
          P->graph_x = x;
          P->graph_precond = P->precond;
          P->graph_dtype = (int)sizeof(T);
        }
        // order the graph after the work already on the context's stream, and the stream after the graph
        BLS_CUDA(cudaEventRecord(P->ev_in, s));
        BLS_CUDA(cudaStreamWaitEvent(P->cap_stream, P->ev_in, 0));
        BLS_CUDA(cudaGraphLaunch(P->graph, P->cap_stream));
        BLS_CUDA(cudaEventRecord(P->ev_out, P->cap_stream));
        BLS_CUDA(cudaStreamWaitEvent(s, P->ev_out, 0));
        P->launches += 1 + (P->cols6 ? 4 : 3) * P->K;
      } else {
        run_block<T>(P, S, x, (int)std::min<int64_t>(P->K, left), s);
      }
      BLS_CUDA(cudaMemcpyAsync(P->host + 4, flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      BLS_CUDA(cudaStreamSynchronize(s));
      const int* hf = reinterpret_cast<const int*>(P->host + 4);
      done_here = hf[1];
      if (hf[0]) break;
    }
    iters += done_here;
    // the explicit FP64 residual of the result
    spmv<T>(P, S, x, g, P->r.as<double>(), true, s);
    k_zero_d<<<1, 32, 0, s>>>(tr, 1);
    k_dot_self<<<std::max(1, std::min(grid_for(P->nr, 256), 296)), 256, 0, s>>>(P->nr, P->r.as<double>(), tr);
    P->launches += 2;
    BLS_CUDA(cudaMemcpyAsync(P->host, tr, sizeof(double), cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaStreamSynchronize(s));
    rel = std::sqrt(P->host[0] / gnorm2);
    if (rel <= tol || iters >= maxit || !std::isfinite(rel)) break;
  }
  BLS_CUDA(cudaGetLastError());
  *iters_out = iters;
  *rel_out = rel;
  return rel <= tol ? BLS_OK : BLS_NOT_CONVERGED;
}

// Mixed-precision solve refined against the FP64 reduced operator. PCG on the stored S (e.g. the FP32 reduction)
// solves for a correction d; the outer residual r = g - A x uses A x = S0 x + lambda sc_r .* x - C' E^-1 C x in FP64,
// where S0 is R on S's pattern (the reset system without damping) and the point term is applied from the reduction's
// own FP64 E^-1 (bls_schur_apply_elimination), so x converges to the solution of the system the FP64 reduction of the
// same stored inputs would give, while every PCG iteration reads only the compact S.
template <class T>
static int solve_refined(PCGPlan* P, bls_schur_plan* SP, const T* S, const T* S0, const double* sc_r, double lambda, const T* C,
                         const double* g, double* x, double tol, double inner_tol, int64_t max_outer, int64_t inner_maxit,
                         int64_t* outer_out, int64_t* inner_out, double* rel_out, int64_t* failed_block) {
  if (!(tol > 0) || !(inner_tol > 0) || max_outer < 1 || inner_maxit < 1) throw Error(BLS_EINVAL, "tolerances must be positive, iteration limits >= 1");
  if (!SP || !S || !S0 || !sc_r || !g || !x) throw Error(BLS_EINVAL, "a pointer is NULL");
  if (!(std::isfinite(lambda) && lambda >= 0)) throw Error(BLS_EINVAL, "lambda must be finite and non-negative");
  cudaStream_t s = P->ctx->stream;
  const int64_t n = P->nr;
  if (!P->ref_r.p) {
    P->ref_r.alloc(sizeof(double) * std::max<int64_t>(n, 1));
    P->ref_d.alloc(sizeof(double) * std::max<int64_t>(n, 1));
    P->ref_y.alloc(sizeof(double) * std::max<int64_t>(n, 1));
  }
  double* r = P->ref_r.as<double>();
  double* d = P->ref_d.as<double>();
  double* y = P->ref_y.as<double>();
  double* tr = P->scal.as<double>() + (P->K + 1) * PS_W + 2;
  const int gb = std::max(1, grid_for(n, 256));
  auto norm2 = [&](const double* v) {
    k_zero_d<<<1, 32, 0, s>>>(tr, 1);
    k_dot_self<<<std::max(1, std::min(grid_for(n, 256), 296)), 256, 0, s>>>(n, v, tr);
    P->launches += 2;
    BLS_CUDA(cudaMemcpyAsync(P->host, tr, sizeof(double), cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaStreamSynchronize(s));
    return P->host[0];
  };
  const int dt = sizeof(T) == 8 ? BLS_F64 : BLS_F32;
  k_zero_d<<<gb, 256, 0, s>>>(x, n);
  BLS_CUDA(cudaMemcpyAsync(r, g, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  P->launches += 1;
  const double gnorm2 = norm2(g);
  int64_t outer = 0, inner = 0;
  double rel = gnorm2 == 0.0 ? 0.0 : 1.0;
  while (rel > tol && outer < max_outer) {
    k_zero_d<<<gb, 256, 0, s>>>(d, n);
    P->launches += 1;
    int64_t its = 0, fb = 0;
    double irel = 0.0;
    const int rc = pcg_solve<T>(P, S, r, d, inner_tol, inner_maxit, true, &its, &irel, &fb);
    inner += its;
    if (rc == BLS_NOT_PD) {
      if (failed_block) *failed_block = fb;
      *outer_out = outer;
      *inner_out = inner;
      *rel_out = rel;
      return BLS_NOT_PD;
    }
    ++outer;
    k_add<<<gb, 256, 0, s>>>(n, x, d);
    // y = S0 x + lambda sc_r .* x - C' E^-1 C x; r = g - y
    spmv<T>(P, S0, x, nullptr, y, false, s);
    k_add_damping<<<gb, 256, 0, s>>>(n, y, lambda, sc_r, x);
    P->launches += 2;
    const int arc = bls_schur_apply_elimination(SP, dt, d, y, x, C);   // d is free once added into x
    if (arc != BLS_OK) throw Error(arc, bls_last_error());
    k_residual<<<gb, 256, 0, s>>>(n, r, g, d);
    P->launches += 1;
    rel = std::sqrt(norm2(r) / gnorm2);
    if (!std::isfinite(rel)) break;
  }
  BLS_CUDA(cudaGetLastError());
  *outer_out = outer;
  *inner_out = inner;
  *rel_out = rel;
  return rel <= tol ? BLS_OK : BLS_NOT_CONVERGED;
}

void pcg_spmv(PCGPlan* P, int dtype, const void* S, const double* x, const double* g, double* y, bool residual, cudaStream_t s) {
  if (dtype == BLS_F64) spmv<double>(P, (const double*)S, x, g, y, residual, s);
  else spmv<float>(P, (const float*)S, x, g, y, residual, s);
}

void pcg_extract_diag(PCGPlan* P, int dtype, const void* S, double* D, cudaStream_t s) {
  if (dtype == BLS_F64) extract_diag<double>(P, (const double*)S, D, s);
  else extract_diag<float>(P, (const float*)S, D, s);
}

int64_t pcg_factor_blocks(PCGPlan* P, double* D, cudaStream_t s) {
  long long* failed = reinterpret_cast<long long*>(P->flags.as<int>() + 4);
  const long long none = LLONG_MAX;
  BLS_CUDA(cudaMemcpyAsync(failed, &none, sizeof(long long), cudaMemcpyHostToDevice, s));
  k_factor_blocks<double><<<grid_for(P->nrb, 128), 128, 0, s>>>(P->nrb, P->r_dims.as<int32_t>(), P->doff.as<int64_t>(), D, failed);
  P->launches += 1;
  long long h = 0;
  BLS_CUDA(cudaMemcpyAsync(&h, failed, sizeof(long long), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  return h == none ? -1 : (int64_t)h;
}

}  // namespace bls

struct bls_pcg_plan : bls::PCGPlan {};
using namespace bls;

#define PCG_GUARD(...)                        \
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

int bls_pcg_plan_create(bls_ctx* ctx, int64_t nrblocks, const int64_t* r_dims, const int64_t* block_colptr, const int64_t* block_rowval,
                        const int64_t* block_row_offsets, const int64_t* col_heights, const int64_t* S_colptr, bls_pcg_plan** out) {
  PCG_GUARD({
    if (!ctx || !out) throw Error(BLS_EINVAL, "null argument");
    BLS_CUDA(cudaSetDevice(ctx->device));
    PCGPlan* P = pcg_plan_create(ctx, nrblocks, r_dims, block_colptr, block_rowval, block_row_offsets, col_heights, S_colptr);
    cudaError_t e1 = cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking);
    cudaError_t e2 = cudaEventCreateWithFlags(&P->ev_in, cudaEventDisableTiming);
    cudaError_t e3 = cudaEventCreateWithFlags(&P->ev_out, cudaEventDisableTiming);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      delete P;
      throw Error(BLS_ECUDA, "could not create the PCG plan's stream and events");
    }
    *out = static_cast<bls_pcg_plan*>(P);
    return BLS_OK;
  })
}

int bls_pcg_plan_destroy(bls_pcg_plan* P) {
  if (P) {
    cudaStreamSynchronize(P->ctx->stream);
    delete static_cast<PCGPlan*>(P);
  }
  return BLS_OK;
}

int bls_spmv_sym(bls_pcg_plan* P, int dtype, const void* S, const double* x, double* y) {
  PCG_GUARD({
    if (!P) throw Error(BLS_EINVAL, "null argument");
    if (dtype == BLS_F64) spmv<double>(P, (const double*)S, x, nullptr, y, false, P->ctx->stream);
    else if (dtype == BLS_F32) spmv<float>(P, (const float*)S, x, nullptr, y, false, P->ctx->stream);
    else throw Error(BLS_EINVAL, "unknown dtype");
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

int bls_extract_diagonal_blocks(bls_pcg_plan* P, int dtype, const void* S, double* D) {
  PCG_GUARD({
    if (!P) throw Error(BLS_EINVAL, "null argument");
    if (dtype == BLS_F64) extract_diag<double>(P, (const double*)S, D, P->ctx->stream);
    else if (dtype == BLS_F32) extract_diag<float>(P, (const float*)S, D, P->ctx->stream);
    else throw Error(BLS_EINVAL, "unknown dtype");
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

int bls_pcg_solve(bls_pcg_plan* P, int dtype, const void* S, const double* g, double* x, double tol, int64_t maxit, int use_graph,
                  int64_t* iterations, double* rel_residual, int64_t* failed_block) {
  PCG_GUARD({
    if (!P || !iterations || !rel_residual) throw Error(BLS_EINVAL, "null argument");
    if (failed_block) *failed_block = 0;
    if (dtype == BLS_F64)
      return pcg_solve<double>(P, (const double*)S, g, x, tol, maxit, use_graph != 0, iterations, rel_residual, failed_block);
    if (dtype == BLS_F32)
      return pcg_solve<float>(P, (const float*)S, g, x, tol, maxit, use_graph != 0, iterations, rel_residual, failed_block);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_pcg_solve_refined(bls_pcg_plan* P, bls_schur_plan* schur, int dtype, const void* S, const void* S0, const double* scaling_r,
                          double lambda, const void* C, const double* g, double* x, double tol, double inner_tol, int64_t max_outer,
                          int64_t inner_maxit, int64_t* outer_iterations, int64_t* inner_iterations, double* rel_residual,
                          int64_t* failed_block) {
  PCG_GUARD({
    if (!P || !outer_iterations || !inner_iterations || !rel_residual) throw Error(BLS_EINVAL, "null argument");
    if (failed_block) *failed_block = 0;
    if (dtype == BLS_F64)
      return solve_refined<double>(P, schur, (const double*)S, (const double*)S0, scaling_r, lambda, (const double*)C, g, x, tol, inner_tol,
                                   max_outer, inner_maxit, outer_iterations, inner_iterations, rel_residual, failed_block);
    if (dtype == BLS_F32)
      return solve_refined<float>(P, schur, (const float*)S, (const float*)S0, scaling_r, lambda, (const float*)C, g, x, tol, inner_tol,
                                  max_outer, inner_maxit, outer_iterations, inner_iterations, rel_residual, failed_block);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_pcg_set_preconditioner(bls_pcg_plan* P, const double* blocks) {
  if (!P) return BLS_EINVAL;
  P->precond = blocks;
  return BLS_OK;
}

int64_t bls_pcg_plan_counters(bls_pcg_plan* P) {
  if (!P) return -1;
  const int64_t n = P->launches;
  P->launches = 0;
  return n;
}

// ---- block-Jacobi on a flat array of diagonal blocks (src/diagonal_blocks.jl:6-61) ----

struct bls_block_jacobi {
  bls_ctx* ctx = nullptr;
  int64_t nb = 0;
  DevBuf dims, doff, voff, failed;
  long long* host = nullptr;
  ~bls_block_jacobi() { if (host) cudaFreeHost(host); }
};

int bls_block_jacobi_create(bls_ctx* ctx, int64_t nb, const int64_t* dims, bls_block_jacobi** out) {
  PCG_GUARD({
    if (!ctx || !out || nb < 0 || (nb > 0 && !dims)) throw Error(BLS_EINVAL, "null argument");
    std::unique_ptr<bls_block_jacobi> J(new bls_block_jacobi());
    J->ctx = ctx;
    J->nb = nb;
    std::vector<int32_t> d(nb);
    std::vector<int64_t> doff(nb + 1, 0), voff(nb + 1, 0);
    for (int64_t b = 0; b < nb; ++b) {
      if (dims[b] < 1 || dims[b] > 16) throw Error(BLS_EUNSUPPORTED, "block sizes above 16 are not supported on the device");
      d[b] = (int32_t)dims[b];
      doff[b + 1] = doff[b] + dims[b] * dims[b];
      voff[b + 1] = voff[b] + dims[b];
    }
    upload(J->dims, d, ctx->stream);
    upload(J->doff, doff, ctx->stream);
    upload(J->voff, voff, ctx->stream);
    J->failed.alloc(sizeof(long long));
    BLS_CUDA(cudaMallocHost(&J->host, sizeof(long long)));
    BLS_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = J.release();
    return BLS_OK;
  })
}

int bls_block_jacobi_destroy(bls_block_jacobi* J) {
  if (J) {
    cudaStreamSynchronize(J->ctx->stream);
    delete J;
  }
  return BLS_OK;
}

int bls_factor_diagonal_blocks(bls_block_jacobi* J, int dtype, void* D, int64_t* failed_block) {
  PCG_GUARD({
    if (!J || !failed_block) throw Error(BLS_EINVAL, "null argument");
    cudaStream_t s = J->ctx->stream;
    const long long none = LLONG_MAX;
    BLS_CUDA(cudaMemcpyAsync(J->failed.p, &none, sizeof(long long), cudaMemcpyHostToDevice, s));
    if (J->nb > 0) {
      if (dtype == BLS_F64)
        k_factor_blocks<double><<<grid_for(J->nb, 128), 128, 0, s>>>(J->nb, J->dims.as<int32_t>(), J->doff.as<int64_t>(), (double*)D,
                                                                      J->failed.as<long long>());
      else if (dtype == BLS_F32)
        k_factor_blocks<float><<<grid_for(J->nb, 128), 128, 0, s>>>(J->nb, J->dims.as<int32_t>(), J->doff.as<int64_t>(), (float*)D,
                                                                     J->failed.as<long long>());
      else throw Error(BLS_EINVAL, "unknown dtype");
    }
    BLS_CUDA(cudaMemcpyAsync(J->host, J->failed.p, sizeof(long long), cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaStreamSynchronize(s));
    *failed_block = J->host[0] == none ? 0 : (int64_t)J->host[0] + 1;
    return J->host[0] == none ? BLS_OK : BLS_NOT_PD;
  })
}

int bls_solve_diagonal_blocks(bls_block_jacobi* J, int dtype, double* y, const void* D, const double* x) {
  PCG_GUARD({
    if (!J) throw Error(BLS_EINVAL, "null argument");
    cudaStream_t s = J->ctx->stream;
    if (J->nb == 0) return BLS_OK;
    if (dtype == BLS_F64)
      k_solve_blocks<double><<<grid_for(J->nb, 128), 128, 0, s>>>(J->nb, J->dims.as<int32_t>(), J->doff.as<int64_t>(), J->voff.as<int64_t>(),
                                                                  (const double*)D, x, y);
    else if (dtype == BLS_F32)
      k_solve_blocks<float><<<grid_for(J->nb, 128), 128, 0, s>>>(J->nb, J->dims.as<int32_t>(), J->doff.as<int64_t>(), J->voff.as<int64_t>(),
                                                                 (const float*)D, x, y);
    else throw Error(BLS_EINVAL, "unknown dtype");
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

}  // extern "C"
