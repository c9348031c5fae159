// A learned correction to the 6x6 block-Jacobi preconditioner of PCG on the reduced system (no counterpart in the
// reference): a graph network over the camera covisibility graph (the block pattern of S), trained and run with the
// kernels of this file.
//
// Graph. Nodes are the retained (camera) blocks, edges the stored off-diagonal blocks S_bc. With L_b the Cholesky
// factor of S_bb, the normalised coupling is E_bc = L_b^-1 S_bc L_c^-T (the off-diagonal blocks of the block-Jacobi-
// preconditioned matrix S^ = L^-1 S L^-T). Edge weight a_bc = ||E_bc||_F; node features (8): log(1 + e_b,i) for the six
// row energies e_b,i = sum over neighbours and columns of E_bc(i, j)^2, log(1 + sum_i e_b,i), log(1 + degree) / 4.
//
// Network (width 64): h0 = relu(W_in f + b_in); three layers h_l = relu(W_s,l h_(l-1) + W_m,l m_(l-1) + b_l) with
// m_b = sum_c (a_bc / sum_c' a_bc') h_c; t = W_out h3 + b_out (21 values). T_b = the lower triangle (row-major order
// (0,0), (1,0), (1,1), (2,0) ...) of t_b, G_b = I + T_b, and the preconditioner block is
// B_b = L_b^-T G_b' G_b L_b^-1 (symmetric positive definite for any finite T with G_b nonsingular; T = 0 is block-Jacobi).
//
// Loss (training): with M = G S^ G' and probes z, L = Z N2 / N1^2 where N1 = sum z'Mz, N2 = sum |Mz|^2,
// Z = sum |z|^2: an estimate of n sum(lambda^2) / (sum lambda)^2 over M's spectrum, 1 when the spectrum is one point and
// blind to a uniform scaling of the preconditioner (as CG is). With w = S^ G' z, y = G w and s = S^ G' y,
// dL/dG = (Z / N1^2) (2 sum (y w' + z s') - 4 (N2 / N1) sum z w'); S^ is applied as L^-1 (S (L^-T x)) with the PCG
// plan's y = S x.
//
// Precision: training runs the network in FP32; inference stores activations and weights in BF16 and accumulates in
// FP32. The linear algebra around it (L, S^, B) is FP64.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <type_traits>
#include <vector>

#include "pcg_plan.hpp"

namespace bls {

constexpr int GNN_F = 8, GNN_H = 64, GNN_T = 21, GNN_LAYERS = 3;
constexpr int GNN_OFF_WIN = 0, GNN_OFF_BIN = GNN_H * GNN_F;
constexpr int GNN_OFF_L0 = GNN_OFF_BIN + GNN_H, GNN_LSTRIDE = 2 * GNN_H * GNN_H + GNN_H;
constexpr int GNN_OFF_WOUT = GNN_OFF_L0 + GNN_LAYERS * GNN_LSTRIDE, GNN_OFF_BOUT = GNN_OFF_WOUT + GNN_T * GNN_H;
constexpr int GNN_NPARAMS = GNN_OFF_BOUT + GNN_T;

struct GNNPlan {
  PCGPlan* pcg = nullptr;
  int64_t n = 0, nedges = 0, nnb = 0;
  DevBuf e_b, e_c, e_base, e_stride, e_norm;   // edges (b < c)
  DevBuf nb_ptr, nb_other, nb_edge, w_fwd, w_rev;
  DevBuf energy, feat, asum, L, t, B;
  DevBuf h[GNN_LAYERS + 1], m[GNN_LAYERS];     // activations (FP32 or BF16)
  DevBuf dt, dh, dh2, dm, grad_tmp;            // backward scratch
  DevBuf y, yh, w, v, s, u, loss, accA, accB;  // loss vectors (FP64) and the two gradient accumulators
  bool prepared = false;
};

// ---------------------------------------------------------------------------------------------------------------
// Small dense helpers on 6 x 6 FP64 blocks (column-major, lower-triangular L)
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void lower_solve6(const double* __restrict__ L, double* x) {   // x = L^-1 x
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    x[j] /= L[j * 6 + j];
#pragma unroll
    for (int i = j + 1; i < 6; ++i) x[i] -= L[j * 6 + i] * x[j];
  }
}
__device__ __forceinline__ void upper_solve6(const double* __restrict__ L, double* x) {   // x = L^-T x
#pragma unroll
  for (int j = 5; j >= 0; --j) {
    double t = x[j];
#pragma unroll
    for (int i = j + 1; i < 6; ++i) t -= L[j * 6 + i] * x[i];
    x[j] = t / L[j * 6 + j];
  }
}
// G = I + T from the 21 lower-triangle values (row-major order)
__device__ __forceinline__ void make_G(const float* __restrict__ t, double (&G)[6][6]) {
  int q = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      if (j <= i) G[i][j] = (double)t[q++] + (i == j ? 1.0 : 0.0);
      else G[i][j] = 0.0;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Graph features
// ---------------------------------------------------------------------------------------------------------------
template <class T>
__global__ void k_gnn_edges(int64_t ne, const int32_t* __restrict__ eb, const int32_t* __restrict__ ec, const int64_t* __restrict__ ebase,
                            const int32_t* __restrict__ estride, const double* __restrict__ L, const T* __restrict__ S,
                            double* __restrict__ enorm, double* __restrict__ energy) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int b = eb[e], c = ec[e];
  const T* Bm = S + ebase[e];
  const int64_t st = estride[e];
  const double* Lb = L + 36 * (int64_t)b;
  const double* Lc = L + 36 * (int64_t)c;
  double X[6][6];   // X[i][j]: row i, column j
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double col[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) col[i] = (double)Bm[i + j * st];
    lower_solve6(Lb, col);
#pragma unroll
    for (int i = 0; i < 6; ++i) X[i][j] = col[i];
  }
  double rowE[6], colE[6] = {0, 0, 0, 0, 0, 0}, tot = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double row[6];
#pragma unroll
    for (int j = 0; j < 6; ++j) row[j] = X[i][j];
    lower_solve6(Lc, row);   // (L_c^-1 X(i,:)')' = X(i,:) L_c^-T
    double r2 = 0.0;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const double v2 = row[j] * row[j];
      r2 += v2;
      colE[j] += v2;
    }
    rowE[i] = r2;
    tot += r2;
  }
  enorm[e] = sqrt(tot);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    atomicAdd(energy + 6 * (int64_t)b + i, rowE[i]);
    atomicAdd(energy + 6 * (int64_t)c + i, colE[i]);
  }
}

__global__ void k_gnn_nodes(int64_t n, const int64_t* __restrict__ nb_ptr, const int32_t* __restrict__ nb_edge, const double* __restrict__ enorm,
                            const double* __restrict__ energy, double* __restrict__ asum, float* __restrict__ feat) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= n) return;
  double a = 0.0, tot = 0.0;
  for (int64_t q = nb_ptr[b]; q < nb_ptr[b + 1]; ++q) a += enorm[nb_edge[q]];
  asum[b] = a;
  float* f = feat + GNN_F * b;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const double e = energy[6 * b + i];
    tot += e;
    f[i] = (float)log1p(e);
  }
  f[6] = (float)log1p(tot);
  f[7] = (float)(log1p((double)(nb_ptr[b + 1] - nb_ptr[b])) * 0.25);
}

__global__ void k_gnn_weights(int64_t n, const int64_t* __restrict__ nb_ptr, const int32_t* __restrict__ nb_other, const int32_t* __restrict__ nb_edge,
                              const double* __restrict__ enorm, const double* __restrict__ asum, float* __restrict__ wf, float* __restrict__ wr) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= n) return;
  const double ab = asum[b];
  for (int64_t q = nb_ptr[b]; q < nb_ptr[b + 1]; ++q) {
    const double a = enorm[nb_edge[q]];
    const double ac = asum[nb_other[q]];
    wf[q] = ab > 0 ? (float)(a / ab) : 0.f;   // weight of neighbour c in b's mean
    wr[q] = ac > 0 ? (float)(a / ac) : 0.f;   // weight of b in neighbour c's mean (for the backward pass)
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Network kernels: activations of type A (float or BF16), FP32 accumulation, FP32 parameters (rounded to A on load)
// ---------------------------------------------------------------------------------------------------------------
template <class A> __device__ __forceinline__ float to_f(A x);
template <> __device__ __forceinline__ float to_f<float>(float x) { return x; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }
template <class A> __device__ __forceinline__ A from_f(float x);
template <> __device__ __forceinline__ float from_f<float>(float x) { return x; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float x) { return __float2bfloat16(x); }

// out[b, o] = act(bias[o] + W1[o, :] in1[b, :] + W2[o, :] in2[b, :]); one thread per (node, output); weights in shared
// memory, rounded to A. in1 has K1 columns, in2 (optional) K2. Output to A (outA) or FP32 (outF).
template <class A, class IN1>
__global__ void __launch_bounds__(256) k_lin_fwd(int64_t n, int K1, const IN1* __restrict__ in1, int K2, const A* __restrict__ in2,
                                                 const float* __restrict__ W1, const float* __restrict__ W2, const float* __restrict__ bias, int O,
                                                 bool relu, A* __restrict__ outA, float* __restrict__ outF) {
  extern __shared__ float wsm[];
  const int K = K1 + K2;
  for (int i = threadIdx.x; i < O * K; i += blockDim.x) {
    const int o = i / K, k = i - o * K;
    const float wv = k < K1 ? W1[o * K1 + k] : W2[o * K2 + (k - K1)];
    wsm[i] = to_f<A>(from_f<A>(wv));
  }
  __syncthreads();
  const int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t b = id / O;
  const int o = (int)(id - b * O);
  if (b >= n) return;
  float acc = bias[o];
  const float* w = wsm + o * K;
  for (int k = 0; k < K1; ++k) acc += w[k] * to_f<A>(from_f<A>((float)in1[b * K1 + k]));
  for (int k = 0; k < K2; ++k) acc += w[K1 + k] * to_f<A>(in2[b * K2 + k]);
  if (relu) acc = fmaxf(acc, 0.f);
  if (outA) outA[b * O + o] = from_f<A>(acc);
  if (outF) outF[b * O + o] = acc;
}

// The BF16 inference form of k_lin_fwd on the tensor cores: out[b, :] = act(bias + [in1 in2][b, :] W'), BF16 operands
// and FP32 accumulation by mma.sync m16n8k16; a warp per 16 nodes, the layer's weights rounded to BF16 in shared memory
// (O padded to a multiple of 8, row o = column o of the B operand). Needs K1 and K2 multiples of 16, K1 + K2 <= 128,
// O <= 64.
__device__ __forceinline__ void mma_bf16_16816(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
constexpr int LIN_MMA_KMAX = 128, LIN_MMA_OMAX = 64;
__global__ void __launch_bounds__(128) k_lin_mma(int64_t n, int K1, const __nv_bfloat16* __restrict__ in1, int K2,
                                                 const __nv_bfloat16* __restrict__ in2, const float* __restrict__ W1,
                                                 const float* __restrict__ W2, const float* __restrict__ bias, int O, bool relu,
                                                 __nv_bfloat16* __restrict__ outA, float* __restrict__ outF) {
  __shared__ __align__(16) __nv_bfloat16 wsm[LIN_MMA_OMAX * LIN_MMA_KMAX];
  __shared__ float bsm[LIN_MMA_OMAX];
  const int K = K1 + K2, NT8 = (O + 7) / 8;
  for (int i = threadIdx.x; i < NT8 * 8 * K; i += blockDim.x) {
    const int o = i / K, k = i - o * K;
    const float wv = o >= O ? 0.f : (k < K1 ? W1[o * K1 + k] : W2[o * K2 + (k - K1)]);
    wsm[i] = __float2bfloat16(wv);
  }
  for (int o = threadIdx.x; o < LIN_MMA_OMAX; o += blockDim.x) bsm[o] = o < O ? bias[o] : 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int64_t r0 = ((int64_t)blockIdx.x * (blockDim.x >> 5) + warp) * 16;
  if (r0 >= n) return;
  const int64_t ra = r0 + g, rb = r0 + g + 8;
  // two BF16 entries (columns k, k + 1) of row r of [in1 in2]; zero past the last node
  auto ld2 = [&](int64_t r, int k) -> uint32_t {
    if (r >= n) return 0u;
    const __nv_bfloat16* src = k < K1 ? in1 + r * K1 + k : in2 + r * K2 + (k - K1);
    return *reinterpret_cast<const uint32_t*>(src);
  };
  float acc[LIN_MMA_OMAX / 8][4];
#pragma unroll
  for (int j = 0; j < LIN_MMA_OMAX / 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  for (int kk = 0; kk < K; kk += 16) {
    const uint32_t a0 = ld2(ra, kk + 2 * t), a1 = ld2(rb, kk + 2 * t), a2 = ld2(ra, kk + 8 + 2 * t), a3 = ld2(rb, kk + 8 + 2 * t);
#pragma unroll
    for (int j = 0; j < LIN_MMA_OMAX / 8; ++j)
      if (j < NT8) {
        const __nv_bfloat16* wb = wsm + (j * 8 + g) * K + kk + 2 * t;
        mma_bf16_16816(acc[j], a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(wb), *reinterpret_cast<const uint32_t*>(wb + 8));
      }
  }
#pragma unroll
  for (int j = 0; j < LIN_MMA_OMAX / 8; ++j)
    if (j < NT8) {
      const int c = j * 8 + 2 * t;
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const int64_t r = h < 2 ? ra : rb;
        const int o = c + (h & 1);
        if (r >= n || o >= O) continue;
        float v = acc[j][h] + bsm[o];
        if (relu) v = fmaxf(v, 0.f);
        if (outA) outA[r * O + o] = __float2bfloat16(v);
        if (outF) outF[r * O + o] = v;
      }
    }
}

// m[b, :] = sum_q w[q] h[other_q, :]; one warp per node, two channels per lane
template <class A>
__global__ void k_gnn_agg(int64_t n, const int64_t* __restrict__ nb_ptr, const int32_t* __restrict__ nb_other, const float* __restrict__ w,
                          const A* __restrict__ h, A* __restrict__ m) {
  const int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (b >= n) return;
  float a0 = 0.f, a1 = 0.f;
  for (int64_t q = nb_ptr[b]; q < nb_ptr[b + 1]; ++q) {
    const float wq = w[q];
    const A* hc = h + (int64_t)nb_other[q] * GNN_H;
    a0 += wq * to_f<A>(hc[lane]);
    a1 += wq * to_f<A>(hc[lane + 32]);
  }
  m[b * GNN_H + lane] = from_f<A>(a0);
  m[b * GNN_H + lane + 32] = from_f<A>(a1);
}

// Backward of k_lin_fwd (FP32): dpre = dout * (out > 0 when relu); din1[b, k] = sum_o W1[o, k] dpre[b, o] (written),
// din2 likewise (written)
__global__ void __launch_bounds__(256) k_lin_bwd_data(int64_t n, int O, const float* __restrict__ dout, const float* __restrict__ out, bool relu,
                                                      int K1, const float* __restrict__ W1, float* __restrict__ din1, int K2,
                                                      const float* __restrict__ W2, float* __restrict__ din2) {
  const int K = K1 + K2;
  const int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t b = id / K;
  const int k = (int)(id - b * K);
  if (b >= n) return;
  float acc = 0.f;
  for (int o = 0; o < O; ++o) {
    float d = dout[b * O + o];
    if (relu && !(out[b * O + o] > 0.f)) d = 0.f;
    acc += (k < K1 ? W1[o * K1 + k] : W2[o * K2 + (k - K1)]) * d;
  }
  if (k < K1) din1[b * K1 + k] = acc;
  else din2[b * K2 + (k - K1)] = acc;
}

// dW1[o, k] += sum_b dpre[b, o] in1[b, k], dW2 likewise, db[o] += sum_b dpre[b, o]; thread per (o, k), nodes split
// over gridDim.y chunks
__global__ void __launch_bounds__(256) k_lin_bwd_weight(int64_t n, int O, const float* __restrict__ dout, const float* __restrict__ out, bool relu,
                                                        int K1, const float* __restrict__ in1, int K2, const float* __restrict__ in2,
                                                        float* __restrict__ dW1, float* __restrict__ dW2, float* __restrict__ db) {
  const int K = K1 + K2 + 1;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= O * K) return;
  const int o = id / K, k = id - o * K;
  const int64_t chunk = (n + gridDim.y - 1) / gridDim.y;
  const int64_t b0 = blockIdx.y * chunk, b1 = min(n, b0 + chunk);
  float acc = 0.f;
  for (int64_t b = b0; b < b1; ++b) {
    float d = dout[b * O + o];
    if (relu && !(out[b * O + o] > 0.f)) d = 0.f;
    const float x = k < K1 ? in1[b * K1 + k] : (k < K1 + K2 ? in2[b * K2 + (k - K1)] : 1.f);
    acc += d * x;
  }
  if (acc == 0.f) return;
  if (k < K1) atomicAdd(dW1 + o * K1 + k, acc);
  else if (k < K1 + K2) atomicAdd(dW2 + o * K2 + (k - K1), acc);
  else atomicAdd(db + o, acc);
}

// dh[c, :] += sum over c's neighbours b of (a_bc / A_b) dm[b, :]
__global__ void k_gnn_agg_bwd(int64_t n, const int64_t* __restrict__ nb_ptr, const int32_t* __restrict__ nb_other, const float* __restrict__ wr,
                              const float* __restrict__ dm, float* __restrict__ dh) {
  const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= n) return;
  float a0 = 0.f, a1 = 0.f;
  for (int64_t q = nb_ptr[c]; q < nb_ptr[c + 1]; ++q) {
    const float wq = wr[q];
    const float* d = dm + (int64_t)nb_other[q] * GNN_H;
    a0 += wq * d[lane];
    a1 += wq * d[lane + 32];
  }
  dh[c * GNN_H + lane] += a0;
  dh[c * GNN_H + lane + 32] += a1;
}

// ---------------------------------------------------------------------------------------------------------------
// Preconditioner blocks and the loss
// ---------------------------------------------------------------------------------------------------------------
// B_b = C' C with C = G_b L_b^-1 (FP64)
__global__ void k_gnn_precond(int64_t n, const float* __restrict__ t, const double* __restrict__ L, double* __restrict__ B) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= n) return;
  double G[6][6];
  make_G(t + GNN_T * b, G);
  const double* Lb = L + 36 * b;
  double C[6][6];   // C' column j = L^-T (row j of G)'
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double x[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) x[i] = G[j][i];
    upper_solve6(Lb, x);
#pragma unroll
    for (int i = 0; i < 6; ++i) C[j][i] = x[i];   // C[j][i] = (G L^-1)(j, i)
  }
  double* out = B + 36 * b;
#pragma unroll
  for (int c = 0; c < 6; ++c)
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) acc += C[k][r] * C[k][c];
      out[c * 6 + r] = acc;
    }
}

// Block operations of the loss (thread per node): op 0: out = G' in; 1: out = L^-T in; 2: out = L^-1 in;
// 3: out = G in, with sum(out . in2) into acc[0] and sum(out . out) into acc[1]
__global__ void k_gnn_block(int64_t n, int op, const float* __restrict__ t, const double* __restrict__ L, const double* __restrict__ in,
                            const double* __restrict__ in2, double* __restrict__ out, double* __restrict__ acc) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double part = 0.0, part2 = 0.0;
  if (b < n) {
    double x[6], y[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) x[i] = in[6 * b + i];
    if (op == 1) {
      upper_solve6(L + 36 * b, x);
#pragma unroll
      for (int i = 0; i < 6; ++i) y[i] = x[i];
    } else if (op == 2) {
      lower_solve6(L + 36 * b, x);
#pragma unroll
      for (int i = 0; i < 6; ++i) y[i] = x[i];
    } else {
      double G[6][6];
      make_G(t + GNN_T * b, G);
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) s += (op == 0 ? G[j][i] : G[i][j]) * x[j];
        y[i] = s;
      }
      if (op == 3)
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          part += y[i] * in2[6 * b + i];
          part2 += y[i] * y[i];
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) out[6 * b + i] = y[i];
  }
  if (op == 3) {
    for (int o = 16; o > 0; o >>= 1) {
      part += __shfl_xor_sync(0xffffffffu, part, o);
      part2 += __shfl_xor_sync(0xffffffffu, part2, o);
    }
    if ((threadIdx.x & 31) == 0) {
      if (part != 0.0) atomicAdd(acc, part);
      if (part2 != 0.0) atomicAdd(acc + 1, part2);
    }
  }
}

// acc_b += lower(a_b c_b' + e_b f_b') (e, f may be null), FP64 accumulators of 21 per node
__global__ void k_gnn_outer(int64_t n, const double* __restrict__ a, const double* __restrict__ c, const double* __restrict__ e,
                            const double* __restrict__ f, double* __restrict__ acc) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= n) return;
  int q = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) {
      double g = a[6 * b + i] * c[6 * b + j];
      if (e) g += e[6 * b + i] * f[6 * b + j];
      acc[GNN_T * b + q] += g;
      ++q;
    }
}

// dt = ca * A + cb * B (FP32 result)
__global__ void k_gnn_combine(int64_t m, double ca, const double* __restrict__ A, double cb, const double* __restrict__ B, float* __restrict__ dt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) dt[i] = (float)(ca * A[i] + cb * B[i]);
}

__global__ void k_dot_sq(int64_t n, const double* __restrict__ v, double* __restrict__ out) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) s += v[i] * v[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(out, s);
}

__global__ void k_adam(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ---------------------------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------------------------
static GNNPlan* gnn_create(PCGPlan* P, const int64_t* bcolptr, const int64_t* browval, const int64_t* brow_off, const int64_t* col_h,
                           const int64_t* Scolptr) {
  std::unique_ptr<GNNPlan> G(new GNNPlan());
  G->pcg = P;
  const int64_t n = P->nrb;
  G->n = n;
  std::vector<int32_t> eb, ec, est;
  std::vector<int64_t> ebase;
  std::vector<std::vector<std::pair<int32_t, int32_t>>> nb(n);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t k = bcolptr[c]; k < bcolptr[c + 1]; ++k) {
      const int64_t b = browval[k];
      if (b == c) continue;
      const int32_t e = (int32_t)eb.size();
      eb.push_back((int32_t)b);
      ec.push_back((int32_t)c);
      ebase.push_back(Scolptr[6 * c] + brow_off[k]);
      est.push_back((int32_t)col_h[c]);
      nb[b].push_back({(int32_t)c, e});
      nb[c].push_back({(int32_t)b, e});
    }
  G->nedges = (int64_t)eb.size();
  std::vector<int64_t> nptr(n + 1, 0);
  std::vector<int32_t> nother, nedge;
  for (int64_t b = 0; b < n; ++b) {
    for (auto& x : nb[b]) { nother.push_back(x.first); nedge.push_back(x.second); }
    nptr[b + 1] = (int64_t)nother.size();
  }
  G->nnb = (int64_t)nother.size();
  cudaStream_t s = P->ctx->stream;
  upload(G->e_b, eb, s); upload(G->e_c, ec, s); upload(G->e_base, ebase, s); upload(G->e_stride, est, s);
  upload(G->nb_ptr, nptr, s); upload(G->nb_other, nother, s); upload(G->nb_edge, nedge, s);
  G->e_norm.alloc(sizeof(double) * std::max<int64_t>(1, G->nedges));
  G->w_fwd.alloc(sizeof(float) * std::max<int64_t>(1, G->nnb));
  G->w_rev.alloc(sizeof(float) * std::max<int64_t>(1, G->nnb));
  G->energy.alloc(sizeof(double) * 6 * n);
  G->feat.alloc(sizeof(float) * GNN_F * n);
  G->asum.alloc(sizeof(double) * n);
  G->L.alloc(sizeof(double) * 36 * n);
  G->t.alloc(sizeof(float) * GNN_T * n);
  G->B.alloc(sizeof(double) * 36 * n);
  for (int l = 0; l <= GNN_LAYERS; ++l) G->h[l].alloc(sizeof(float) * GNN_H * n);
  for (int l = 0; l < GNN_LAYERS; ++l) G->m[l].alloc(sizeof(float) * GNN_H * n);
  G->dt.alloc(sizeof(float) * GNN_T * n);
  G->dh.alloc(sizeof(float) * GNN_H * n);
  G->dh2.alloc(sizeof(float) * GNN_H * n);
  G->dm.alloc(sizeof(float) * GNN_H * n);
  G->grad_tmp.alloc(sizeof(float) * GNN_F * n);
  for (DevBuf* v : {&G->y, &G->yh, &G->w, &G->v, &G->s, &G->u}) v->alloc(sizeof(double) * 6 * n);
  G->loss.alloc(sizeof(double) * 4);
  G->accA.alloc(sizeof(double) * GNN_T * n);
  G->accB.alloc(sizeof(double) * GNN_T * n);
  BLS_CUDA(cudaStreamSynchronize(s));
  return G.release();
}

// Features of the graph of S: L (the block-Jacobi factors), edge weights, node features. Returns the lowest diagonal
// block (0-based) that is not positive definite, or -1.
static int64_t gnn_prepare(GNNPlan* G, int dtype, const void* S) {
  PCGPlan* P = G->pcg;
  cudaStream_t s = P->ctx->stream;
  pcg_extract_diag(P, dtype, S, G->L.as<double>(), s);
  const int64_t fb = pcg_factor_blocks(P, G->L.as<double>(), s);
  if (fb >= 0) return fb;
  BLS_CUDA(cudaMemsetAsync(G->energy.p, 0, G->energy.bytes, s));
  if (G->nedges > 0) {
    if (dtype == BLS_F64)
      k_gnn_edges<double><<<grid_for(G->nedges, 128), 128, 0, s>>>(G->nedges, G->e_b.as<int32_t>(), G->e_c.as<int32_t>(), G->e_base.as<int64_t>(),
                                                                   G->e_stride.as<int32_t>(), G->L.as<double>(), (const double*)S,
                                                                   G->e_norm.as<double>(), G->energy.as<double>());
    else
      k_gnn_edges<float><<<grid_for(G->nedges, 128), 128, 0, s>>>(G->nedges, G->e_b.as<int32_t>(), G->e_c.as<int32_t>(), G->e_base.as<int64_t>(),
                                                                  G->e_stride.as<int32_t>(), G->L.as<double>(), (const float*)S,
                                                                  G->e_norm.as<double>(), G->energy.as<double>());
  }
  k_gnn_nodes<<<grid_for(G->n, 128), 128, 0, s>>>(G->n, G->nb_ptr.as<int64_t>(), G->nb_edge.as<int32_t>(), G->e_norm.as<double>(),
                                                  G->energy.as<double>(), G->asum.as<double>(), G->feat.as<float>());
  k_gnn_weights<<<grid_for(G->n, 128), 128, 0, s>>>(G->n, G->nb_ptr.as<int64_t>(), G->nb_other.as<int32_t>(), G->nb_edge.as<int32_t>(),
                                                    G->e_norm.as<double>(), G->asum.as<double>(), G->w_fwd.as<float>(), G->w_rev.as<float>());
  P->launches += 4;
  BLS_CUDA(cudaGetLastError());
  G->prepared = true;
  return -1;
}

template <class A, class IN1>
static void lin_fwd(GNNPlan* G, int K1, const IN1* in1, int K2, const A* in2, const float* W1, const float* W2, const float* b, int O, bool relu,
                    A* outA, float* outF) {
  cudaStream_t s = G->pcg->ctx->stream;
  if constexpr (std::is_same<A, __nv_bfloat16>::value && std::is_same<IN1, __nv_bfloat16>::value) {
    if (K1 % 16 == 0 && K2 % 16 == 0 && K1 + K2 <= LIN_MMA_KMAX && O <= LIN_MMA_OMAX) {   // the width-64 layers
      k_lin_mma<<<grid_for(G->n, 64), 128, 0, s>>>(G->n, K1, in1, K2, in2, W1, W2, b, O, relu, outA, outF);
      G->pcg->launches += 1;
      return;
    }
  }
  const size_t smem = sizeof(float) * O * (K1 + K2);
  if (smem > 48 * 1024) BLS_CUDA(cudaFuncSetAttribute(k_lin_fwd<A, IN1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_lin_fwd<A, IN1><<<grid_for(G->n * O, 256), 256, smem, s>>>(G->n, K1, in1, K2, in2, W1, W2, b, O, relu, outA, outF);
  G->pcg->launches += 1;
}

// Forward: activations of type A (float: kept for the backward pass; BF16: inference), t (FP32)
template <class A>
static void gnn_forward(GNNPlan* G, const float* prm) {
  cudaStream_t s = G->pcg->ctx->stream;
  A* h[GNN_LAYERS + 1];
  A* m[GNN_LAYERS];
  for (int l = 0; l <= GNN_LAYERS; ++l) h[l] = G->h[l].as<A>();
  for (int l = 0; l < GNN_LAYERS; ++l) m[l] = G->m[l].as<A>();
  lin_fwd<A, float>(G, GNN_F, G->feat.as<float>(), 0, nullptr, prm + GNN_OFF_WIN, nullptr, prm + GNN_OFF_BIN, GNN_H, true, h[0], nullptr);
  for (int l = 0; l < GNN_LAYERS; ++l) {
    k_gnn_agg<A><<<grid_for(G->n * 32, 256), 256, 0, s>>>(G->n, G->nb_ptr.as<int64_t>(), G->nb_other.as<int32_t>(), G->w_fwd.as<float>(), h[l], m[l]);
    G->pcg->launches += 1;
    const float* base = prm + GNN_OFF_L0 + l * GNN_LSTRIDE;
    lin_fwd<A, A>(G, GNN_H, h[l], GNN_H, m[l], base, base + GNN_H * GNN_H, base + 2 * GNN_H * GNN_H, GNN_H, true, h[l + 1], nullptr);
  }
  lin_fwd<A, A>(G, GNN_H, h[GNN_LAYERS], 0, nullptr, prm + GNN_OFF_WOUT, nullptr, prm + GNN_OFF_BOUT, GNN_T, false, nullptr, G->t.as<float>());
  BLS_CUDA(cudaGetLastError());
}

static void gnn_precond(GNNPlan* G) {
  k_gnn_precond<<<grid_for(G->n, 128), 128, 0, G->pcg->ctx->stream>>>(G->n, G->t.as<float>(), G->L.as<double>(), G->B.as<double>());
  G->pcg->launches += 1;
}

// S^ x = L^-1 (S (L^-T x)) into out (uses G->yh as scratch)
static void apply_Shat(GNNPlan* G, int dtype, const void* S, const double* x, double* out) {
  cudaStream_t s = G->pcg->ctx->stream;
  const unsigned gb = (unsigned)grid_for(G->n, 128);
  k_gnn_block<<<gb, 128, 0, s>>>(G->n, 1, nullptr, G->L.as<double>(), x, nullptr, G->yh.as<double>(), nullptr);
  pcg_spmv(G->pcg, dtype, S, G->yh.as<double>(), nullptr, out, false, s);
  k_gnn_block<<<gb, 128, 0, s>>>(G->n, 2, nullptr, G->L.as<double>(), out, nullptr, out, nullptr);
  G->pcg->launches += 2;
}

// Loss and gradient (FP32 network): grad (GNN_NPARAMS floats) overwritten; the loss Z N2 / N1^2 over the probes
// (P vectors of length 6 n, one after another).
static double gnn_loss_grad(GNNPlan* G, int dtype, const void* S, const float* prm, const double* probes, int64_t P, float* grad) {
  cudaStream_t s = G->pcg->ctx->stream;
  const int64_t n = G->n, nr = 6 * n;
  const unsigned gb = (unsigned)grid_for(n, 128);
  gnn_forward<float>(G, prm);
  BLS_CUDA(cudaMemsetAsync(G->accA.p, 0, G->accA.bytes, s));
  BLS_CUDA(cudaMemsetAsync(G->accB.p, 0, G->accB.bytes, s));
  BLS_CUDA(cudaMemsetAsync(G->loss.p, 0, G->loss.bytes, s));
  double* acc = G->loss.as<double>();   // [0] N1, [1] N2, [2] Z
  const float* t = G->t.as<float>();
  for (int64_t p = 0; p < P; ++p) {
    const double* z = probes + p * nr;
    k_dot_sq<<<std::max(1, std::min(grid_for(nr, 256), 148)), 256, 0, s>>>(nr, z, acc + 2);
    k_gnn_block<<<gb, 128, 0, s>>>(n, 0, t, nullptr, z, nullptr, G->y.as<double>(), nullptr);                // G' z
    apply_Shat(G, dtype, S, G->y.as<double>(), G->w.as<double>());                                             // w = S^ G' z
    k_gnn_block<<<gb, 128, 0, s>>>(n, 3, t, nullptr, G->w.as<double>(), z, G->v.as<double>(), acc);           // y = G w
    k_gnn_block<<<gb, 128, 0, s>>>(n, 0, t, nullptr, G->v.as<double>(), nullptr, G->u.as<double>(), nullptr);   // G' y
    apply_Shat(G, dtype, S, G->u.as<double>(), G->s.as<double>());                                             // s = S^ G' y
    k_gnn_outer<<<gb, 128, 0, s>>>(n, G->v.as<double>(), G->w.as<double>(), z, G->s.as<double>(), G->accA.as<double>());
    k_gnn_outer<<<gb, 128, 0, s>>>(n, z, G->w.as<double>(), nullptr, nullptr, G->accB.as<double>());
    G->pcg->launches += 6;
  }
  double* hz = G->pcg->host;
  BLS_CUDA(cudaMemcpyAsync(hz, acc, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  const double N1 = hz[0], N2 = hz[1], Z = hz[2];
  const double loss = Z * N2 / (N1 * N1);
  const double c = Z / (N1 * N1);
  k_gnn_combine<<<grid_for(GNN_T * n, 256), 256, 0, s>>>(GNN_T * n, 2.0 * c, G->accA.as<double>(), -4.0 * c * N2 / N1, G->accB.as<double>(),
                                                       G->dt.as<float>());
  G->pcg->launches += 1;
  // backward through the network
  BLS_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * GNN_NPARAMS, s));
  const int ych = (int)std::max<int64_t>(1, std::min<int64_t>(64, n / 64));
  auto bwd_w = [&](int O, const float* dout, const float* out, bool relu, int K1, const float* in1, int K2, const float* in2, float* dW1,
                   float* dW2, float* db) {
    dim3 grid((unsigned)grid_for(O * (K1 + K2 + 1), 256), (unsigned)ych);
    k_lin_bwd_weight<<<grid, 256, 0, s>>>(n, O, dout, out, relu, K1, in1, K2, in2, dW1, dW2, db);
    G->pcg->launches += 1;
  };
  auto bwd_d = [&](int O, const float* dout, const float* out, bool relu, int K1, const float* W1, float* din1, int K2, const float* W2,
                   float* din2) {
    k_lin_bwd_data<<<grid_for(n * (K1 + K2), 256), 256, 0, s>>>(n, O, dout, out, relu, K1, W1, din1, K2, W2, din2);
    G->pcg->launches += 1;
  };
  const float* hL = G->h[GNN_LAYERS].as<float>();
  // output head: t = W_out h3 + b_out
  bwd_w(GNN_T, G->dt.as<float>(), nullptr, false, GNN_H, hL, 0, nullptr, grad + GNN_OFF_WOUT, nullptr, grad + GNN_OFF_BOUT);
  bwd_d(GNN_T, G->dt.as<float>(), nullptr, false, GNN_H, prm + GNN_OFF_WOUT, G->dh.as<float>(), 0, nullptr, nullptr);
  for (int l = GNN_LAYERS - 1; l >= 0; --l) {
    const float* base = prm + GNN_OFF_L0 + l * GNN_LSTRIDE;
    float* gbase = grad + GNN_OFF_L0 + l * GNN_LSTRIDE;
    const float* out = G->h[l + 1].as<float>();
    const float* hin = G->h[l].as<float>();
    const float* min_ = G->m[l].as<float>();
    bwd_w(GNN_H, G->dh.as<float>(), out, true, GNN_H, hin, GNN_H, min_, gbase, gbase + GNN_H * GNN_H, gbase + 2 * GNN_H * GNN_H);
    bwd_d(GNN_H, G->dh.as<float>(), out, true, GNN_H, base, G->dh2.as<float>(), GNN_H, base + GNN_H * GNN_H, G->dm.as<float>());
    k_gnn_agg_bwd<<<grid_for(n * 32, 256), 256, 0, s>>>(n, G->nb_ptr.as<int64_t>(), G->nb_other.as<int32_t>(), G->w_rev.as<float>(),
                                                        G->dm.as<float>(), G->dh2.as<float>());
    G->pcg->launches += 1;
    std::swap(G->dh.p, G->dh2.p);
  }
  // input layer: h0 = relu(W_in f + b_in)
  bwd_w(GNN_H, G->dh.as<float>(), G->h[0].as<float>(), true, GNN_F, G->feat.as<float>(), 0, nullptr, grad + GNN_OFF_WIN, nullptr,
        grad + GNN_OFF_BIN);
  BLS_CUDA(cudaGetLastError());
  BLS_CUDA(cudaStreamSynchronize(s));
  return loss;
}

}  // namespace bls

struct bls_gnn : bls::GNNPlan {};
struct bls_pcg_plan : bls::PCGPlan {};
using namespace bls;

#define GNN_GUARD(...)                        \
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

int64_t bls_gnn_param_count(void) { return GNN_NPARAMS; }

int bls_gnn_create(bls_pcg_plan* pcg, const int64_t* block_colptr, const int64_t* block_rowval, const int64_t* block_row_offsets,
                   const int64_t* col_heights, const int64_t* S_colptr, bls_gnn** out) {
  GNN_GUARD({
    if (!pcg || !out || !block_colptr || !block_rowval || !block_row_offsets || !col_heights || !S_colptr) throw Error(BLS_EINVAL, "null argument");
    PCGPlan* P = static_cast<PCGPlan*>(pcg);
    if (P->max_d != 6 || (int64_t)P->nr != 6 * P->nrb) throw Error(BLS_EUNSUPPORTED, "the learned preconditioner needs 6 x 6 retained blocks");
    *out = static_cast<bls_gnn*>(gnn_create(P, block_colptr, block_rowval, block_row_offsets, col_heights, S_colptr));
    return BLS_OK;
  })
}

int bls_gnn_destroy(bls_gnn* g) {
  if (g) {
    cudaStreamSynchronize(g->pcg->ctx->stream);
    delete static_cast<GNNPlan*>(g);
  }
  return BLS_OK;
}

int bls_gnn_prepare(bls_gnn* g, int dtype, const void* S, int64_t* failed_block) {
  GNN_GUARD({
    if (!g || !failed_block) throw Error(BLS_EINVAL, "null argument");
    if (dtype != BLS_F64 && dtype != BLS_F32) throw Error(BLS_EINVAL, "unknown dtype");
    const int64_t fb = gnn_prepare(g, dtype, S);
    *failed_block = fb + 1;
    return fb >= 0 ? BLS_NOT_PD : BLS_OK;
  })
}

int bls_gnn_forward(bls_gnn* g, const float* params, int bf16, double* blocks) {
  GNN_GUARD({
    if (!g || !params || !blocks) throw Error(BLS_EINVAL, "null argument");
    if (!g->prepared) throw Error(BLS_EINVAL, "bls_gnn_prepare has not been called");
    if (bf16) gnn_forward<__nv_bfloat16>(g, params);
    else gnn_forward<float>(g, params);
    gnn_precond(g);
    cudaStream_t s = g->pcg->ctx->stream;
    BLS_CUDA(cudaMemcpyAsync(blocks, g->B.p, sizeof(double) * 36 * g->n, cudaMemcpyDeviceToDevice, s));
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

int bls_gnn_outputs(bls_gnn* g, float* t_out, float* features_out, double* edge_norms_out) {
  GNN_GUARD({
    if (!g) throw Error(BLS_EINVAL, "null argument");
    cudaStream_t s = g->pcg->ctx->stream;
    if (t_out) BLS_CUDA(cudaMemcpyAsync(t_out, g->t.p, sizeof(float) * GNN_T * g->n, cudaMemcpyDeviceToDevice, s));
    if (features_out) BLS_CUDA(cudaMemcpyAsync(features_out, g->feat.p, sizeof(float) * GNN_F * g->n, cudaMemcpyDeviceToDevice, s));
    if (edge_norms_out && g->nedges) BLS_CUDA(cudaMemcpyAsync(edge_norms_out, g->e_norm.p, sizeof(double) * g->nedges, cudaMemcpyDeviceToDevice, s));
    return BLS_OK;
  })
}

int64_t bls_gnn_edge_count(bls_gnn* g) { return g ? g->nedges : -1; }

int bls_gnn_loss_grad(bls_gnn* g, int dtype, const void* S, const float* params, const double* probes, int64_t nprobes, double* loss,
                      float* grad) {
  GNN_GUARD({
    if (!g || !params || !probes || !loss || !grad || nprobes < 1) throw Error(BLS_EINVAL, "null argument");
    if (!g->prepared) throw Error(BLS_EINVAL, "bls_gnn_prepare has not been called");
    if (dtype != BLS_F64 && dtype != BLS_F32) throw Error(BLS_EINVAL, "unknown dtype");
    *loss = gnn_loss_grad(g, dtype, S, params, probes, nprobes, grad);
    return BLS_OK;
  })
}

int bls_adam_step(bls_ctx* ctx, float* params, const float* grad, float* m, float* v, int64_t n, float lr, float beta1, float beta2, float eps,
                  int64_t step) {
  GNN_GUARD({
    if (!ctx || n < 0 || step < 1) throw Error(BLS_EINVAL, "bad argument");
    const float c1 = 1.f - std::pow(beta1, (float)step), c2 = 1.f - std::pow(beta2, (float)step);
    if (n > 0) k_adam<<<grid_for(n, 256), 256, 0, ctx->stream>>>(n, params, grad, m, v, lr, beta1, beta2, eps, c1, c2);
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

}  // extern "C"
