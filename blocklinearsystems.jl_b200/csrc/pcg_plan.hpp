// The device plan of block-Jacobi PCG on the reduced system (shared by the PCG and the learned-preconditioner code).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace bls {

// Slot layout of the per-iteration scalars: rz (r'z entering the iteration), pq, rz_next, rr_next
constexpr int PS_RZ = 0, PS_PQ = 1, PS_RZN = 2, PS_RRN = 3, PS_W = 4;

struct RowEntry {
  int64_t base;     // S offset of the block's first entry
  int32_t stride;   // column stride of the block in S
  int32_t xo;       // offset of the other block's variables in x
  int16_t dother;   // dimension of the other block
  int16_t mode;     // 0: B x (block right of the diagonal), 1: B' x (block above), 2: diagonal (symmetric)
  int32_t pad;
};

struct PCGPlan {
  bls_ctx* ctx = nullptr;
  int64_t nrb = 0, nr = 0, nnz = 0, ndiag = 0;
  int max_d = 0;
  DevBuf row_ptr, rows, r_dims, boff, doff, diag_base, diag_stride;
  // solver state (FP64)
  DevBuf D;                 // factored diagonal blocks (L in the lower triangle)
  DevBuf r, z, p, q, scal, flags;
  // q = S p by block columns (every r_dim 6): per block column its blocks, per block its S offset and its row
  // variables' offset; S is read once, the products scattered into q with FP64 atomics
  bool cols6 = false;
  DevBuf c_ptr, c_base, c_xo, c_stride;
  DevBuf ref_r, ref_d, ref_y;   // refined solve: outer residual, correction, operator product (FP64, allocated at its first call)
  int K = 8;                // iterations per replayed graph
  cudaGraphExec_t graph = nullptr;
  const void* graph_S = nullptr;
  const double* graph_x = nullptr;
  const double* graph_precond = nullptr;
  int graph_dtype = -1;
  cudaStream_t cap_stream = nullptr;   // the plan's own stream: graphs are captured and replayed there
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  const double* precond = nullptr;     // dense preconditioner blocks (doff layout), or null for block-Jacobi
  double* host = nullptr;   // pinned scratch for scalars read back
  int64_t launches = 0;
  ~PCGPlan() {
    if (graph) cudaGraphExecDestroy(graph);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (host) cudaFreeHost(host);
  }
};

// Host hooks into the PCG kernels (dtype BLS_F64 / BLS_F32 for S's storage)
void pcg_spmv(PCGPlan* P, int dtype, const void* S, const double* x, const double* g, double* y, bool residual, cudaStream_t s);
void pcg_extract_diag(PCGPlan* P, int dtype, const void* S, double* D, cudaStream_t s);
// Factor the d x d blocks of D (doff layout) in place; the lowest failing block (0-based) or -1. Synchronises.
int64_t pcg_factor_blocks(PCGPlan* P, double* D, cudaStream_t s);

}  // namespace bls
