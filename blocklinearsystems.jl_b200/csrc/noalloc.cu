// bls_reduce_schur_dense_noalloc: reduce_schur_dense! for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code whose device memory belongs to an allocator it does not
// own (a Julia session whose CuArrays come from CUDA.jl's pool, a PyTorch process under its caching allocator), code
// held to a fixed device-memory budget, and loops that cannot afford a driver allocation each time a new structure
// arrives. Every other reduction entry point needs a plan, and a plan allocates (its index arrays and its scratch).
// This one takes the structure's two index arrays from the caller, already in device memory, and keeps its scratch
// -- each point's damped inverse and z, and a status word -- in a file-scope static device array. It allocates
// nothing: no cudaMalloc, no cudaFree, no allocating library routine.
//
// Scope: retained blocks of size 6 and eliminated blocks of size 3 in the canonical layout (the layout
// SchurStructure builds for such blocks: coupling c at C_data[18c], point e at E_data[9e]), dense S, at most
// BLS_NOALLOC_MAX_POINTS eliminated blocks. The arithmetic of the point inverse is the plan path's; the pair products
// are accumulated point by point with atomic adds, which suits the small problems this size limit admits.
#include <climits>
#include <cmath>
#include <mutex>

#include "closed_inverse.cuh"
#include "common.cuh"

namespace bls {

constexpr long long NA_NONE = LLONG_MAX;

// Scratch shared by every call on a device: per point E^-1 (9) and z (3), then the status words (failed block,
// first bad scaling entry). Every GPU that loads the library holds it (12 * 65536 * 8 bytes + 32, about 6.3 MB)
// until the process exits. Calls whose work overlaps on the GPU (different streams, or host threads) race on it.
__device__ __align__(256) double g_noalloc_scratch[12 * BLS_NOALLOC_MAX_POINTS + 4];

// In host code `g_noalloc_scratch` names a host-side stand-in, not a device address: kernels must be given the address
// that cudaGetSymbolAddress returns, which is looked up once per device (with that device current) and cached.
static std::mutex g_na_mutex;
static double* g_na_addr[128];

static double* noalloc_scratch(int device) {
  if (device < 0 || device >= 128) throw Error(BLS_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_na_mutex);
  if (!g_na_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) throw Error(BLS_ECUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") + cudaGetErrorString(e));
    g_na_addr[device] = static_cast<double*>(p);
  }
  return g_na_addr[device];
}

__device__ __forceinline__ long long* na_status(double* scratch) {
  return reinterpret_cast<long long*>(scratch + 12 * BLS_NOALLOC_MAX_POINTS);
}

// status[0] failed block, status[1] first bad scaling_e entry, status[2] a malformed structure index
__global__ void k_na_begin(double* scratch) {
  long long* st = na_status(scratch);
  st[0] = NA_NONE;
  st[1] = NA_NONE;
  st[2] = NA_NONE;
}

__global__ void k_na_check(const double* __restrict__ sc, int64_t n, double* scratch) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = sc[i];
  if (!(isfinite(x) && x >= 0.0)) atomicMin(na_status(scratch) + 1, (long long)i);
}

// structure check: eliminated_ptr ascending within [0, ncoup], entry_retained ascending per point within [0, nrb)
__global__ void k_na_validate(int64_t neb, int64_t nrb, int64_t ncoup, const int64_t* __restrict__ eptr,
                              const int64_t* __restrict__ eret, double* scratch) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= neb) return;
  const int64_t p0 = eptr[e], p1 = eptr[e + 1];
  bool ok = p0 >= 0 && p0 <= p1 && p1 <= ncoup;
  for (int64_t c = p0; ok && c < p1; ++c) {
    const int64_t r = eret[c];
    ok = r >= 0 && r < nrb && (c == p0 || eret[c - 1] < r);
  }
  if (!ok) atomicMin(na_status(scratch) + 2, (long long)e);
}

__device__ __forceinline__ bool na_live(double* scratch) {
  const long long* st = na_status(scratch);
  return st[0] == NA_NONE && st[1] == NA_NONE && st[2] == NA_NONE;
}

template <class T>
__global__ void k_na_factor(int64_t neb, const T* __restrict__ E, const double* __restrict__ b_e, const double* __restrict__ sc_e,
                            double lambda, double* scratch) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= neb || !na_live(scratch)) return;
  double H[9], damp[3], inv[9];
  for (int i = 0; i < 9; ++i) H[i] = (double)E[9 * e + i];
  for (int i = 0; i < 3; ++i) damp[i] = mul(lambda, sc_e[3 * e + i]);
  if (!inv_sym_closed(3, H, damp, inv)) {
    atomicMin(na_status(scratch), (long long)e);
    return;
  }
  double* q = scratch + 12 * e;
  for (int i = 0; i < 9; ++i) q[i] = inv[i];
  for (int i = 0; i < 3; ++i) q[9 + i] = inv[i] * b_e[3 * e] + inv[i + 3] * b_e[3 * e + 1] + inv[i + 6] * b_e[3 * e + 2];
}

__global__ void k_na_ginit(double* __restrict__ g, const double* __restrict__ b_r, int64_t nr, double* scratch) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nr || !na_live(scratch)) return;
  g[i] = b_r[i];
}

// One warp per point: its k(k+1)/2 pair blocks C_ci' (E^-1 C_cj), i <= j (upper triangle of the diagonal blocks), and
// the gradient terms C_cj' z, added to S and g_S with atomics. Work indices are 64-bit (a point may couple to many
// retained blocks), and the pair (i, j) of a work index is found in closed form from the triangular numbers.
template <class T>
__global__ void k_na_accumulate(int64_t neb, int64_t nr, const int64_t* __restrict__ eptr, const int64_t* __restrict__ eret,
                                const T* __restrict__ C, T* __restrict__ S, double* __restrict__ g, double* scratch) {
  const int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (e >= neb || !na_live(scratch)) return;
  const int64_t p0 = eptr[e];
  const int64_t k = eptr[e + 1] - p0;
  const double* q = scratch + 12 * e;
  double Ei[9], z[3];
  for (int i = 0; i < 9; ++i) Ei[i] = q[i];
  for (int i = 0; i < 3; ++i) z[i] = q[9 + i];
  const int64_t npairs = k * (k + 1) / 2;
  for (int64_t t = lane; t < npairs * 36; t += 32) {
    const int64_t pi = t / 36;
    const int ent = (int)(t - 36 * pi), rho = ent / 6, w = ent - 6 * rho;
    // pair pi = (i, j) with i <= j, ordered by j then i: j is the largest with j (j + 1) / 2 <= pi
    int64_t j = (int64_t)((sqrt(8.0 * (double)pi + 1.0) - 1.0) * 0.5);
    while ((j + 1) * (j + 2) / 2 <= pi) ++j;
    while (j * (j + 1) / 2 > pi) --j;
    const int64_t i = pi - j * (j + 1) / 2;
    if (i == j && rho > w) continue;
    const T* ci = C + 18 * (p0 + i) + 3 * rho;
    const T* cj = C + 18 * (p0 + j) + 3 * w;
    double u[3];
    for (int s = 0; s < 3; ++s) u[s] = Ei[s] * (double)cj[0] + Ei[s + 3] * (double)cj[1] + Ei[s + 6] * (double)cj[2];
    const double v = (double)ci[0] * u[0] + (double)ci[1] * u[1] + (double)ci[2] * u[2];
    const int64_t ri = eret[p0 + i], rj = eret[p0 + j];
    atomicAdd(S + (6 * ri + rho) + (6 * rj + w) * nr, T(-v));
  }
  for (int64_t t = lane; t < 6 * k; t += 32) {
    const int64_t j = t / 6;
    const int w = (int)(t - 6 * j);
    const T* cj = C + 18 * (p0 + j) + 3 * w;
    atomicAdd(g + 6 * eret[p0 + j] + w, -((double)cj[0] * z[0] + (double)cj[1] * z[1] + (double)cj[2] * z[2]));
  }
}

template <class T>
static void na_launch(cudaStream_t s, double* sc, int64_t nrb, int64_t neb, int64_t ncoup, const int64_t* eptr, const int64_t* eret, T* S,
                      double* g, const double* b_r, const double* b_e, const double* sc_e, double lambda, const T* E, const T* C) {
  const int64_t nr = 6 * nrb;
  k_na_begin<<<1, 1, 0, s>>>(sc);
  k_na_check<<<grid_for(3 * neb, 256), 256, 0, s>>>(sc_e, 3 * neb, sc);
  k_na_validate<<<grid_for(neb, 256), 256, 0, s>>>(neb, nrb, ncoup, eptr, eret, sc);
  k_na_factor<T><<<grid_for(neb, 256), 256, 0, s>>>(neb, E, b_e, sc_e, lambda, sc);
  k_na_ginit<<<grid_for(nr, 256), 256, 0, s>>>(g, b_r, nr, sc);
  k_na_accumulate<T><<<grid_for(neb * 32, 256), 256, 0, s>>>(neb, nr, eptr, eret, C, S, g, sc);
  BLS_CUDA(cudaGetLastError());
}

// The verdict of the last call on this device, from the status words of the static array (copied on `s`, which
// waits for that call's kernels when it is the call's stream). Allocates nothing.
static int na_verdict(cudaStream_t s, double* sc, int64_t* failed_block) {
  long long st[3];
  BLS_CUDA(cudaMemcpyAsync(st, sc + 12 * BLS_NOALLOC_MAX_POINTS, sizeof(st), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  if (failed_block) *failed_block = 0;
  if (st[2] != NA_NONE) throw Error(BLS_EINVAL, "malformed structure: eliminated block " + std::to_string(st[2] + 1) + " has out-of-range couplings");
  if (st[1] != NA_NONE) throw Error(BLS_EINVAL, "scaling_e must be finite and non-negative, but entry " + std::to_string(st[1] + 1) + " is not");
  if (st[0] != NA_NONE) {
    if (failed_block) *failed_block = st[0] + 1;
    return BLS_NOT_PD;
  }
  return BLS_OK;
}

}  // namespace bls

using namespace bls;

extern "C" int bls_reduce_schur_dense_noalloc(void* cuda_stream, int dtype, int64_t nrblocks, int64_t neblocks, int64_t ncouplings,
                                              const int64_t* eliminated_ptr_dev, const int64_t* entry_retained_dev, void* S_dev,
                                              double* g_S_dev, const double* b_r_dev, const double* b_e_dev,
                                              const double* scaling_e_dev, double lambda, const void* E_dev, const void* C_dev,
                                              int64_t* failed_block) {
  try {
    if (neblocks < 1 || neblocks > BLS_NOALLOC_MAX_POINTS)
      throw Error(BLS_EUNSUPPORTED, "bls_reduce_schur_dense_noalloc handles 1 to " + std::to_string(BLS_NOALLOC_MAX_POINTS) +
                                        " eliminated blocks (its scratch is a fixed static array); got " + std::to_string(neblocks));
    if (nrblocks < 1 || ncouplings < 0) throw Error(BLS_EINVAL, "nrblocks must be positive and ncouplings non-negative");
    if (!(std::isfinite(lambda) && lambda >= 0)) throw Error(BLS_EINVAL, "lambda must be finite and non-negative, got " + std::to_string(lambda));
    if (dtype != BLS_F64 && dtype != BLS_F32) throw Error(BLS_EINVAL, "unknown dtype");
    int dev = 0;
    BLS_CUDA(cudaGetDevice(&dev));
    double* sc = noalloc_scratch(dev);
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    if (dtype == BLS_F64)
      na_launch<double>(s, sc, nrblocks, neblocks, ncouplings, eliminated_ptr_dev, entry_retained_dev, (double*)S_dev, g_S_dev, b_r_dev,
                        b_e_dev, scaling_e_dev, lambda, (const double*)E_dev, (const double*)C_dev);
    else
      na_launch<float>(s, sc, nrblocks, neblocks, ncouplings, eliminated_ptr_dev, entry_retained_dev, (float*)S_dev, g_S_dev, b_r_dev,
                       b_e_dev, scaling_e_dev, lambda, (const float*)E_dev, (const float*)C_dev);
    if (!failed_block) return BLS_OK;
    return na_verdict(s, sc, failed_block);
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  }
}

extern "C" int bls_reduce_schur_dense_noalloc_status(void* cuda_stream, int64_t* failed_block) {
  try {
    int dev = 0;
    BLS_CUDA(cudaGetDevice(&dev));
    return na_verdict(static_cast<cudaStream_t>(cuda_stream), noalloc_scratch(dev), failed_block);
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  }
}
