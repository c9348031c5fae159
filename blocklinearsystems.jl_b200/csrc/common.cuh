// Shared device/host helpers of libblsgpu.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "host_layout.hpp"

namespace bls {

void set_error(const std::string& msg);

#define BLS_CUDA(x)                                                                                     \
  do {                                                                                                  \
    cudaError_t e_ = (x);                                                                               \
    if (e_ != cudaSuccess) throw ::bls::Error(BLS_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Device status word of a plan. `failed` is the lowest failing eliminated block; `einval_r` / `einval_e` the lowest
// non-finite or negative entry of the reset's scaling_r / the reduction's scaling_e; LLONG_MAX means none. Kernels read
// it to skip their work, as the reference throws before writing (src/utils.jl:100-107) and returns before phase 2
// after a failure (src/schur_reduction.jl:499).
struct Status {
  long long failed;
  long long einval_r;
  long long einval_e;
  long long pad;
};

template <class T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

inline int grid_for(int64_t n, int threads) { return (int)((n + threads - 1) / threads); }

// A device buffer that frees itself.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (p) cudaFree(p); }
  void alloc(size_t b) {
    if (p) { cudaFree(p); p = nullptr; }
    bytes = b;
    if (b) BLS_CUDA(cudaMalloc(&p, b));
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

template <class T>
void upload(DevBuf& buf, const std::vector<T>& v, cudaStream_t s) {
  buf.alloc(v.size() * sizeof(T));
  if (!v.empty()) BLS_CUDA(cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

// One block of symmetrifyfull!: data[src ...] (rd x cd, column-major) to mat's rows rs.. and columns cs.., and
// transposed to rows cs.. and columns rs.. unless diag.
struct SymBlock {
  int64_t src, rs, cs;
  int32_t rd, cd, diag, pad;
};
// Zeroes the m x m matrix and copies the blocks (a host list, copied to the device on stream s).
void launch_symmetrify(cudaStream_t s, int dtype, const void* data, const SymBlock* blocks_host, int64_t nblocks, void* mat,
                       int64_t m);

}  // namespace bls

struct bls_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int* flag = nullptr;   // device scratch word for calls that report a device-side decision (allocated at first use)
};
