// Bulk (TMA, 1-D) global -> shared copies completed on an mbarrier, shared by the kernels that stage contiguous
// spans (QR tables, the Schur phase-2 column stages). Local memory only: no cluster multicast, no peer memory.
//
// A 1-D bulk copy needs a 16-byte-aligned source and destination and a size that is a multiple of 16 bytes. A span
// of elements that starts or ends inside a 16-byte chunk is copied from the aligned chunk boundary below its start
// (the destination keeps the source's offset within the chunk), and up to the aligned boundary above its end when that
// boundary is still inside the source buffer; otherwise the last partial chunk is copied by the issuing thread with
// plain loads (span_bytes gives the bytes the mbarrier must expect).
//
// Every wait is bounded: a wait that gives up returns false and the caller records a fault and drains its copies.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bls {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// make the initialised barrier visible to the async proxy (the bulk copies complete on it)
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// Wait for the phase of `parity` to complete; false after `limit` unsuccessful polls (each poll may suspend the
// thread for a hardware-chosen time, so the bound is on the order of seconds, far above any copy's duration).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = 1u << 24) {
  for (uint32_t n = 0; n < limit; ++n)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// Order this thread's earlier generic-proxy accesses of shared memory before later async-proxy (bulk copy) writes to it.
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// The bulk part of staging `n` elements at `src` (inside a global buffer that ends at `buf_end`, exclusive, and starts
// at a 16-byte boundary or earlier): the aligned chunk range [lo, hi) copied by one bulk copy (hi == lo: none).
struct Span {
  uintptr_t src, lo, hi, end;
};
template <class T>
__device__ __forceinline__ Span span_of(const T* src, int64_t n, const T* buf_end) {
  Span s;
  s.src = reinterpret_cast<uintptr_t>(src);
  s.lo = s.src & ~uintptr_t(15);
  s.end = s.src + (uintptr_t)n * sizeof(T);
  s.hi = (s.end + 15) & ~uintptr_t(15);
  if (s.hi > reinterpret_cast<uintptr_t>(buf_end)) s.hi = s.end & ~uintptr_t(15);   // stop before the buffer's end
  if (s.hi < s.lo) s.hi = s.lo;
  return s;
}
__device__ __forceinline__ uint32_t span_bytes(const Span& s) { return (uint32_t)(s.hi - s.lo); }

// Issue the span's bulk copy to shared memory at `dst16` (16-byte aligned, room for n * sizeof(T) + 32 bytes) and copy
// the tail it does not cover with plain loads (visible to other threads after the caller's wait and a barrier).
// Returns the shared address of src[0]. One thread calls this per span, after the mbarrier expects span_bytes.
template <class T>
__device__ __forceinline__ T* span_issue(T* dst16, const Span& s, uint64_t* bar) {
  char* d = reinterpret_cast<char*>(dst16);
  if (s.hi > s.lo) bulk_g2s(d, reinterpret_cast<const void*>(s.lo), (uint32_t)(s.hi - s.lo), bar);
  for (uintptr_t a = s.hi > s.src ? s.hi : s.src; a < s.end; a += sizeof(T))
    *reinterpret_cast<T*>(d + (a - s.lo)) = *reinterpret_cast<const T*>(a);
  return reinterpret_cast<T*>(d + (s.src - s.lo));
}
// The shared address of src[0] for a span staged at dst16 (any thread).
template <class T>
__device__ __forceinline__ T* span_first(T* dst16, const Span& s) {
  return reinterpret_cast<T*>(reinterpret_cast<char*>(dst16) + (s.src - s.lo));
}

// Shared -> global bulk copy (both 16-byte aligned, bytes a multiple of 16), in this thread's bulk group.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)), "r"(bytes) : "memory");
}

// Store n elements from shared memory at src to global memory at dst, both at the same offset within a 16-byte chunk:
// the aligned interior by one bulk copy, the ragged head and tail (under 16 bytes each) by plain stores, so nothing
// outside [dst, dst + n) is written. One thread calls it, after every thread that wrote src has run
// fence_proxy_async_shared() and a barrier with it; it returns once the copy has read src (so src may be reused or the
// CTA may exit); the global writes complete before the kernel does.
template <class T>
__device__ __forceinline__ void span_store(T* dst, const T* src, int64_t n) {
  const uintptr_t d0 = reinterpret_cast<uintptr_t>(dst), d1 = d0 + (uintptr_t)n * sizeof(T);
  const uintptr_t lo = (d0 + 15) & ~uintptr_t(15), hi = d1 & ~uintptr_t(15);
  const char* s = reinterpret_cast<const char*>(src);
  if (hi <= lo) {
    for (int64_t i = 0; i < n; ++i) dst[i] = src[i];
    return;
  }
  for (uintptr_t a = d0; a < lo; a += sizeof(T)) *reinterpret_cast<T*>(a) = *reinterpret_cast<const T*>(s + (a - d0));
  for (uintptr_t a = hi; a < d1; a += sizeof(T)) *reinterpret_cast<T*>(a) = *reinterpret_cast<const T*>(s + (a - d0));
  bulk_s2g(reinterpret_cast<void*>(lo), s + (lo - d0), (uint32_t)(hi - lo));
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

}  // namespace bls
