// pipeline.cuh -- asynchronous global->shared staging primitives for sm_100a (inline PTX).
//
//   cp.async (LDGSTS, 4/8-byte)        irregular gathers of node values through the restriction offsets
//   cp.async.bulk + mbarrier (TMA)     contiguous per-element blocks (qdata, stored Jacobian data)
//   cp.async.bulk.prefetch.L2          warming L2 ahead of a later request
// Every wait on an mbarrier is bounded: after kMbarSpin unsuccessful try_wait rounds the caller gets `false`, records an
// error status for the host and leaves the kernel instead of spinning forever.
#pragma once

#include <stdint.h>

namespace hb {

constexpr int kMbarSpin = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// wait until at most N of this thread's most recently committed groups are still pending
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *m, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *m, unsigned bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *m, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *m, unsigned parity) {
  for (int i = 0; i < kMbarSpin; i++)
    if (mbar_try_wait(m, parity)) return true;
  return false;
}
// Order earlier generic-proxy accesses of shared memory before later async-proxy (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One-dimensional bulk copy global -> shared, completing `bytes` transactions on mbarrier m.  dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void tma_load_1d(void *dst, const void *src, unsigned bytes, uint64_t *m) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)), "l"(src),
               "r"(bytes), "r"(smem_u32(m))
               : "memory");
}

// warm L2 with the 128-byte line holding p
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

__device__ __forceinline__ void prefetch_l2_bulk(const void *p, size_t bytes) {
  const uintptr_t a = (uintptr_t)p, lo = (a + 15) & ~(uintptr_t)15, hi = (a + bytes) & ~(uintptr_t)15;
  if (hi > lo) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)(hi - lo)) : "memory");
}

// Stage `count` values of a contiguous per-element block into shared memory.  With `tma` (host-checked: 16-byte aligned
// source and a size that is a multiple of 16) one thread issues a bulk copy on mbarrier m and returns the bytes it
// expects; otherwise every thread issues its share of 8- or 4-byte cp.async copies.
template <typename T, int NT>
__device__ __forceinline__ unsigned stage_block(T *dst, const T *src, int count, bool tma, uint64_t *m) {
  const unsigned bytes = (unsigned)(count * sizeof(T));
  if (tma) {
    if (threadIdx.x == 0) tma_load_1d(dst, src, bytes, m);
    return bytes;
  }
  if (sizeof(T) == 8 || (((uintptr_t)src & 7) == 0 && (count & 1) == 0)) {
    const int n8 = (int)(bytes / 8);
    for (int i = threadIdx.x; i < n8; i += NT) cp_async8((char *)dst + 8 * i, (const char *)src + 8 * i);
  } else {
    for (int i = threadIdx.x; i < count; i += NT) cp_async4(dst + i, src + i);
  }
  return 0;
}

}  // namespace hb
