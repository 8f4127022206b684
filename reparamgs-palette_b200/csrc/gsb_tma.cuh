// 1-D bulk copies (TMA, cp.async.bulk) between global and shared memory,
// completed through an mbarrier.  No cluster multicast is used anywhere.
//
// Every wait is bounded: mbar_wait gives up after a fixed number of
// try_wait polls and reports failure, so a kernel can record an error status
// and return instead of hanging.
#pragma once

#include "gsb_common.cuh"
#include "gsb_stage.cuh"

namespace gsb {

constexpr uint32_t kMbarPollLimit = 1u << 22;

// Device status bits (read with gsb_device_status / gsb_device_status_fetch).
constexpr uint32_t kStatusBulkTimeout = 1u;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Global -> shared bulk copy; `bytes` a multiple of 16, both addresses 16-byte
// aligned.  Completion is signalled on `bar` as transaction bytes.
__device__ __forceinline__ void bulk_load(void* sdst, const void* gsrc, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(sdst)),
      "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// true once the barrier's phase `parity` has completed; false after `limit`
// polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          uint32_t limit = kMbarPollLimit) {
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Shared -> global bulk copy (bulk async-group); the issuing thread must call
// bulk_store_drain() before the CTA's shared memory is released.
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst),
               "r"(smem_u32(ssrc)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_store_drain() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Makes this thread's generic-proxy shared-memory writes visible to the bulk
// copy (async proxy).
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool aligned16(const void* p) {
  return ((uintptr_t)p & 15u) == 0;
}

// Copies the block's rows of one input array into shared memory: a bulk copy
// when `bulk` (issued by thread 0, counted on `bar`), else a batched
// per-thread copy.  Returns the bytes the bulk copy will deliver.
template <int ROWLEN, typename T>
__device__ __forceinline__ uint32_t stage_rows(const T* g, int64_t row0, int64_t n, float* s,
                                               bool bulk, uint64_t* bar) {
  if (bulk) {
    const uint32_t bytes = (uint32_t)(blockDim.x * ROWLEN * sizeof(float));
    if (threadIdx.x == 0) bulk_load(s, g + row0 * ROWLEN, bytes, bar);
    return bytes;
  }
  stage_in_plain<ROWLEN>(g, row0, n, s);
  return 0;
}

}  // namespace gsb
