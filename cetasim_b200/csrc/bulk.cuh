// Bulk asynchronous copies global -> shared memory (cp.async.bulk, no tensor
// map, no multicast), completed through an mbarrier's transaction count.
// Both addresses 16-byte aligned, sizes multiples of 16 bytes.
#pragma once
#include <cstdint>
#include "umma.cuh"

namespace cg {
namespace bulk {

// mbarrier.init results visible to the asynchronous proxy
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive on `bar` (one of its `count` arrivals) and expect `bytes` more
// transaction bytes before the phase completes.
__device__ __forceinline__ void arrive_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :
               : "r"(bar), "r"(bytes)
               : "memory");
}

// Copy `bytes` from global `src` to shared `dst` (this CTA's); the bytes
// count against the transaction count of `bar`.
__device__ __forceinline__ void load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :
      : "r"(dst), "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

}  // namespace bulk
}  // namespace cg
