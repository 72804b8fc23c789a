// Asynchronous copies into shared memory and mbarrier waits (sm_90+ PTX),
// shared by the streaming kernels.  Every wait is bounded.
#pragma once
#include <cstdint>

namespace cxb {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *m, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *m, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(m)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *m) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(
                   smem_u32(m))
               : "memory");
}
// Arrives on m (one arrival) and raises its expected transaction bytes by
// `bytes` in one step.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *m, uint32_t bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(
                   smem_u32(m)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *m, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok)
               : "r"(smem_u32(m)), "r"(parity)
               : "memory");
  return ok != 0;
}
// Default bound of a wait, in SM clock cycles: about a second.
constexpr long long kWaitCycles = 1ll << 31;
// Waits for the phase of parity `parity` to complete, polling for at most
// `limit` clock cycles (each poll may suspend the thread for a short
// hardware-defined time); false if it gave up.  A limit of 0 gives up at
// once without polling: tests use it to force the give-up path.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *m, uint32_t parity,
                                                  long long limit = kWaitCycles) {
  if (limit <= 0)
    return false;
  const long long t0 = clock64();
  while (!mbar_try(m, parity))
    if (clock64() - t0 > limit)
      return false;
  return true;
}
// Bulk copy global -> this CTA's shared memory (no multicast), completing
// `bytes` on mbarrier m; both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *m) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
               "[%3];\n" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(m))
               : "memory");
}
// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

} // namespace cxb
