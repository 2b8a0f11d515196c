// Bulk global->shared copies (cp.async.bulk, the TMA engine's untiled form) completing on a CTA mbarrier, with a
// bounded wait. Shared by the kernels that stage static operands into shared memory.
#pragma once
#include <cuda_runtime.h>

namespace drape {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// Orders the generic-proxy initialisation of the barrier before the async proxy's use of it.
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// dst and src 16-byte aligned, bytes a multiple of 16 (the instruction's rules; the callers guarantee them).
__device__ __forceinline__ void bulk_copy_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// Polls the barrier's phase `parity` for at most `limit` clock cycles; true when the phase completed.
__device__ __forceinline__ bool mbar_wait_parity(unsigned bar, unsigned parity, long long limit) {
  const long long t0 = clock64();
  while (true) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}

}  // namespace drape
