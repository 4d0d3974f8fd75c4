// sb200_tma.cuh -- shared-memory barriers and bulk / tensor copies (TMA) for
// sm_100a, as inline PTX.  No cluster multicast is used anywhere: every copy
// moves data of this GPU's own memory into the issuing CTA's shared memory.
//
// Every wait is bounded: mbar_wait gives up after SB200_WAIT_CYCLES clock
// cycles (about a second) and returns false, so a copy that never completes
// turns into an error status instead of a hung GPU.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#ifndef SB200_WAIT_CYCLES
#define SB200_WAIT_CYCLES 2000000000LL
#endif

namespace sb200 {
namespace tma {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

// make barrier initialisation visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order the CTA's earlier generic-proxy shared-memory accesses (after a CTA
// barrier) before later asynchronous-proxy writes to the same memory
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait for the phase with the given parity to complete; false after
// SB200_WAIT_CYCLES cycles without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > SB200_WAIT_CYCLES) return false;
  }
  return true;
}

// 1-D bulk copy global -> shared (both 16-byte aligned, bytes % 16 == 0),
// completion counted on the barrier.
// bytes (a multiple of 16, 16-byte aligned) of global memory into L2, no completion tracking
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(saddr(dst)),
      "l"(src), "r"(bytes), "r"(saddr(bar))
      : "memory");
}

// 4-D tiled tensor load of one box at element coordinates (c0 innermost);
// box elements outside the tensor are filled with zeros.  The tensor map is a
// kernel parameter (__grid_constant__) or lives in global memory.
__device__ __forceinline__ void tensor_load_4d(void* dst, const void* tmap, int c0, int c1, int c2, int c3,
                                               uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(saddr(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(saddr(bar))
      : "memory");
}

}  // namespace tma
}  // namespace sb200
