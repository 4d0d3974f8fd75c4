// sb200_tmem.cuh -- tensor memory (TMEM) of sm_100a as per-thread storage,
// as inline PTX (tcgen05.*).
//
// TMEM is 128 lanes x 512 columns of 32-bit cells per SM.  A warp reaches the
// 32 lanes of its quarter, 32 * (warp % 4) .. + 31, one lane per thread, so a
// thread can park values in "its" lane across any columns its warp owns.  The
// kernels here hold no MMA accumulators in TMEM: they use it as storage that
// costs neither registers nor shared memory (the Taylor accumulator psi_out,
// per-point potential and map words), read and written with the 32x32b
// shape.  Every load / store below waits for its own completion in the same
// asm statement, so the values are valid as soon as the statement returns.
//
// Allocation is by one whole warp; the CTA must hold the columns only while it
// runs: dealloc them (after a CTA barrier) before the kernel exits.  The
// kernels that use TMEM run one CTA per SM (their shared memory allows no
// more), so an allocation never waits for columns held by another CTA.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace sb200 {
namespace tmem {

// one whole warp: allocate ncols columns (a power of two, 32..512); the TMEM
// address (lane 0, first column) is written to *dst in shared memory
__device__ __forceinline__ void alloc(uint32_t* dst, uint32_t ncols) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// one whole warp, after every thread's last TMEM access (CTA barrier between)
__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// order TMEM operations around a CTA barrier
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM address of column `col` in the lanes of the calling warp's quarter
__device__ __forceinline__ uint32_t warp_addr(uint32_t base, int warp, uint32_t col) {
  return base + ((uint32_t)(32 * (warp & 3)) << 16) + col;
}

__device__ __forceinline__ void ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void st4(uint32_t taddr, const uint32_t (&r)[4]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};\n\t"
      "tcgen05.wait::st.sync.aligned;" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3])
      : "memory");
}

__device__ __forceinline__ void ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n\t"
      "tcgen05.wait::st.sync.aligned;" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
      : "memory");
}

__device__ __forceinline__ void ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15, %16};\n\t"
      "tcgen05.wait::st.sync.aligned;" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
      "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}

__device__ __forceinline__ double as_double(uint32_t lo, uint32_t hi) {
  return __hiloint2double((int)hi, (int)lo);
}
__device__ __forceinline__ uint32_t lo_word(double v) { return (uint32_t)__double2loint(v); }
__device__ __forceinline__ uint32_t hi_word(double v) { return (uint32_t)__double2hiint(v); }

}  // namespace tmem
}  // namespace sb200
