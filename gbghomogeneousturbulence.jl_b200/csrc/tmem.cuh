// Tensor memory (TMEM) as per-thread storage on sm_100a: allocation, release and 32-bit loads and
// stores of the 32x32b shape, in inline PTX (tcgen05.*).
//
// TMEM holds 128 lanes × 512 columns of 32-bit words per SM. Warp w of a CTA reaches lanes
// 32·(w mod 4) .. 32·(w mod 4) + 31; with the 32x32b shape, thread i of the warp reads and writes
// lane 32·(w mod 4) + i, so every thread owns a private row of columns. A TMEM address is
// (lane << 16) | column.
//
// Every tcgen05 instruction here is warp-collective (.sync.aligned): the whole warp executes it
// with the same address. A CTA allocates once at its start and frees before it exits; an
// allocation waits while the SM's other CTAs hold the columns it asks for, and they free them when
// they finish, so the wait always ends.
#pragma once

#include <cstdint>

#include "tma.cuh"

namespace gbght {

#if defined(__CUDACC__) && !defined(GBGHT_EMU)

// One warp allocates `ncols` columns (a power of two in [32, 512]) and writes the base address
// to shared memory at `slot`.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// Order TMEM accesses across a CTA barrier.
__device__ __forceinline__ void tmem_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_st2(uint32_t taddr, uint32_t a, uint32_t b) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(a), "r"(b) : "memory");
}
__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(a), "r"(b), "r"(c),
               "r"(d)
               : "memory");
}
// Wait until this thread's earlier stores have landed (before it loads them back).
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Loads complete inside the same asm statement (load, then wait::ld), so no use of the
// destination registers can be scheduled before the data has arrived.
__device__ __forceinline__ void tmem_ld2(uint32_t taddr, uint32_t (&r)[2]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
      : "r"(taddr)
      : "memory");
}
// Three 2-word or 4-word loads at independent addresses, one wait.
__device__ __forceinline__ void tmem_ld2x3(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t (&r)[6]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%6];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%2, %3}, [%7];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%4, %5}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5])
      : "r"(a0), "r"(a1), "r"(a2)
      : "memory");
}
__device__ __forceinline__ void tmem_ld4x3(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t (&r)[12]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%12];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%4, %5, %6, %7}, [%13];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%8, %9, %10, %11}, [%14];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
      : "r"(a0), "r"(a1), "r"(a2)
      : "memory");
}

#endif

}  // namespace gbght
