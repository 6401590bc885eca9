// Asynchronous copies global -> shared memory of this CTA by the TMA engine:
// contiguous bulk copies (cp.async.bulk) and 3-D box copies described by a
// tensor map (cp.async.bulk.tensor), completed on an mbarrier, with bounded
// waits. Sources are this GPU's own memory; no multicast.
#pragma once
#include <cstdint>

namespace fe {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// One-thread set-up of a transaction barrier expecting one arrival per phase.
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// The arrival of this phase, announcing `bytes` of copies that complete it.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// A hint: bytes (a multiple of 16) of global memory at src (16-byte
// aligned) brought into L2 by the copy engine; nothing waits for it.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// bytes (a multiple of 16) from global src to shared dst, both 16-byte
// aligned; completion is counted on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// The box at element coordinates (x, y, z) of the 3-D tensor `tmap` (a
// CUtensorMap in global memory) to shared dst (128-byte aligned), counted on
// bar. x times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_box3(void* dst, const void* tmap, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Wait for the phase of parity `parity` to complete, at most `tries` polls
// (each may suspend the thread for a short, hardware-defined time). False
// when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int tries) {
  const uint32_t a = smem_u32(bar);
  for (int t = 0; t < tries; ++t) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace fe
