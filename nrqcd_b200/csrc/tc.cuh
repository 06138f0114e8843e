// Minimal tcgen05 (5th-generation tensor core) helpers for sm_100a: tensor
// memory allocation, BF16 x BF16 -> FP32 MMAs on shared-memory operands in
// the no-swizzle K-major canonical layout, commit to an mbarrier, and loads
// of the FP32 accumulator from tensor memory.  Inline PTX per the PTX ISA
// (tcgen05 instructions, shared memory matrix descriptor, instruction
// descriptor for .kind::f16).
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace nrq {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of element (r, k) of an R x K BF16 operand tile stored as
// 8 x 8 core matrices (8 rows of 16 bytes each, 128 contiguous bytes): core
// matrices of one 8-element K chunk are contiguous along the rows, chunks
// follow each other.  Leading byte offset (next K chunk) = R * 16 bytes,
// stride byte offset (next 8-row group) = 128 bytes.
__host__ __device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int R) {
  return ((uint32_t)((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((uint32_t)(r & 7) << 4) + ((uint32_t)(k & 7) << 1);
}

// Shared memory matrix descriptor of K step s (16 BF16 elements = 2 chunks)
// of such a tile at shared address `saddr` (16-byte aligned).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, int R, int s) {
  const uint32_t start = saddr + (uint32_t)s * 2u * (uint32_t)R * 16u;
  uint64_t d = 0;
  d |= (uint64_t)((start >> 4) & 0x3FFFu);                     // bits 0-13  start address >> 4
  d |= (uint64_t)((((uint32_t)R * 16u) >> 4) & 0x3FFFu) << 16;  // bits 16-29 leading byte offset >> 4
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 32;                // bits 32-45 stride byte offset >> 4
  d |= (uint64_t)1 << 46;                                      // bits 46-47 descriptor version 1
  return d;                                                    // base offset 0, no swizzle
}

// Instruction descriptor: D F32 (bits 4-5 = 1), A BF16 (bits 7-9 = 1), B BF16
// (bits 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---- tensor memory allocation (one full warp) ----
__device__ __forceinline__ void tmem_alloc(uint32_t *slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- MMA (one thread) ----
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}
// arrive on the mbarrier when every MMA this thread issued has completed
__device__ __forceinline__ void mma_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// make generic-proxy shared memory writes visible to the tensor core
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// ---- mbarrier ----
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false once `max_spins` polls failed (the caller records the
// failure and skips the dependent work).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t max_spins) {
  for (uint32_t i = 0; i < max_spins; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// ---- tensor memory -> registers: 32 lanes x 16 columns of 32 bits ----
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
// address of (lane, column) in the allocation starting at `base`
__device__ __forceinline__ uint32_t tmem_addr(uint32_t base, int lane, int col) {
  return base + ((uint32_t)lane << 16) + (uint32_t)col;
}

}  // namespace tc
}  // namespace nrq
