// umma.cuh -- the sm_100a fifth-generation tensor-core path (tcgen05) for
// small dense layers: shared-memory operand descriptors, the instruction
// descriptor, TMEM allocation, one-thread MMA issue with completion on an
// mbarrier, and the TMEM-to-register loads of the epilogue.
//
// Operands are BF16, K-major, without swizzle: an M x K (or N x K) tile is
// stored as core matrices of 8 rows x 16 bytes (8 elements along K, rows 16
// bytes apart, 128 bytes each); the core matrices of one 8-row group lie
// 128 bytes apart along the rows' direction (SBO) and the two 8-element K
// chunks of one MMA (K = 16) lie LBO = (rows / 8) * 128 bytes apart.  Element
// (r, k) of a tile with R rows sits at byte
//   (k / 8) * (R / 8) * 128 + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
// The fp32 accumulator of an M = 128 MMA holds row m in TMEM lane m and
// column n in TMEM column base + n; warp w of the CTA reads lanes
// 32 (w % 4) .. 32 (w % 4) + 31.
#pragma once
#include <cstdint>

namespace argot {
namespace umma {

// byte offset of element (r, k) in a K-major tile of R rows
__host__ __device__ constexpr uint32_t kmajor_offset(int R, int r, int k) {
  return (uint32_t)((k / 8) * (R / 8) * 128 + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2);
}

// Shared-memory matrix descriptor (sm_100 format): start address, leading
// (K chunk) and stride (8-row group) byte offsets in 16-byte units,
// descriptor version 1 at bits 46-47, no swizzle (layout type 0 at bits
// 61-63), base offset 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B (K-major), fp32
// accumulator, M x N: c_format 1 (bits 4-5), a_format 1 (bits 7-9),
// b_format 1 (bits 10-12), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// TMEM columns for the CTA (one warp, all lanes); the address lands in *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

// The mbarrier completes one phase when every MMA issued before by this
// thread has completed.
__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the phase with the given parity to complete, at most `limit`
// polls (each poll may suspend the thread for a while); false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t i = 0; i < limit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor cores
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  // the load and its wait in one statement, so that no use of the
  // registers can be scheduled between them
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace argot
