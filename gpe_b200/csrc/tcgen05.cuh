// tcgen05.cuh -- 5th-generation tensor core (tcgen05) and TMEM wrappers for
// sm_100a, written from the PTX ISA's instruction and descriptor formats.
//
// Shared-memory matrix descriptor (64 bit), no-swizzle ("interleave") form:
//   bits  0-13  start address >> 4
//   bits 16-29  leading-dimension byte offset >> 4 (LBO)
//   bits 32-45  stride-dimension byte offset >> 4 (SBO)
//   bits 46-47  descriptor version (1 on sm_100)
//   bits 61-63  layout / swizzle mode (0 = none)
// K-major operand: 8-row x 16-byte core matrices; SBO = stride between
// 8-row groups along M/N, LBO = stride between the two 16-byte K halves of
// a K=16 (bf16) step.  MN-major operand: core matrix = 8 K-rows of 16 bytes
// (8 M/N elements each); SBO = stride between 8-element M/N groups, LBO =
// stride between 8-row K groups.
//
// Instruction descriptor (32 bit) of kind::f16:
//   bits 4-5 D format (1 = f32), 7-9 A format (1 = bf16), 10-12 B format,
//   bit 15 A major (0 = K, 1 = MN), bit 16 B major, 17-22 N >> 3,
//   24-28 M >> 4.
#pragma once

#include <cstdint>

namespace gpe {
namespace tc {

__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo,
                                                 uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) |
         ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N, bool a_mn,
                                                      bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) |
         ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// Allocate ncols TMEM columns (power of two >= 32); the base address is
// written to shared memory at holder.  Whole warp.
__device__ __forceinline__ void tmem_alloc(uint32_t holder_saddr, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               ::"r"(holder_saddr), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
               ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one thread issues.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc,
                                         uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive once on the mbarrier when every tcgen05 operation this thread has
// issued so far has completed.
__device__ __forceinline__ void commit(uint32_t mbar_saddr) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
      ::"r"(mbar_saddr) : "memory");
}

// 32 lanes x 16 columns of 32-bit values: this thread's lane, 16 columns.
__device__ __forceinline__ void ld_32x32b_x16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
        "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
        "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 2 columns: this thread's lane, columns 0-1 into v[0], v[1].
__device__ __forceinline__ void ld_32x32b_x2(uint32_t taddr, float (&v)[16]) {
  uint32_t r0, r1;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];"
               : "=r"(r0), "=r"(r1) : "r"(taddr) : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  v[0] = __uint_as_float(r0);
  v[1] = __uint_as_float(r1);
}
__device__ __forceinline__ void st_32x32b_x2_zero(uint32_t taddr) {
  const uint32_t z = 0;
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1,%1};" ::"r"(taddr), "r"(z)
               : "memory");
}

// Zero 32 lanes x 16 columns (this thread's lane).  Complete with wait_st.
__device__ __forceinline__ void st_32x32b_x16_zero(uint32_t taddr) {
  const uint32_t z = 0;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
      "{%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};"
      ::"r"(taddr), "r"(z) : "memory");
}
__device__ __forceinline__ void wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// 1-D bulk copy global -> this CTA's shared memory (no multicast); both
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(uint32_t dst_saddr, const void* src, uint32_t bytes,
                                          uint32_t mbar_saddr) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(dst_saddr), "l"(src), "r"(bytes), "r"(mbar_saddr)
      : "memory");
}

}  // namespace tc
}  // namespace gpe
