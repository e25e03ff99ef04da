// tcgen05 (5th-generation tensor core) primitives for single-CTA kernels:
// tensor-memory allocation, the UMMA shared-memory and instruction
// descriptors, kind::tf32 MMA, commit to an mbarrier and 32x32b loads of the
// TMEM accumulator.  No clusters, no multicast.
#pragma once
#include "bulk.cuh"

namespace fame {
namespace umma {

// Allocate ncols (power of two, >= 32) TMEM columns; the whole warp executes
// it and the base address lands in *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Order tcgen05 operations around a thread barrier.
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory descriptor of a K-major operand in the 128-byte swizzled
// canonical layout: rows of 128 B (32 TF32 values of K), 8-row atoms of 1024 B
// packed along M/N, 16-byte chunk c of row r stored at chunk c ^ (r % 8).  The
// atom base must be 1024-byte aligned; stepping K inside the atom adds the
// byte offset to the start address.
__device__ __forceinline__ uint64_t desc_kmajor_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address, 16-byte units
  d |= (uint64_t)1 << 16;                           // leading byte offset (unused when swizzled)
  d |= (uint64_t)(1024 >> 4) << 32;                 // stride byte offset: atom pitch
  d |= (uint64_t)1 << 46;                           // descriptor version of sm_100
  d |= (uint64_t)2 << 61;                           // layout: 128-byte swizzle
  return d;
}

// Byte offset of element (row, k) (k < 32, 4-byte elements) in such an operand.
// (atom row * 1024 + row-in-atom * 128 is row * 128.)
__host__ __device__ __forceinline__ uint32_t sw128_offset(int row, int k) {
  return (uint32_t)(row * 128 + ((((k >> 2) ^ row) & 7) << 4) + (k & 3) * 4);
}

// Instruction descriptor: D (F32) = A (TF32, K-major) x B (TF32, K-major)^T, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K-step of 8 TF32 values; issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

// Arrive once on bar when every tcgen05 operation this thread issued so far has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 consecutive accumulator columns of the warp's 32 TMEM lanes (lane = thread);
// the values are valid once wait_ld has consumed them.
__device__ __forceinline__ void ld_32x32b_x32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void wait_ld(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                 "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                 "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}

// 16 consecutive accumulator columns of the warp's 32 TMEM lanes, waited on in place.
__device__ __forceinline__ void ld_32x32b_x16_wait(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

// Round to the nearest TF32 value (ties away from zero); low 13 mantissa bits zero.
__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// v ~ big + small with both parts TF32 (relative representation error <= 2^-22).
__device__ __forceinline__ void tf32_split(double v, float& big, float& small) {
  big = tf32_rna((float)v);
  small = tf32_rna((float)(v - (double)big));
}

// The split of an FP32 value (the remainder v - big is exact).
__device__ __forceinline__ void tf32_split_f32(float v, float& big, float& small) {
  big = tf32_rna(v);
  small = tf32_rna(v - big);
}

// The same split rounded directly from FP64: v's significand rounded to 11 bits
// (ties away from zero) on its bit pattern, the exact remainder rounded likewise;
// both parts convert to FP32 exactly (for |v| within the FP32 normal range).
__device__ __forceinline__ double round11(double v) {
  // bit 41 and the cleared bits 0..41 of the pattern: bit 9 / bits 0..9 of the high word, all of the low word
  return __hiloint2double((int)(((unsigned)__double2hiint(v) + 0x200u) & 0xFFFFFC00u), 0);
}
__device__ __forceinline__ void tf32_split_fast(double v, float& big, float& small) {
  const double h = round11(v);
  big = (float)h;
  small = (float)round11(v - h);
}

}  // namespace umma
}  // namespace fame
