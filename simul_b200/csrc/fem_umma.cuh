// Blackwell tensor-core helpers (tcgen05 / TMEM) for the BF16 dense layers
// of the learned preconditioner.
//
// Operands live in shared memory in the canonical K-major, no-swizzle layout:
// 8-row x 8-element (16-byte) core matrices of 128 contiguous bytes, the
// k-chunks of a row group adjacent (leading byte offset 128 B) and row groups
// kext * 16 B apart (stride byte offset).  One tcgen05.mma consumes K = 16
// (two k-chunks); the next K-step starts 256 B further.  Accumulators are
// FP32 in TMEM: row m of an M = 128 tile is TMEM lane m, column n is column
// base + n.  Warp w of the CTA reads lanes 32 (w % 4) .. + 31.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace femb200 {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (row, k) in a K-major canonical tile with K extent kext
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int kext) {
  return (uint32_t)((row >> 3) * (kext * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: K-major, no swizzle, version 1 (sm_100)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, int kext) {
  const uint64_t lbo = 128u >> 4;
  const uint64_t sbo = (uint64_t)(kext * 16) >> 4;
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((lbo & 0x3FFFu) << 16) | ((sbo & 0x3FFFu) << 32) |
         (1ull << 46);
}

// instruction descriptor, kind::f16: A = B = BF16, D = FP32, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// instruction descriptor, kind::tf32: A = B = TF32 (FP32 words in shared
// memory, low mantissa bits ignored), D = FP32; a_mn / b_mn: the operand is
// MN-major instead of K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// shared-memory matrix descriptor, no swizzle, version 1 (sm_100), with
// explicit leading / stride byte offsets.  K-major: lbo = the offset between
// the two 16-byte k-chunks an MMA reads, sbo = between 8-row groups.
// MN-major: sbo = between 16-byte MN chunks, lbo = between 8-deep k groups.
__device__ __forceinline__ uint64_t smem_desc_lbo_sbo(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// Waits for phase `parity` of the barrier; gives up after max_polls polls
// and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, int max_polls) {
  const uint32_t a = smem_u32(mbar);
  for (int i = 0; i < max_polls; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// After a completion wait that gave up, the MMA may still be writing the
// TMEM columns: wait once more, again bounded, before they are freed.
__device__ __forceinline__ void drain_mma(uint64_t* mbar, uint32_t parity, bool ok, int max_polls) {
  if (!ok) (void)mbar_wait(mbar, parity, max_polls);
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// whole warp: allocate ncols (power of two >= 32) TMEM columns, address to *dst
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
      "%13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// TMEM address of (lane, column) relative to an allocation base
__device__ __forceinline__ uint32_t taddr(uint32_t base, int lane, int col) {
  return base + ((uint32_t)lane << 16) + (uint32_t)col;
}

}  // namespace umma
}  // namespace femb200
