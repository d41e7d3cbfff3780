// tc.cuh -- fifth-generation tensor-core primitives (sm_100a): tensor memory,
// shared-memory matrix descriptors, single-CTA tcgen05.mma of kind::tf32,
// commit to an mbarrier, and bounded waits.
//
// Operand layout (K-major, no swizzle): a matrix of R rows (M or N) and Kp
// columns (Kp a multiple of 8 tf32 values) is stored as 8-row x 16-byte core
// matrices; element (r, k) sits at byte
//   (r / 8) * SBO + (k / 4) * 128 + (r % 8) * 16 + (k % 4) * 4,   SBO = Kp * 32,
// so the core matrices of one 8-row group are contiguous along K (leading byte
// offset 128) and one MMA of K = 8 starts (k0 / 4) * 128 bytes into the matrix.
// The accumulator D (M = 128 rows, fp32) lives in tensor memory: row i is
// lane i, column j is column base + j; warp w of the CTA reads lanes 32 (w % 4) ..
// 32 (w % 4) + 31.
#pragma once

#include <cstdint>

namespace fmmb {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) in a K-major operand of kp columns
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int kp) {
  return (uint32_t)((r >> 3) * (kp * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// shared-memory matrix descriptor: start address, leading byte offset 128,
// stride byte offset sbo (both >> 4), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)(128u >> 4) << 16;
  d |= (uint64_t)((sbo_bytes & 0x3FFFFu) >> 4) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;                // base offset 0, lbo mode 0, layout type 0 (no swizzle)
}

// instruction descriptor of kind::tf32, fp32 accumulator, A and B K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4)                      // D format f32
         | (2u << 7) | (2u << 10)       // A, B format tf32
         | ((uint32_t)(N >> 3) << 17)   // N / 8
         | ((uint32_t)(M >> 4) << 24);  // M / 16
}

// D (tensor memory) (+)= A (smem) x B (smem)^T, issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

// the mbarrier completes one phase when every MMA issued so far by this thread is done
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// waits for the phase of the given parity; gives up after `limit` polls (false)
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_test(mbar, parity)) return true;
  return false;
}

// generic-proxy shared-memory writes made visible to the tensor cores (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// one full warp: allocate ncols (power of two >= 32) columns, address written to smem
__device__ __forceinline__ void tmem_alloc(uint32_t dst_saddr, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_saddr), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive fp32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// x = big + small with big exactly representable in tf32 (3xTF32 products:
// big*big + big*small + small*big)
__device__ __forceinline__ void split_tf32(float x, float& big, float& small) {
  uint32_t b;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b) : "f"(x));
  big = __uint_as_float(b);
  small = x - big;
}

}  // namespace tc
}  // namespace fmmb
