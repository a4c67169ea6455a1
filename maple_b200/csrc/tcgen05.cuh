// Fifth-generation tensor core (tcgen05) helpers for sm_100a: shared-memory
// matrix descriptors, instruction descriptors, tensor-memory allocation, MMA
// issue, completion through an mbarrier and tensor-memory loads, as inline
// PTX.  Used by the BF16 convolutions of the learned initial guess (forward,
// data and weight gradients) and the element-batched operator.
//
// Operand layout (K-major, no swizzle).  An operand tile of R rows and K
// columns of 16-bit values is stored as "core matrices" of 8 rows x 16 bytes
// (8 values along K), each 128 contiguous bytes with row i at byte 16*i.
// Within an 8-row group the K-chunks follow each other (128 bytes apart), and
// the 8-row groups follow each other (KB * 128 bytes apart, KB = K / 8):
//   byte(r, k) = (r / 8) * KB * 128 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
// One MMA consumes 16 values of K (two chunks): its descriptor starts at the
// chunk pair, with leading-dimension offset 128 (chunk to chunk along K) and
// stride-dimension offset KB * 128 (8-row group to 8-row group).
#pragma once

#include <cstdint>

namespace maple_tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of (row r, k) in the K-major core-matrix layout above
__host__ __device__ constexpr uint32_t kmajor_offset(int r, int k, int KB) {
  return (uint32_t)((r >> 3) * KB * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all >> 4), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// instruction descriptor of kind::f16 with BF16 A and B, FP32 accumulator,
// each operand K-major (0) or MN-major (1), M x N tile
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N, int b_mn_major = 0, int a_mn_major = 0) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn_major << 15) | ((uint32_t)b_mn_major << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// MN-major operand layout (no swizzle), used for B when N is the contiguous
// dimension in global memory: core matrices of 8 K-rows x 16 bytes (8 values
// along N), 128 contiguous bytes with K-row i at byte 16*i; K-groups of 8 rows
// follow each other at the leading-dimension offset LBO and N-groups of 8 at
// the stride-dimension offset SBO:
//   byte(n, k) = (n / 8) * SBO + (k / 8) * LBO + (k % 8) * 16 + (n % 8) * 2.
__host__ __device__ constexpr uint32_t mnmajor_offset(int n, int k, uint32_t lbo, uint32_t sbo) {
  return (uint32_t)((n >> 3) * sbo + (k >> 3) * lbo + (k & 7) * 16 + (n & 7) * 2);
}

// ---- tensor memory (one warp allocates and frees; ncols a power of 2 >= 32)
__device__ __forceinline__ void tmem_alloc(uint32_t* slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (tensor memory) (+)= A * B^T, one thread issues
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive on the mbarrier once every MMA this thread issued has completed
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for phase `parity` of the mbarrier: true once it completed,
// false after max_polls polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, long long max_polls) {
  const uint32_t a = smem_u32(mbar);
  for (long long i = 0; i < max_polls; ++i) {
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

// 8 consecutive FP32 columns of this thread's tensor-memory lane (warp w of
// the CTA reads lanes 32w..32w+31: taddr must carry lane 32*(w%4))
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace maple_tc
