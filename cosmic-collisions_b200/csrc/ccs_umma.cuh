// ccs_umma.cuh -- the few sm_100a tensor-core pieces the learned correction
// uses: shared-memory matrix descriptors, the instruction descriptor of a
// BF16 x BF16 -> FP32 tcgen05.mma, tensor-memory allocation and loads, and a
// bounded mbarrier wait.
//
// Operand layout: K-major with no swizzle.  An R x K BF16 operand is stored as
// 8-row x 16-byte core matrices (8 rows of 8 consecutive K elements, 128
// contiguous bytes); the core matrices of one 8-row group follow each other
// along K (leading byte offset 128) and the groups follow each other every
// K/8 x 128 bytes (stride byte offset).  One MMA consumes K = 16, i.e. two core
// matrices per row group, so the k-th step starts 256 bytes further on.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace ccs {
namespace umma {

__host__ __device__ constexpr uint32_t canon(int r, int k, int K) {
  return (uint32_t)((((r >> 3) * (K >> 3) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: start address, leading / stride byte offsets (all >> 4),
// the sm_100 descriptor version (1) at bit 46, base offset 0, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, int K) {
  const uint64_t lbo = 128, sbo = (uint64_t)(K >> 3) * 128;
  return (uint64_t)((addr >> 4) & 0x3FFFu) | (((lbo >> 4) & 0x3FFFu) << 16) | (((sbo >> 4) & 0x3FFFu) << 32) |
         ((uint64_t)1 << 46);
}

// instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive on the mbarrier once every MMA this thread issued before has completed
__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" : : : "memory");
}

// wait for the phase with the given parity to complete; gives up after `limit` polls
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" : : : "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" : : : "memory"); }
// generic-proxy writes to shared memory become visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" : : : "memory"); }

// warp-wide: the column count is a power of two >= 32; the address lands in *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :
               : "r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" : : : "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's lane (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// completes the loads issued before it; the registers are threaded through so no use moves above it
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15])
               :
               : "memory");
}

// n columns (a multiple of 16) of this thread's lane into v
template <int n>
__device__ __forceinline__ void tmem_load(uint32_t taddr, float (&v)[n]) {
  static_assert(n % 16 == 0, "16-column loads");
  uint32_t r[n / 16][16];
#pragma unroll
  for (int c = 0; c < n / 16; ++c) tmem_ld16(taddr + 16 * c, r[c]);
#pragma unroll
  for (int c = 0; c < n / 16; ++c) tmem_wait16(r[c]);
#pragma unroll
  for (int c = 0; c < n / 16; ++c)
#pragma unroll
    for (int k = 0; k < 16; ++k) v[16 * c + k] = __uint_as_float(r[c][k]);
}

__device__ __forceinline__ uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_value(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
__device__ __forceinline__ uint32_t pack2(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

}  // namespace umma
}  // namespace ccs
