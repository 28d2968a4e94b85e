// Minimal sm_100a tensor-core (tcgen05 / UMMA) toolkit used by the closure MLP kernels: TMEM
// allocation, BF16 x BF16 -> FP32 MMA from shared-memory descriptors (no swizzle, K-major operands),
// completion through an mbarrier with a bounded wait, and TMEM -> register loads.
//
// Operand layout ("K-major, no swizzle" canonical UMMA layout): an R x K BF16 tile is stored as 8 x 8
// core matrices of 128 contiguous bytes (8 rows of 16 bytes); core matrix (r/8, k/8) sits at byte
// ((r/8) * (K/8) + k/8) * 128.  The leading-dimension byte offset (next core matrix along K) is
// therefore 128 and the stride-dimension byte offset (next 8-row group) K/8 * 128; one MMA consumes
// K = 16, i.e. two core matrices along K, and the next K step starts 256 bytes further.
#pragma once

#include <cstdint>

namespace cruna {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// element index of (row r, column k) in an R x K tile of the layout above
__host__ __device__ __forceinline__ int kmaj(int r, int k, int K) {
  return (((r >> 3) * (K >> 3) + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}

// shared-memory matrix descriptor (SWIZZLE_NONE, version 1, base offset 0)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// descriptor of K-step s (16 columns) of an R x K tile at saddr
__device__ __forceinline__ uint64_t tile_desc(uint32_t saddr, int K, int s) {
  return sdesc(saddr + (uint32_t)s * 256u, 128u, (uint32_t)(K >> 3) * 128u);
}

// instruction descriptor: kind::f16, A = B = BF16, D = FP32, both operands K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K = 16 step; issued by a single thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// D = A(R_A x K) * B(N x K)^T accumulated over K / 16 steps
__device__ __forceinline__ void gemm_bf16(uint32_t tmem_d, uint32_t a_saddr, uint32_t b_saddr, int K, int N,
                                          bool accumulate_first) {
  const uint32_t id = idesc_bf16(128, N);
  for (int s = 0; s < K / 16; ++s)
    mma_bf16(tmem_d, tile_desc(a_saddr, K, s), tile_desc(b_saddr, K, s), id,
             (s > 0 || accumulate_first) ? 1u : 0u);
}

__device__ __forceinline__ void commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait on the phase `parity` of an mbarrier; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, long long max_iter) {
  const uint32_t a = smem_addr(mbar);
  for (long long i = 0; i < max_iter; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// whole warp: allocate ncols (power of two >= 32) TMEM columns, address written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32*(w%4) .. +31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace cruna
