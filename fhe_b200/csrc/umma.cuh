// Building blocks of the INT8 tensor-core contractions (tcgen05 on sm_100a): UMMA
// shared-memory descriptors for K-major operands without swizzle, the kind::i8 MMA
// issued by one thread, tensor-memory loads, and a bounded mbarrier wait.  The
// forms are those of the PTX ISA for tcgen05 (the same strings CUTLASS's sm100
// atoms emit).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace fhe_b200 {
namespace umma {

// The shape both contractions use: a CTA owns 128 coefficients (the MMA's M and the
// tensor-memory lanes) with two warpgroups; one MMA round covers 16 target limbs x 8
// byte columns = 128 columns (the MMA's N and the tensor-memory columns).
constexpr int kTcCoeffs = 128;
constexpr int kTcThreads = 256;  // warp w reads tensor-memory lanes 32 (w % 4) ...
constexpr int kTcTargets = 16;
constexpr int kTcColumns = 128;
constexpr uint32_t kTcWaitLimit = 1u << 22;
// Instruction descriptor of tcgen05.mma kind::i8: U8 x U8 -> S32, both K-major.
constexpr uint32_t kTcIdesc = (2u << 4) | (static_cast<uint32_t>(kTcColumns >> 3) << 17) |
                              (static_cast<uint32_t>(kTcCoeffs >> 4) << 24);

// Byte offset of element (row, k) of a K-major operand of `rows` rows stored as
// UMMA core matrices (8 rows x 16 bytes): [k / 16][row / 8][row % 8][k % 16].
__host__ __device__ inline int core_offset(int row, int k, int rows) {
  return ((k / 16) * (rows / 8) + row / 8) * 128 + (row % 8) * 16 + (k % 16);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major without swizzle; lbo = bytes between the
// two 16-byte halves of a 32-byte K step, sbo = bytes between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFF) |
         (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(addr), "r"(parity)
      : "memory");
  return done != 0;
}

// Polls the mbarrier phase at most `limit` times (0: gives up at once).
__device__ inline bool mbar_wait(uint32_t addr, uint32_t parity, uint32_t limit = kTcWaitLimit) {
  for (uint32_t i = 0; i < limit; i++)
    if (mbar_try_wait(addr, parity)) return true;
  return false;
}

__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void tmem_load16(uint32_t addr, uint32_t (&d)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
        "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]),
        "=r"(d[14]), "=r"(d[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot) {  // one whole warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(slot)),
               "r"(kTcColumns));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t tmem) {  // the allocating warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
               "r"(kTcColumns));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(1));
}

// Arrives on the mbarrier once every MMA issued so far by this thread completes.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

// Shared-memory writes of the generic proxy become visible to the MMA (async proxy).
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// D (128 x 128, S32) = A (128 x kb bytes) x B (128 x kb bytes)^T, both K-major core
// matrices in shared memory; one thread issues the kb / 32 K steps.
__device__ __forceinline__ void mma_round(uint32_t tmem, const uint8_t *a, const uint8_t *b,
                                          int kb) {
  for (int k = 0; k < kb / 32; k++) {
    const uint64_t da = umma_desc(smem_addr(a) + k * 2 * (kTcCoeffs / 8) * 128,
                                  (kTcCoeffs / 8) * 128, 128);
    const uint64_t db = umma_desc(smem_addr(b) + k * 2 * (kTcColumns / 8) * 128,
                                  (kTcColumns / 8) * 128, 128);
    mma_i8(tmem, da, db, kTcIdesc, k > 0 ? 1u : 0u);
  }
}

// X = sum_b D_b 2^(8b) of 8 partial sums below 2^24 (byte columns 0-7), as a
// 128-bit word below 2^81.
__device__ __forceinline__ void fold8(const uint32_t *dv, uint64_t &lo, uint64_t &hi) {
  const uint64_t low = static_cast<uint64_t>(dv[0]) + (static_cast<uint64_t>(dv[1]) << 8) +
                       (static_cast<uint64_t>(dv[2]) << 16) + (static_cast<uint64_t>(dv[3]) << 24) +
                       (static_cast<uint64_t>(dv[4]) << 32);  // below 2^57
  const uint64_t a5 = static_cast<uint64_t>(dv[5]) << 40;     // below 2^64
  const uint64_t a6 = static_cast<uint64_t>(dv[6]) << 48, a7 = static_cast<uint64_t>(dv[7]) << 56;
  uint64_t l = low + a5;
  uint64_t carry = l < low ? 1 : 0;
  uint64_t l2 = l + a6;
  carry += l2 < l ? 1 : 0;
  l = l2 + a7;
  carry += l < l2 ? 1 : 0;
  lo = l;
  hi = (static_cast<uint64_t>(dv[6]) >> 16) + (static_cast<uint64_t>(dv[7]) >> 8) + carry;
}

}  // namespace umma
}  // namespace fhe_b200
