// Tensor-core ModUp contraction (tcgen05.mma kind::i8 on sm_100a).
//
// ModUp raises each partition's mixed-radix digits d_0 .. d_{a-1} to every limb j of
// the extended chain (core_key_switch.cpp:92-108): the reference's chain of
// REDC(d_i * C_ij) terms (C_0j = R^2, C_ij the partition's product constants) has
// the value sum_i d_i C_ij R^-1 modulo q_j.  The extended limbs feed only
// value-only consumers (the forward NTT in Harvey's form, the key inner product,
// ModDown's reduced inverse transform), so any representative in [0, 2q_j) of that
// value gives the reference's final words.  Here:
//   * A holds the 8 little-endian bytes d_i[a] of every digit (K = 8a bytes);
//   * B (per moduli id and partition, built on the host) holds, for 16 targets per
//     MMA round, the 8 bytes of e_iaj = C_ij 2^(8a) mod q_j, so the 8 exact partial
//     sums D_b = sum_(i,a) d_i[a] e_iaj[b] (each below 2^23) give
//     X_j = sum_b D_b 2^(8b) = sum_(i,a) d_i[a] e_iaj == sum_i d_i C_ij (mod q_j),
//     with X_j below 2^80;
//   * one REDC of X_j on the CUDA cores leaves a word below q_j + 2^18 < 2 q_j.
// A coefficient with a digit of 2^61 or more takes the reference's chain term by
// term.  The values equal mod_up_contract_kernel's.
#include "kernels.cuh"
#include "modarith.cuh"
#include "params.hpp"
#include "umma.cuh"

namespace fhe_b200 {

namespace {

using namespace umma;

constexpr int digit_row_bytes(int A) { return (8 * A + 31) / 32 * 32; }
template <int A>
__global__ void __launch_bounds__(kTcThreads, 4)
    mod_up_tc_kernel(PrimeTables t, DevicePartitions dp, ModUpTcTables tc, int n, int moduli_id,
                     const int64_t *digits, int64_t *ext, TcStatus status, bool skip_own) {
  constexpr int KB = digit_row_bytes(A);
  const int p = blockIdx.y;
  if (dp.size[p] != A) return;  // uniform per CTA, before any barrier
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t *sA = smem;                                               // [128][KB]
  uint8_t *sB = smem + kTcCoeffs * KB;                              // one round: [128][KB]
  int64_t *sd = reinterpret_cast<int64_t *>(sB + kTcColumns * KB);  // [A][128] digits
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ int fast[kTcCoeffs];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int coeff0 = blockIdx.x * kTcCoeffs;
  const int start = dp.start[p];
  const int E = dp.extended;

  // 1. Digits of one coefficient per thread: the A row, a copy for the quotients.
  if (tid < kTcCoeffs) {
    uint64_t w[KB / 8];
#pragma unroll
    for (int i = 0; i < KB / 8; i++) w[i] = 0;
    bool ok = true;
#pragma unroll
    for (int i = 0; i < A; i++) {
      const int64_t d = digits[static_cast<long long>(start + i) * n + coeff0 + tid];
      ok = ok && redc_operand_ok(d);
      w[i] = static_cast<uint64_t>(d);
      sd[i * kTcCoeffs + tid] = d;
    }
    fast[tid] = ok;
#pragma unroll
    for (int ch = 0; ch < KB / 16; ch++) {
      const uint4 v = make_uint4(static_cast<uint32_t>(w[2 * ch]), static_cast<uint32_t>(w[2 * ch] >> 32),
                                 static_cast<uint32_t>(w[2 * ch + 1]),
                                 static_cast<uint32_t>(w[2 * ch + 1] >> 32));
      *reinterpret_cast<uint4 *>(sA + core_offset(tid, ch * 16, kTcCoeffs)) = v;
    }
  }
  if (warp == 0) tmem_alloc(&tmem_base);
  if (tid == 0) mbar_init(&mbar);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t bar = smem_addr(&mbar);

  const int lane_base = (warp & 3) * 32;
  const int row = lane_base + lane;
  const int half = warp >> 2;
  const int64_t *cst = dp.product_r_squared + static_cast<long long>(p) * 16 * E;
  const uint8_t *bp = tc.b + tc.b_offset[p];
  int64_t *out = ext + static_cast<long long>(p) * E * n + coeff0 + row;
  bool ok = true;
  int round = 0;
  for (; round < tc.rounds; round++) {
    {
      constexpr int chunks = kTcColumns * KB / 16;
      const uint4 *src = reinterpret_cast<const uint4 *>(bp) + static_cast<size_t>(round) * chunks;
      uint4 *dst = reinterpret_cast<uint4 *>(sB);
      for (int i = tid; i < chunks; i += kTcThreads) dst[i] = src[i];
      fence_async_smem();
      __syncthreads();
    }
    if (tid == 0) {
      mma_round(tmem, sA, sB, KB);
      mma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, round & 1, status.wait_limit)) != 0;
    if (!ok) break;
    tc_fence_after();
    // Each warpgroup folds 8 of the round's 16 targets, two per tensor-memory load.
    for (int jp = half * (kTcTargets / 2); jp < (half + 1) * (kTcTargets / 2); jp += 2) {
      const int j0 = round * kTcTargets + jp;
      if (j0 >= E) break;  // uniform across the warp
      uint32_t d[16];
      tmem_load16(tmem + (static_cast<uint32_t>(lane_base) << 16) + jp * 8, d);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = j0 + h;
        if (j >= E) break;  // uniform across the warp
        if (skip_own && j >= start && j < start + A) continue;  // uniform across the warp
        const int prime = moduli_id + j;
        const uint64_t q = t.q[prime], kq = t.k[prime];
        if (fast[row]) {
          uint64_t lo, hi;
          fold8(d + 8 * h, lo, hi);
          out[static_cast<long long>(j) * n] = redc_wide(lo, hi, q, kq);
        } else {
          // The reference's chain term by term (mod_up_contract_kernel's slow path).
          const int64_t q2 = static_cast<int64_t>(q << 1);
          int64_t v = mont_mult(sd[row], t.r_squared[prime], q, kq);
#pragma unroll
          for (int i = 1; i < A; i++)
            v = guard(mont_mult(sd[i * kTcCoeffs + row], cst[(i - 1) * E + j], q, kq) + v, q2);
          out[static_cast<long long>(j) * n] = v;
        }
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (!ok) {
    if (tid == 0) atomicExch(status.error, 1);
    if (warp == 0) mbar_wait(bar, round & 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem);
}

size_t mod_up_tc_smem(int A) {
  const int kb = digit_row_bytes(A);
  return static_cast<size_t>(kTcCoeffs) * kb * 2 + static_cast<size_t>(A) * kTcCoeffs * 8;
}

}  // namespace

bool mod_up_tc_supported(int max_size, int n) {
  return max_size >= 1 && max_size <= 16 && n >= kTcCoeffs && n % kTcCoeffs == 0;
}

ModUpTcHost make_mod_up_tc_tables(const std::vector<uint64_t> &q,
                                  const std::vector<int64_t> &r_squared, int moduli_id,
                                  int extended, const std::vector<Partition> &parts,
                                  const std::vector<PartitionConstants> &constants) {
  using u128 = unsigned __int128;
  ModUpTcHost h;
  const int E = extended;
  h.rounds = (E + kTcTargets - 1) / kTcTargets;
  for (size_t p = 0; p < parts.size(); p++) {
    const int A = parts[p].size;
    const int kb = digit_row_bytes(A);
    h.b_offset.push_back(static_cast<long long>(h.b.size()));
    h.b.resize(h.b.size() + static_cast<size_t>(h.rounds) * kTcColumns * kb, 0);
    uint8_t *b = h.b.data() + h.b_offset.back();
    for (int j = 0; j < E; j++) {
      const uint64_t qj = q[moduli_id + j];
      uint8_t *round = b + static_cast<size_t>(j / kTcTargets) * kTcColumns * kb;
      const int jl = j % kTcTargets;
      for (int i = 0; i < A; i++) {
        const uint64_t c = i == 0 ? static_cast<uint64_t>(r_squared[moduli_id + j])
                                  : static_cast<uint64_t>(
                                        constants[p].product_r_squared[static_cast<size_t>(i - 1) * E + j]);
        uint64_t e = c % qj;  // C_ij 2^(8a) mod q_j for a = 0, 1, ...
        for (int a = 0; a < 8; a++) {
          for (int bb = 0; bb < 8; bb++)
            round[core_offset(jl * 8 + bb, i * 8 + a, kTcColumns)] = static_cast<uint8_t>(e >> (8 * bb));
          e = static_cast<uint64_t>((static_cast<u128>(e) << 8) % qj);
        }
      }
    }
  }
  return h;
}

cudaError_t launch_mod_up_contract_tc(const PrimeTables &t, const DevicePartitions &dp,
                                      const ModUpTcTables &tc, int n, int moduli_id,
                                      const int64_t *digits, int64_t *ext, const TcStatus &status,
                                      cudaStream_t s, bool skip_own) {
  if (!mod_up_tc_supported(dp.max_size, n) || tc.b == nullptr || status.error == nullptr ||
      tc.rounds != (dp.extended + kTcTargets - 1) / kTcTargets)
    return cudaErrorInvalidValue;
  static int raised[17] = {};
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  const int bit = 1 << (device & 31);
  const dim3 grid(n / kTcCoeffs, dp.count);
  for (int size = 1; size <= 16; size++) {
    if (!(dp.size_mask & (1u << size))) continue;
    switch (size) {
#define FHE_UP_CASE(AA)                                                                           \
  case AA:                                                                                        \
    if (!(raised[AA] & bit)) {                                                                    \
      e = cudaFuncSetAttribute(mod_up_tc_kernel<AA>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                               static_cast<int>(mod_up_tc_smem(16)));                             \
      if (e != cudaSuccess) return e;                                                             \
      raised[AA] |= bit;                                                                          \
    }                                                                                             \
    note_launch();                                                                                \
    mod_up_tc_kernel<AA><<<grid, kTcThreads, mod_up_tc_smem(AA), s>>>(t, dp, tc, n, moduli_id,    \
                                                                      digits, ext, status, skip_own); \
    break;
      FHE_UP_CASE(1) FHE_UP_CASE(2) FHE_UP_CASE(3) FHE_UP_CASE(4) FHE_UP_CASE(5) FHE_UP_CASE(6)
      FHE_UP_CASE(7) FHE_UP_CASE(8) FHE_UP_CASE(9) FHE_UP_CASE(10) FHE_UP_CASE(11) FHE_UP_CASE(12)
      FHE_UP_CASE(13) FHE_UP_CASE(14) FHE_UP_CASE(15) FHE_UP_CASE(16)
#undef FHE_UP_CASE
      default: return cudaErrorInvalidValue;
    }
  }
  return cudaGetLastError();
}

}  // namespace fhe_b200
