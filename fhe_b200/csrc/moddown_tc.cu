// Tensor-core ModDown epilogue (tcgen05.mma kind::i8 on sm_100a).
//
// The reference divides every normal limb by the special primes one after another
// (core_key_switch.cpp:123-160).  Unrolled, limb j of a coefficient becomes
//   v_j = x_j * prod_s pinv_s - sum_s d_s * prod_{t>=s} pinv_t   (mod q_j),
// where d_s is the divisor of step s (special limb K-1-s after s divisions) and
// pinv_s the step's inverse special prime modulo q_j; its final make_unsigned
// leaves v_j canonical in [0, q_j), so any exact evaluation gives the same word.
// Here the sum over s runs on the INT8 tensor pipe:
//   * A (128 coefficients x kb bytes): the 8 little-endian bytes of every d_s as an
//     unsigned word, then one byte [d_s < 0] per divisor (a negative d_s read as
//     unsigned is d_s + 2^64, which the sign byte takes back);
//   * B (per moduli id, built on the host): for target j, the 8 bytes of
//     e_saj = w'_sj 2^(8a) R mod q_j against byte a of d_s, where
//     w'_sj = -prod_{t>=s} pinv_t mod q_j, and of z_sj = -2^64 w'_sj R mod q_j
//     against the sign byte of d_s;
//   * D (tensor memory, S32): 8 columns per target, column b = the exact partial sum
//     of byte b of the constants (each below 2^24), so X_j = sum_b D_b 2^(8b) is
//     congruent to R sum_s d_s w'_sj and below 2^81; one MMA round covers 16
//     targets, so a CTA holds 128 tensor-memory columns and the B of one round, and
//     four CTAs fit on an SM.
// The epilogue folds the 8 partial sums into a 128-bit word, takes one REDC of it
// (a word below q_j + 2^19), adds x_j prod pinv (one Montgomery product) and
// reduces the total (below 4 q_j) to [0, q_j).
// The divisor triangle (K(K-1)/2 divisions per coefficient) stays on the CUDA
// cores, as in the CUDA-core form.
#include <cstring>
#include <vector>

#include "epilogue.cuh"
#include "kernels.cuh"
#include "modarith.cuh"
#include "umma.cuh"

namespace fhe_b200 {

namespace {

using namespace umma;

constexpr int row_bytes(int K) { return (9 * K + 31) / 32 * 32; }  // d_s bytes + sign bytes

// Four CTAs per SM (64 registers) where that costs no spills, fewer otherwise.
template <int K>
__global__ void __launch_bounds__(kTcThreads, K <= 10 && K != 7 ? 4 : (K <= 13 ? 3 : 1))
    mod_down_tc_kernel(PrimeTables t, KeySwitchTables ks, ModDownTcTables tc, int n,
                       int moduli_id, int L, const int64_t *acc, EpilogueOps ops, int64_t *out,
                       TcStatus status) {
  constexpr int KB = row_bytes(K);
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t *sA = smem;                   // [128 rows][KB], core matrices
  uint8_t *sB = smem + kTcCoeffs * KB;  // one round: [128 columns][KB]
  int64_t *divided = reinterpret_cast<int64_t *>(sB + kTcColumns * KB);
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ int64_t first_limb[kTcCoeffs];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int poly = blockIdx.y;
  const int coeff0 = blockIdx.x * kTcCoeffs;
  const int P = ks.prime_count;
  const int64_t *x = acc + static_cast<long long>(poly) * (L + K) * n + coeff0;

  // 1. Divisor triangle of one coefficient per thread, then its A row.
  if (tid < kTcCoeffs) {
    int64_t sp[K];
#pragma unroll
    for (int i = 0; i < K; i++) sp[i] = x[static_cast<long long>(L + i) * n + tid];
    uint64_t w[KB / 8];
#pragma unroll
    for (int i = 0; i < KB / 8; i++) w[i] = 0;
#pragma unroll
    for (int s = 0; s < K; s++) {
      const int64_t d = sp[K - 1 - s];
      w[s] = static_cast<uint64_t>(d);
      if (d < 0) w[K + (s >> 3)] |= 1ull << (8 * (s & 7));
#pragma unroll
      for (int i = 0; i < K - 1 - s; i++) {
        const int prime = moduli_id + L + i;
        const uint64_t q = t.q[prime];
        const int64_t q2 = static_cast<int64_t>(q << 1);
        sp[i] = mont_mult(guard(sp[i] + q2 - d, q2), ks.p_inverse_mult_r[s * P + prime], q,
                          t.k[prime]);
      }
    }
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

  // 3. One MMA round per 16 targets; each thread folds 8 targets of its coefficient.
  const int lane_base = (warp & 3) * 32;
  const int row = lane_base + lane;
  const int half = warp >> 2;
  bool ok = true;
  int round = 0;
  for (; round < tc.rounds; round++) {
    {
      // The round's slice of the constant B matrix, already in core-matrix order
      // (the previous round's MMAs have completed: every thread passed its wait).
      constexpr int chunks = kTcColumns * KB / 16;
      const uint4 *src = reinterpret_cast<const uint4 *>(tc.b) + static_cast<size_t>(round) * chunks;
      uint4 *dst = reinterpret_cast<uint4 *>(sB);
      for (int i = tid; i < chunks; i += kTcThreads) dst[i] = src[i];
      fence_async_smem();
      __syncthreads();
    }
    if (tid == 0) {
      mma_round(tmem, sA, sB, KB);
      mma_commit(bar);
    }
    // This thread's words x_j of the round, loaded while the MMAs run.
    constexpr int kHalfTargets = kTcTargets / 2;
    int64_t xs[kHalfTargets];
#pragma unroll
    for (int u = 0; u < kHalfTargets; u++) {
      const int j = round * kTcTargets + half * kHalfTargets + u;
      xs[u] = j < L ? __ldg(x + static_cast<long long>(j) * n + row) : 0;
    }
    ok = __syncthreads_and(mbar_wait(bar, round & 1, status.wait_limit)) != 0;
    if (!ok) break;
    tc_fence_after();
    // Each warpgroup folds 8 of the round's 16 targets, two per tensor-memory load.
#pragma unroll
    for (int u2 = 0; u2 < kHalfTargets / 2; u2++) {
      const int jp = half * kHalfTargets + 2 * u2;
      const int j0 = round * kTcTargets + jp;
      if (j0 >= L) continue;  // uniform across the warp
      uint32_t d[16];
      tmem_load16(tmem + (static_cast<uint32_t>(lane_base) << 16) + jp * 8, d);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = j0 + h;
        if (j >= L) continue;  // uniform across the warp
        const int prime = moduli_id + j;
        const uint64_t q = t.q[prime], kq = t.k[prime];
        uint64_t lo, hi;
        fold8(d + 8 * h, lo, hi);
        const int64_t xj = xs[2 * u2 + h];
        // REDC(X) < q + 2^19, and x_j prod pinv by Shoup's product is below 2q (its
        // value is all that matters: the total is reduced to [0, q) below).
        const uint64_t v = static_cast<uint64_t>(redc_wide(lo, hi, q, kq)) +
                           shoup_mult(static_cast<uint64_t>(tc.c_shoup[2 * j]),
                                      static_cast<uint64_t>(tc.c_shoup[2 * j + 1]),
                                      static_cast<uint64_t>(xj), q);
        uint64_t r = v >= (q << 1) ? v - (q << 1) : v;
        r = r >= q ? r - q : r;
        divided[j * kTcCoeffs + row] = static_cast<int64_t>(r);
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (!ok) {
    // The round's MMAs may still be running: wait for them (bounded) before the
    // tensor memory is given back.
    if (tid == 0) atomicExch(status.error, 1);
    if (warp == 0) mbar_wait(bar, round & 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem);
  if (!ok) return;

  // 4. The caller's operations on the divided limbs.
  mod_down_store<true>(t, ks, n, moduli_id, L, poly, coeff0, kTcCoeffs, ops, out, first_limb,
                       [&](int j, int c) -> int64_t { return divided[j * kTcCoeffs + c]; });
}

size_t tc_smem_bytes(int K, int L) {
  const int kb = row_bytes(K);
  return static_cast<size_t>(kTcCoeffs) * kb + static_cast<size_t>(kTcColumns) * kb +
         static_cast<size_t>(L) * kTcCoeffs * sizeof(int64_t);
}

using u128 = unsigned __int128;

uint64_t mul_mod(uint64_t a, uint64_t b, uint64_t m) {
  return static_cast<uint64_t>(static_cast<u128>(a) * b % m);
}

uint64_t pow_mod(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  b %= m;
  for (; e; e >>= 1, b = mul_mod(b, b, m))
    if (e & 1) r = mul_mod(r, b, m);
  return r;
}

}  // namespace

bool mod_down_tc_supported(int special_count, int limbs, int n) {
  return special_count >= 1 && special_count <= 16 && limbs >= 1 && n >= kTcCoeffs &&
         n % kTcCoeffs == 0 && tc_smem_bytes(special_count, limbs) <= 200 * 1024;
}

ModDownTcHost make_mod_down_tc_tables(const std::vector<uint64_t> &q,
                                      const std::vector<std::vector<int64_t>> &p_inverse_mult_r,
                                      int moduli_id, int limbs, int special_count) {
  const int K = special_count, L = limbs;
  ModDownTcHost h;
  h.kb = row_bytes(K);
  h.rounds = (L + kTcTargets - 1) / kTcTargets;
  h.b.assign(static_cast<size_t>(h.rounds) * kTcColumns * h.kb, 0);
  h.c_r.resize(L);
  h.c_shoup.resize(2 * static_cast<size_t>(L));
  for (int j = 0; j < L; j++) {
    const int prime = moduli_id + j;
    const uint64_t m = q[prime];
    const uint64_t r = pow_mod(2, 62, m);
    const uint64_t r_inv = pow_mod(r, m - 2, m);  // m is prime
    std::vector<uint64_t> w(K);
    uint64_t prod = 1 % m;
    for (int s = K - 1; s >= 0; s--) {
      const uint64_t pr = static_cast<uint64_t>(p_inverse_mult_r[s][prime]) % m;
      prod = mul_mod(prod, mul_mod(pr, r_inv, m), m);  // times p_s^-1 mod q_j
      w[s] = prod;
    }
    h.c_r[j] = static_cast<int64_t>(mul_mod(prod, r, m));
    h.c_shoup[2 * j] = static_cast<int64_t>(prod);
    h.c_shoup[2 * j + 1] = static_cast<int64_t>((static_cast<u128>(prod) << 64) / m);
    const uint64_t two64 = static_cast<uint64_t>((static_cast<u128>(1) << 64) % m);
    const int round = j / kTcTargets, jl = j % kTcTargets;
    uint8_t *b = h.b.data() + static_cast<size_t>(round) * kTcColumns * h.kb;
    for (int s = 0; s < K; s++) {
      const uint64_t wn = mul_mod((m - w[s]) % m, r, m);  // w'_sj R
      const uint64_t z = (m - mul_mod(two64, wn, m)) % m;  // -2^64 w'_sj R
      uint64_t e = wn;  // w'_sj 2^(8a) R for a = 0, 1, ...
      for (int a = 0; a < 8; a++) {
        for (int bb = 0; bb < 8; bb++)
          b[core_offset(jl * 8 + bb, s * 8 + a, kTcColumns)] = static_cast<uint8_t>(e >> (8 * bb));
        e = static_cast<uint64_t>((static_cast<u128>(e) << 8) % m);
      }
      for (int bb = 0; bb < 8; bb++)
        b[core_offset(jl * 8 + bb, 8 * K + s, kTcColumns)] = static_cast<uint8_t>(z >> (8 * bb));
    }
  }
  return h;
}

cudaError_t launch_mod_down_epilogue_tc(const PrimeTables &t, const KeySwitchTables &ks,
                                        const ModDownTcTables &tc, int n, int moduli_id,
                                        int limbs, const int64_t *acc, const EpilogueOps &ops,
                                        int64_t *out, const TcStatus &status, cudaStream_t s) {
  const int K = ks.special_count;
  if (!mod_down_tc_supported(K, limbs, n) || tc.b == nullptr || status.error == nullptr ||
      tc.kb != row_bytes(K) || tc.rounds != (limbs + kTcTargets - 1) / kTcTargets ||
      (ops.base_polys > 0 && ops.base == nullptr) || (ops.rescale && ops.signed_perm != nullptr) ||
      ops.polys < 1 || ops.polys > 2 || ops.base_polys > ops.polys)
    return cudaErrorInvalidValue;
  const size_t smem = tc_smem_bytes(K, limbs);
  const dim3 grid(n / kTcCoeffs, ops.polys);
  // The shared-memory limit is raised once per instantiation and device to the most
  // any supported shape needs, so no attribute call falls inside a graph capture.
  static int raised[17] = {};
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  const int bit = 1 << (device & 31);
  switch (K) {
#define FHE_TC_CASE(KK)                                                                         \
  case KK:                                                                                      \
    if (!(raised[KK] & bit)) {                                                                  \
      e = cudaFuncSetAttribute(mod_down_tc_kernel<KK>,                                          \
                               cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);        \
      if (e != cudaSuccess) return e;                                                           \
      raised[KK] |= bit;                                                                        \
    }                                                                                           \
    note_launch();                                                                              \
    mod_down_tc_kernel<KK><<<grid, kTcThreads, smem, s>>>(t, ks, tc, n, moduli_id, limbs, acc,  \
                                                          ops, out, status);                     \
    break;
    FHE_TC_CASE(1) FHE_TC_CASE(2) FHE_TC_CASE(3) FHE_TC_CASE(4) FHE_TC_CASE(5) FHE_TC_CASE(6)
    FHE_TC_CASE(7) FHE_TC_CASE(8) FHE_TC_CASE(9) FHE_TC_CASE(10) FHE_TC_CASE(11) FHE_TC_CASE(12)
    FHE_TC_CASE(13) FHE_TC_CASE(14) FHE_TC_CASE(15) FHE_TC_CASE(16)
#undef FHE_TC_CASE
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace fhe_b200
