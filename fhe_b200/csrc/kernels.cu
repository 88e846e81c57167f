// Device kernels of the B200 CKKS engine: element-wise families, rescale and the
// hybrid key-switching pipeline (see kernels.cuh for the contract of each launcher).
#include "kernels.cuh"
#include "epilogue.cuh"
#include "ntt.cuh"

#include <atomic>

namespace fhe_b200 {

namespace {
std::atomic<unsigned long long> g_launches{0};
}

void note_launch(unsigned count) { g_launches.fetch_add(count, std::memory_order_relaxed); }
unsigned long long kernel_launch_count() { return g_launches.load(std::memory_order_relaxed); }
namespace {
NttTuning g_ntt_tuning[18];  // zero: the default
}

NttTuning ntt_default_tuning(int log_n) {
  NttTuning t;
  t.s_second = log_n >= 15 ? 8 : (log_n >= 13 ? 7 : 6);
  t.first_columns_log = log_n - t.s_second >= 9 ? 3 : 4;
  t.second_tile_log = 12;
  return t;
}

NttTuning ntt_tuning(int log_n) {
  if (log_n >= 0 && log_n < 18 && g_ntt_tuning[log_n].s_second > 0) return g_ntt_tuning[log_n];
  return ntt_default_tuning(log_n);
}

bool set_ntt_tuning(int log_n, const NttTuning &tu) {
  if (log_n < 12 || log_n > 17) return false;
  const int s1 = log_n - tu.s_second;
  const int c2 = tu.second_tile_log - tu.s_second;
  if (tu.s_second < 1 || tu.s_second > 11 || s1 < 1 || s1 > 11) return false;
  if (tu.first_columns_log < 0 || tu.first_columns_log > tu.s_second) return false;
  if (c2 < 0 || c2 > s1) return false;
  if ((sizeof(int64_t) << (tu.first_columns_log + s1)) > static_cast<size_t>(kNttMaxSmem) ||
      (sizeof(int64_t) << tu.second_tile_log) > static_cast<size_t>(kNttMaxSmem))
    return false;
  g_ntt_tuning[log_n] = tu;
  return true;
}

void unnote_launches(unsigned long long count) {
  g_launches.fetch_sub(count, std::memory_order_relaxed);
}

namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(long long work) {
  long long b = (work + kThreads - 1) / kThreads;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

// --------------------------------------------------------------- tensor --

__global__ void tensor_kernel(PrimeTables t, int n, int limbs, int prime_base, const int64_t *a,
                              const int64_t *b, int64_t *z) {
  const long long total = static_cast<long long>(limbs) * n;
  const long long ps = total;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int prime = prime_base + static_cast<int>(i >> (__ffs(n) - 1));
    const uint64_t q = t.q[prime], k = t.k[prime];
    const int64_t qs = static_cast<int64_t>(q), q2 = qs << 1;
    const int64_t a0 = a[i], a1 = a[ps + i], b0 = b[i], b1 = b[ps + i];
    z[i] = mont_mult_lazy(a0, b0, q, k);
    z[ps + i] = guard(guard(mont_mult_lazy(a0, b1, q, k) + mont_mult_lazy(a1, b0, q, k), q2), qs);
    z[2 * ps + i] = mont_mult_lazy(a1, b1, q, k);
  }
}

__global__ void add_reduce_kernel(PrimeTables t, int n, int limbs, int prime_base, long long total,
                                  const int64_t *x1, const int64_t *x2, int64_t *y) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int prime = prime_base + static_cast<int>((i >> (__ffs(n) - 1)) % limbs);
    const int64_t qs = static_cast<int64_t>(t.q[prime]);
    y[i] = guard(guard(x1[i] + x2[i], qs << 1), qs);
  }
}

// -------------------------------------------------------------- rescale --


__global__ void rescale_kernel(PrimeTables t, KeySwitchTables ks, int n, int limbs, int moduli_id,
                               const int64_t *x, long long xs, int64_t *y, long long ys) {
  const int poly = blockIdx.y;
  const long long per_poly = static_cast<long long>(limbs - 1) * n;
  // get_rounder compares the signed word with the unsigned q/2 (unit.cpp:67-70), so
  // a negative word counts as above it.
  const uint64_t q_half = t.q[moduli_id] >> 1;
  const int64_t *xp = x + poly * xs;
  int64_t *yp = y + poly * ys;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < per_poly;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(i >> (__ffs(n) - 1));
    const int c = static_cast<int>(i - static_cast<long long>(j) * n);
    const int prime = moduli_id + 1 + j;
    const int64_t x0 = xp[c];
    const int64_t rounder = static_cast<uint64_t>(x0) > q_half ? 1 : 0;  // get_rounder
    const long long entry = static_cast<long long>(moduli_id) * ks.prime_count + prime;
    yp[i] = rescale_word_shoup(xp[static_cast<long long>(j + 1) * n + c], x0, rounder, t.q[prime],
                               t.k[prime], ks.rescale_scale[entry], ks.rescale_shoup + 2 * entry);
  }
}

// CKKSCore::multiply(ct, double) (core.cpp:196-229) in one pass: every limb entered by
// its scaled constant and reduced (mont_enter + reduce_2q_to_q), then rescale_once_
// by limb 0; limb 0's entered word is recomputed per output instead of stored.
// Each thread serves one coefficient of kScalarLimbsPerThread consecutive output
// limbs, so the dropped limb's entered word e0 is formed once for all of them.
constexpr int kScalarLimbsPerThread = 4;

__global__ void scalar_rescale_kernel(PrimeTables t, KeySwitchTables ks, int log_n, int limbs,
                                      int moduli_id, LimbScalars c, const int64_t *x,
                                      long long xs, int64_t *y, long long ys) {
  const int poly = blockIdx.z;
  const long long cidx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (cidx >= (1LL << log_n)) return;
  const uint64_t q0 = t.q[moduli_id], k0 = t.k[moduli_id];
  const int64_t *xp = x + poly * xs;
  int64_t *yp = y + poly * ys;
  const int64_t e0 = guard(mont_mult_lazy(xp[cidx], c.v[0], q0, k0), static_cast<int64_t>(q0));
  const int64_t rounder = static_cast<uint64_t>(e0) > (q0 >> 1) ? 1 : 0;  // get_rounder
  const int j0 = blockIdx.y * kScalarLimbsPerThread;
#pragma unroll
  for (int u = 0; u < kScalarLimbsPerThread; u++) {
    const int j = j0 + u;
    if (j >= limbs - 1) break;
    const int prime = moduli_id + 1 + j;
    const uint64_t q = t.q[prime], k = t.k[prime];
    const int64_t ej = guard(mont_mult_lazy(xp[(static_cast<long long>(j + 1) << log_n) + cidx],
                                            c.v[j + 1], q, k),
                             static_cast<int64_t>(q));
    const long long entry = static_cast<long long>(moduli_id) * ks.prime_count + prime;
    yp[(static_cast<long long>(j) << log_n) + cidx] =
        rescale_word_shoup(ej, e0, rounder, q, k, ks.rescale_scale[entry], ks.rescale_shoup + 2 * entry);
  }
}

// ---------------------------------------------------------- mixed radix --

// One partition of alpha = A limbs per thread-coefficient (rns_to_mrs,
// core_key_switch.cpp:21-56, Garner's algorithm with the reference's lazy ranges).
// Three CTAs per SM where the digits fit the registers that leaves (A <= 10).
template <int A>
__global__ void __launch_bounds__(256, A <= 10 ? 3 : 2)
    mixed_radix_kernel(PrimeTables t, DevicePartitions dp, int n, int moduli_id,
                                   const int64_t *x, int64_t *digits) {
  const int p = blockIdx.y;
  if (dp.size[p] != A) return;
  const int start = dp.start[p];
  const int coeff = blockIdx.x * blockDim.x + threadIdx.x;
  if (coeff >= n) return;
  int64_t y[A];
  const int64_t first = x[static_cast<long long>(start) * n + coeff];
#pragma unroll
  for (int c = 0; c < A; c++) y[c] = first;
#pragma unroll
  for (int ci = 0; ci < A - 1; ci++) {
    const int yo = ci + 1;
    const int prime = moduli_id + start + yo;
    const uint64_t q = t.q[prime], k = t.k[prime];
    const int64_t qs = static_cast<int64_t>(q), q2 = qs << 1;
    const int64_t xv = x[static_cast<long long>(start + yo) * n + coeff];
    // mont_sub_enter_reduce_2q_to_q (compound.cpp:36-43)
    y[yo] = guard(mont_mult(guard(xv + q2 - y[yo], q2), dp.inverse_r[p * 16 + ci], q, k), qs);
#pragma unroll
    for (int t2 = 0; t2 < A - ci - 2; t2++) {
      const int dst = yo + 1 + t2;
      const int prime2 = moduli_id + start + dst;
      const uint64_t qq = t.q[prime2], kk = t.k[prime2];
      const int64_t qqs = static_cast<int64_t>(qq), qq2 = qqs << 1;
      // mont_enter_add_reduce_2q_to_q (compound.cpp:17-24)
      y[dst] = guard(guard(mont_mult(y[yo], dp.product_r[(p * 16 + ci) * 16 + t2], qq, kk) + y[dst],
                           qq2), qqs);
    }
  }
#pragma unroll
  for (int c = 0; c < A; c++) digits[static_cast<long long>(start + c) * n + coeff] = y[c];
}

// ModUp contraction (core_key_switch.cpp:92-106): extended limb j of partition p
// is the chain acc = guard(REDC(d_i c_ij) + acc, 2q) over the partition's digits
// (c_0j = R^2 mod q_j).  A thread owns one coefficient of one partition, keeps its
// alpha digits in registers and walks all extended limbs.  The extended limbs feed
// only value-only consumers (the forward NTT in Harvey's form, the key inner
// product, ModDown's reduced inverse transform), so only the chain's value modulo
// q_j matters: when every digit is in [0, 2^61), which holds for all digits produced
// from canonical inputs, sum_i d_i c_ij is accumulated exactly and reduced by one
// REDC (WideSum) to a word in [0, 2q); otherwise the chain runs term by term.
constexpr int kContractChunk = 8;  // extended limbs per thread

template <int A>
__global__ void __launch_bounds__(256)
    mod_up_contract_kernel(PrimeTables t, DevicePartitions dp, int n, int moduli_id,
                           const int64_t *digits, int64_t *ext, bool skip_own) {
  const int p = blockIdx.y;
  if (dp.size[p] != A) return;
  const int coeff = blockIdx.x * blockDim.x + threadIdx.x;
  if (coeff >= n) return;
  const int start = dp.start[p];
  const int E = dp.extended;
  const int j_begin = blockIdx.z * kContractChunk;
  if (j_begin >= E) return;
  int64_t d[A];
  bool fast = true;
#pragma unroll
  for (int i = 0; i < A; i++) {
    d[i] = digits[static_cast<long long>(start + i) * n + coeff];
    fast = fast && redc_operand_ok(d[i]);
  }
  const int64_t *cst = dp.product_r_squared + static_cast<long long>(p) * 16 * E;
  int64_t *out = ext + static_cast<long long>(p) * E * n + coeff;
  if (fast) {
    // Four extended limbs at a time: four independent accumulation chains.
    constexpr int kLanes = 4;
#pragma unroll
    for (int j0 = j_begin; j0 < j_begin + kContractChunk; j0 += kLanes) {
      if (j0 >= E) break;
      WideSum sum[kLanes];
      int jl[kLanes];
#pragma unroll
      for (int l = 0; l < kLanes; l++) {
        jl[l] = j0 + l < E ? j0 + l : E - 1;
        sum[l].add(static_cast<uint64_t>(d[0]), static_cast<uint64_t>(t.r_squared[moduli_id + jl[l]]));
      }
#pragma unroll
      for (int i = 1; i < A; i++) {
#pragma unroll
        for (int l = 0; l < kLanes; l++)
          sum[l].add(static_cast<uint64_t>(d[i]), static_cast<uint64_t>(cst[(i - 1) * E + jl[l]]));
      }
#pragma unroll
      for (int l = 0; l < kLanes; l++) {
        if (j0 + l < E && !(skip_own && jl[l] >= start && jl[l] < start + A)) {
          const int prime = moduli_id + jl[l];
          const uint64_t q = t.q[prime];
          out[static_cast<long long>(jl[l]) * n] = sum[l].reduce(q, t.k[prime], q << 1, t.inv_2q[prime]);
        }
      }
    }
    return;
  }
  for (int j = j_begin; j < j_begin + kContractChunk && j < E; j++) {
    if (skip_own && j >= start && j < start + A) continue;
    const int prime = moduli_id + j;
    const uint64_t q = t.q[prime], k = t.k[prime];
    const int64_t q2 = static_cast<int64_t>(q << 1);
    int64_t v = mont_mult(d[0], t.r_squared[prime], q, k);
#pragma unroll
    for (int i = 1; i < A; i++) v = guard(mont_mult(d[i], cst[(i - 1) * E + j], q, k) + v, q2);
    out[static_cast<long long>(j) * n] = v;
  }
}

// ------------------------------------------------------ key inner product --

// The reference chain (mont_mult, then mont_mult_add and reduce_2q_to_q per further
// partition) has the value sum_p REDC(e_p k_p) modulo q.  Its consumers are
// value-only (ModDown's inverse transform reduces every word; the rotation's b*P
// term and the bootstrap's NTT-form rotations and diagonal sums end in ModDown), so
// with every operand in [0, 2^61) the sum is evaluated exactly and reduced to a word
// in [0, q); otherwise the chain runs term by term.
__global__ void key_inner_product_kernel(PrimeTables t, DevicePartitions dp, int n, int moduli_id,
                                         const int64_t *ext, const int64_t *key, int key_primes,
                                         int view_offset, int64_t *acc) {
  const int E = dp.extended;
  const long long total = static_cast<long long>(E) * n;
  const int log_n = __ffs(n) - 1;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(i >> log_n);
    const int prime = moduli_id + j;
    const uint64_t q = t.q[prime], k = t.k[prime];
    const int64_t qs = static_cast<int64_t>(q), q2 = qs << 1;
    // Up to 16 partitions: one REDC of the exact sum; more: the lazy sum of the terms'
    // own REDCs (RedcSum), whose 128-bit accumulators cannot overflow.
    const bool wide = dp.count <= 16;
    bool fast = true;
    WideSum w0, w1;
    RedcSum r0, r1;
    for (int p = 0; p < dp.count && fast; p++) {
      const int64_t e = ext[static_cast<long long>(p) * total + i];
      const int kidx = dp.key_index[p];
      const int64_t k0 = key[(static_cast<long long>(2 * kidx) * key_primes + view_offset) * n + i];
      const int64_t k1 = key[(static_cast<long long>(2 * kidx + 1) * key_primes + view_offset) * n + i];
      if (!(redc_operand_ok(e) && redc_operand_ok(k0) && redc_operand_ok(k1))) {
        fast = false;
        break;
      }
      if (wide) {
        w0.add(static_cast<uint64_t>(e), static_cast<uint64_t>(k0));
        w1.add(static_cast<uint64_t>(e), static_cast<uint64_t>(k1));
      } else {
        r0.add(static_cast<uint64_t>(e), static_cast<uint64_t>(k0), k);
        r1.add(static_cast<uint64_t>(e), static_cast<uint64_t>(k1), k);
      }
    }
    if (fast) {
      acc[i] = wide ? w0.reduce(q, k, q, t.inv_q[prime]) : r0.reduce(q, q, t.inv_q[prime]);
      acc[total + i] = wide ? w1.reduce(q, k, q, t.inv_q[prime]) : r1.reduce(q, q, t.inv_q[prime]);
      continue;
    }
    int64_t x0 = 0, x1 = 0;
    for (int p = 0; p < dp.count; p++) {
      const int64_t e = ext[static_cast<long long>(p) * total + i];
      const int kidx = dp.key_index[p];
      const long long k0 = (static_cast<long long>(2 * kidx) * key_primes + view_offset) * n + i;
      const long long k1 = (static_cast<long long>(2 * kidx + 1) * key_primes + view_offset) * n + i;
      const int64_t a0 = mont_mult(e, key[k0], q, k);
      const int64_t a1 = mont_mult(e, key[k1], q, k);
      if (p == 0) {
        x0 = a0;
        x1 = a1;
      } else {  // mont_mult_add then reduce_2q_to_q
        x0 = guard(guard(a0 + x0, q2), qs);
        x1 = guard(guard(a1 + x1, q2), qs);
      }
    }
    acc[i] = x0;
    acc[total + i] = x1;
  }
}

// The same for P <= 8 partitions known at compile time: every partition's three
// words are loaded before any is used (the key rows' offsets come with the launch),
// and one OR of the operands' high words decides between the exact sum and the
// chain, so the loads of all partitions are in flight together.
template <int P>
__global__ void __launch_bounds__(256, P == 3 ? 4 : 0)  // three partitions: 4 CTAs/SM without spills
key_inner_product_fixed_kernel(PrimeTables t, DevicePartitions dp, int log_n, int moduli_id,
                               const int64_t *ext, const int64_t *key, long long poly_row,
                               KeyRowOffsets rows, int64_t *acc, TensorAddend add) {
  const long long total = static_cast<long long>(dp.extended) << log_n;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int limb = static_cast<int>(i >> log_n);
    const int prime = moduli_id + limb;
    const uint64_t q = t.q[prime], k = t.k[prime];
    // The tensor's factors at this word (a normal limb: index i in [poly][limbs][N]).
    const bool tensor = limb < add.limbs;  // uniform per warp (N >= 32)
    int64_t ta0 = 0, ta1 = 0, tb0 = 0, tb1 = 0;
    const bool product = add.b != nullptr;
    if (tensor) {
      ta0 = add.a[i];
      ta1 = add.a[add.a_stride + i];
      if (product) {
        tb0 = add.b[i];
        tb1 = add.b[add.b_stride + i];
      }
    }
    int64_t e[P], k0[P], k1[P];
#pragma unroll
    for (int p = 0; p < P; p++) {
      e[p] = ext[p * total + i];
      k0[p] = key[rows.off[p] + i];
      k1[p] = key[rows.off[p] + poly_row + i];
    }
    uint32_t high = 0;
    WideSum w0, w1;
#pragma unroll
    for (int p = 0; p < P; p++) {
      high |= static_cast<uint32_t>(static_cast<uint64_t>(e[p]) >> 32) |
              static_cast<uint32_t>(static_cast<uint64_t>(k0[p]) >> 32) |
              static_cast<uint32_t>(static_cast<uint64_t>(k1[p]) >> 32);
      w0.add(static_cast<uint64_t>(e[p]), static_cast<uint64_t>(k0[p]));
      w1.add(static_cast<uint64_t>(e[p]), static_cast<uint64_t>(k1[p]));
    }
    if (tensor) {
      high |= static_cast<uint32_t>((static_cast<uint64_t>(ta0) | static_cast<uint64_t>(ta1) |
                                     static_cast<uint64_t>(tb0) | static_cast<uint64_t>(tb1)) >> 32);
      if (product) {
        // b P as Shoup products (in [0, 2q)), then a0 (b0 P), a0 (b1 P) + a1 (b0 P).
        const uint64_t pw = static_cast<uint64_t>(add.p_shoup[2 * prime]);
        const uint64_t pwp = static_cast<uint64_t>(add.p_shoup[2 * prime + 1]);
        const uint64_t bp0 = shoup_mult(pw, pwp, static_cast<uint64_t>(tb0), q);
        const uint64_t bp1 = shoup_mult(pw, pwp, static_cast<uint64_t>(tb1), q);
        w0.add(static_cast<uint64_t>(ta0), bp0);
        w1.add(static_cast<uint64_t>(ta0), bp1);
        w1.add(static_cast<uint64_t>(ta1), bp0);
      } else {
        const uint64_t pr = static_cast<uint64_t>(add.p_mont[prime]);  // P R mod q, below q
        w0.add(static_cast<uint64_t>(ta0), pr);
        w1.add(static_cast<uint64_t>(ta1), pr);
      }
    }
    if ((high >> 29) == 0) {  // every operand below 2^61
      acc[i] = w0.reduce(q, k, q, t.inv_q[prime]);
      acc[total + i] = w1.reduce(q, k, q, t.inv_q[prime]);
      continue;
    }
    const int64_t qs = static_cast<int64_t>(q), q2 = qs << 1;
    int64_t x0 = 0, x1 = 0;
#pragma unroll
    for (int p = 0; p < P; p++) {
      const int64_t a0 = mont_mult(e[p], k0[p], q, k);
      const int64_t a1 = mont_mult(e[p], k1[p], q, k);
      if (p == 0) {
        x0 = a0;
        x1 = a1;
      } else {  // mont_mult_add then reduce_2q_to_q
        x0 = guard(guard(a0 + x0, q2), qs);
        x1 = guard(guard(a1 + x1, q2), qs);
      }
    }
    if (tensor) {
      // The same values term by term, for words outside the exact sum's range.
      const int64_t pr = add.p_mont[prime];
      if (product) {
        const int64_t bp0 = mont_mult(tb0, pr, q, k), bp1 = mont_mult(tb1, pr, q, k);
        x0 = guard(guard(mont_mult(ta0, bp0, q, k) + x0, q2), qs);
        x1 = guard(guard(mont_mult(ta0, bp1, q, k) + x1, q2), qs);
        x1 = guard(guard(mont_mult(ta1, bp0, q, k) + x1, q2), qs);
      } else {
        x0 = guard(guard(mont_mult(ta0, pr, q, k) + x0, q2), qs);
        x1 = guard(guard(mont_mult(ta1, pr, q, k) + x1, q2), qs);
      }
    }
    acc[i] = x0;
    acc[total + i] = x1;
  }
}

// ------------------------------------------------------ mod down epilogue --

// Sequential exact division by the K special primes, last first
// (core_key_switch.cpp:123-160, mont_sub_enter compound.cpp:45-52 with its
// [0, 2p) outputs carried into the next division), then make_unsigned and the
// caller's combination (see launch_mod_down_epilogue).
// A CTA owns kEpilogueCoeffs consecutive coefficients of one polynomial.  Phase 1
// derives, per coefficient, the divisor sequence d_s = (value of special limb
// K-1-s after s divisions) with one thread per special limb and a barrier per
// division; phase 2 spreads the K dependent divisions of every normal limb over
// all threads (limb-major, coefficient-fastest for coalescing).
constexpr int kEpilogueCoeffs = 16;  // K * 16 <= 256 threads for every K <= 16

template <int K>
__global__ void __launch_bounds__(256)
    mod_down_epilogue_kernel(PrimeTables t, KeySwitchTables ks, int n, int moduli_id, int limbs,
                             const int64_t *acc, EpilogueOps ops, int64_t *out) {
  constexpr int CB = kEpilogueCoeffs;
  __shared__ int64_t divisor[K][CB];
  __shared__ int64_t first_limb[CB];
  const int poly = blockIdx.y;
  const int coeff0 = blockIdx.x * CB;
  const int L = limbs;
  const int E = L + K;
  const int P = ks.prime_count;
  const int64_t *x = acc + static_cast<long long>(poly) * E * n + coeff0;

  // Phase 1: special limbs (thread = (special i, coefficient c)).
  {
    const int i = threadIdx.x / CB, c = threadIdx.x % CB;
    const bool active = i < K && coeff0 + c < n;
    int64_t sp = 0;
    uint64_t q = 0, kk = 0;
    int prime = 0;
    if (active) {
      prime = moduli_id + L + i;
      q = t.q[prime];
      kk = t.k[prime];
      sp = x[static_cast<long long>(L + i) * n + c];
    }
#pragma unroll
    for (int s = 0; s < K; s++) {
      if (active && i == K - 1 - s) divisor[s][c] = sp;
      __syncthreads();
      if (active && i < K - 1 - s) {
        const int64_t q2 = static_cast<int64_t>(q << 1);
        sp = mont_mult(guard(sp + q2 - divisor[s][c], q2), ks.p_inverse_mult_r[s * P + prime], q, kk);
      }
    }
  }

  auto divide = [&](int j, int c) -> int64_t {
    const int prime = moduli_id + j;
    const uint64_t q = t.q[prime], kk = t.k[prime];
    const int64_t qs = static_cast<int64_t>(q), q2 = qs << 1;
    int64_t v = x[static_cast<long long>(j) * n + c];
#pragma unroll
    for (int s = 0; s < K; s++)
      v = mont_mult(guard(v + q2 - divisor[s][c], q2), ks.p_inverse_mult_r[s * P + prime], q, kk);
    return v < 0 ? v + qs : guard(v, qs);  // make_unsigned_reduce_2q_to_q
  };
  const int valid = n - coeff0 < CB ? n - coeff0 : CB;
  mod_down_store(t, ks, n, moduli_id, L, poly, coeff0, valid, ops, out, first_limb, divide);
}

struct TensorLoad {
  const int64_t *a;
  const int64_t *b;
  long long poly_stride;  // limbs * n
  const uint64_t *q;
  const uint64_t *k;
  // Optional sink of the third polynomial's NTT-form words into each partition's own
  // limbs of ModUp's extended buffer [count][extended][N].
  int64_t *own_ext = nullptr;
  const int *part_start = nullptr;
  const int *part_size = nullptr;
  int part_count = 0;
  int extended = 0;
  bool third_only = false;  // a one-polynomial launch of the third polynomial
  __device__ __forceinline__ int64_t operator()(int poly, int limb, int prime, int gi, int n) const {
    const long long i = static_cast<long long>(limb) * n + gi;
    const uint64_t qq = q[prime], kk = k[prime];
    if (third_only) poly = 2;
    if (poly == 0) return mont_mult_lazy(a[i], b[i], qq, kk);
    if (poly == 2) {
      const int64_t v = mont_mult_lazy(a[poly_stride + i], b[poly_stride + i], qq, kk);
      if (own_ext != nullptr) {
        int p = 0;
        while (p + 1 < part_count && limb >= part_start[p] + part_size[p]) p++;
        own_ext[(static_cast<long long>(p) * extended + limb) * n + gi] = v;
      }
      return v;
    }
    const int64_t qs = static_cast<int64_t>(qq);
    return guard(guard(mont_mult_lazy(a[i], b[poly_stride + i], qq, kk) +
                           mont_mult_lazy(a[poly_stride + i], b[i], qq, kk),
                       qs << 1),
                 qs);
  }
};

// The tensor's third polynomial d2 = a1 b1 as a streaming pass before a plain mixed
// inverse transform (TensorLoad's words, with 16-byte accesses by a full grid: the
// loader pass of d2 alone waits on its loads and fills under one wave), and its
// NTT-form words into each partition's own limbs of ModUp's extended buffer when one
// is given.  Same words either way.
__global__ void __launch_bounds__(256)
    tensor_third_kernel(PrimeTables t, TensorLoad ld, int log_n, int limbs, int prime_base,
                        int64_t *y) {
  const long long pairs = static_cast<long long>(limbs) << (log_n - 1);
  const long long n = 1LL << log_n;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < pairs;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long w = 2 * i;
    const int limb = static_cast<int>(w >> log_n);
    const int prime = prime_base + limb;
    const uint64_t q = t.q[prime], k = t.k[prime];
    const longlong2 a = *reinterpret_cast<const longlong2 *>(ld.a + ld.poly_stride + w);
    const longlong2 b = *reinterpret_cast<const longlong2 *>(ld.b + ld.poly_stride + w);
    longlong2 v;
    v.x = mont_mult_lazy(a.x, b.x, q, k);
    v.y = mont_mult_lazy(a.y, b.y, q, k);
    *reinterpret_cast<longlong2 *>(y + w) = v;
    if (ld.own_ext != nullptr) {
      int p = 0;
      while (p + 1 < ld.part_count && limb >= ld.part_start[p] + ld.part_size[p]) p++;
      *reinterpret_cast<longlong2 *>(ld.own_ext + (static_cast<long long>(p) * ld.extended) * n + w) = v;
    }
  }
}

}  // namespace

// ============================================================ launchers ==

cudaError_t launch_tensor(const PrimeTables &t, int n, int limbs, int prime_base, const int64_t *a,
                          const int64_t *b, int64_t *z, cudaStream_t s) {
  note_launch();
  tensor_kernel<<<blocks_for(static_cast<long long>(limbs) * n), kThreads, 0, s>>>(t, n, limbs,
                                                                                  prime_base, a, b, z);
  return cudaGetLastError();
}

cudaError_t launch_add_reduce(const PrimeTables &t, int n, int polys, int limbs, int prime_base,
                              const int64_t *x1, const int64_t *x2, int64_t *y, cudaStream_t s) {
  const long long total = static_cast<long long>(polys) * limbs * n;
  note_launch();
  add_reduce_kernel<<<blocks_for(total), kThreads, 0, s>>>(t, n, limbs, prime_base, total, x1, x2, y);
  return cudaGetLastError();
}

cudaError_t launch_rescale(const PrimeTables &t, const KeySwitchTables &ks, int n, int polys,
                           int limbs, int moduli_id, const int64_t *x, long long xs, int64_t *y,
                           long long ys, cudaStream_t s) {
  const dim3 grid(blocks_for(static_cast<long long>(limbs - 1) * n), polys);
  note_launch();
  rescale_kernel<<<grid, kThreads, 0, s>>>(t, ks, n, limbs, moduli_id, x, xs, y, ys);
  return cudaGetLastError();
}

cudaError_t launch_scalar_rescale(const PrimeTables &t, const KeySwitchTables &ks, int n,
                                  int polys, int limbs, int moduli_id, const LimbScalars &c,
                                  const int64_t *x, long long x_stride, int64_t *y,
                                  long long y_stride, cudaStream_t s) {
  if (limbs < 2 || limbs > kMaxScalarLimbs) return cudaErrorInvalidValue;
  const int log_n = __builtin_ctz(static_cast<unsigned>(n));
  const dim3 grid(blocks_for(n), (limbs - 1 + kScalarLimbsPerThread - 1) / kScalarLimbsPerThread,
                  polys);
  note_launch();
  scalar_rescale_kernel<<<grid, kThreads, 0, s>>>(t, ks, log_n, limbs, moduli_id, c, x, x_stride,
                                                  y, y_stride);
  return cudaGetLastError();
}

cudaError_t launch_mixed_radix(const PrimeTables &t, const DevicePartitions &dp, int n,
                               int moduli_id, const int64_t *x, int64_t *digits, cudaStream_t s) {
  const dim3 grid(blocks_for(n), dp.count);
  // One launch per distinct partition size; blocks of other sizes exit at once.
  for (int size = 1; size <= 16; size++) {
    if (!(dp.size_mask & (1u << size))) continue;
    switch (size) {
#define FHE_MRS_CASE(A) \
  case A: note_launch(); mixed_radix_kernel<A><<<grid, kThreads, 0, s>>>(t, dp, n, moduli_id, x, digits); break;
      FHE_MRS_CASE(1) FHE_MRS_CASE(2) FHE_MRS_CASE(3) FHE_MRS_CASE(4) FHE_MRS_CASE(5)
      FHE_MRS_CASE(6) FHE_MRS_CASE(7) FHE_MRS_CASE(8) FHE_MRS_CASE(9) FHE_MRS_CASE(10)
      FHE_MRS_CASE(11) FHE_MRS_CASE(12) FHE_MRS_CASE(13) FHE_MRS_CASE(14) FHE_MRS_CASE(15)
      FHE_MRS_CASE(16)
#undef FHE_MRS_CASE
      default: return cudaErrorInvalidValue;
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_mod_up_ntt(const PrimeTables &t, const DevicePartitions &dp, int log_n,
                              int moduli_id, const int64_t *digits, int64_t *ext, cudaStream_t s,
                              bool skip_own) {
  const int n = 1 << log_n;
  const dim3 grid(blocks_for(n), dp.count, (dp.extended + kContractChunk - 1) / kContractChunk);
  for (int size = 1; size <= 16; size++) {
    if (!(dp.size_mask & (1u << size))) continue;
    switch (size) {
#define FHE_MU_CASE(A)                                                                    \
  case A:                                                                                 \
    note_launch();                                                                        \
    mod_up_contract_kernel<A><<<grid, kThreads, 0, s>>>(t, dp, n, moduli_id, digits, ext, skip_own); \
    break;
      FHE_MU_CASE(1) FHE_MU_CASE(2) FHE_MU_CASE(3) FHE_MU_CASE(4) FHE_MU_CASE(5)
      FHE_MU_CASE(6) FHE_MU_CASE(7) FHE_MU_CASE(8) FHE_MU_CASE(9) FHE_MU_CASE(10)
      FHE_MU_CASE(11) FHE_MU_CASE(12) FHE_MU_CASE(13) FHE_MU_CASE(14) FHE_MU_CASE(15)
      FHE_MU_CASE(16)
#undef FHE_MU_CASE
      default: return cudaErrorInvalidValue;
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_extended_ntt(t, dp, log_n, moduli_id, ext, s, skip_own);
}

cudaError_t launch_extended_ntt(const PrimeTables &t, const DevicePartitions &dp, int log_n,
                                int moduli_id, int64_t *ext, cudaStream_t s, bool skip_own) {
  const long long stride = static_cast<long long>(dp.extended) << log_n;
  PlainLoad ld{ext, stride};
  PlainStore st{ext, stride};
  // Value-only: the extended polynomial reaches the output only through the key
  // inner product's reduction to [0, q) and ModDown's reduced inverse transform.
  return forward_ntt<PlainLoad, PlainStore, kNttValueOnly>(log_n, dp.count, dp.extended, moduli_id, t,
                                                           ld, st, ext, stride, s,
                                                           skip_own ? dp.start : nullptr,
                                                           skip_own ? dp.size : nullptr);
}

cudaError_t launch_key_inner_product(const PrimeTables &t, const DevicePartitions &dp, int n,
                                     int moduli_id, const int64_t *ext, const int64_t *key,
                                     int key_primes, int view_offset, int64_t *acc, cudaStream_t s,
                                     const TensorAddend &addend) {
  if (addend.limbs > 0 &&
      (dp.count > 8 || addend.limbs > dp.extended || addend.a == nullptr ||
       addend.p_shoup == nullptr || addend.p_mont == nullptr))
    return cudaErrorInvalidValue;
  if (dp.count >= 1 && dp.count <= 8) {
    KeyRowOffsets rows;
    for (int p = 0; p < dp.count; p++)
      rows.off[p] = (2LL * dp.key_index_first[p] * key_primes + view_offset) * n;
    const int log_n = __builtin_ctz(static_cast<unsigned>(n));
    const long long poly_row = static_cast<long long>(key_primes) * n;
    const unsigned grid = blocks_for(static_cast<long long>(dp.extended) * n);
    note_launch();
    switch (dp.count) {
#define FHE_KIP_CASE(P)                                                                           \
  case P:                                                                                         \
    key_inner_product_fixed_kernel<P><<<grid, kThreads, 0, s>>>(t, dp, log_n, moduli_id, ext, key, \
                                                                poly_row, rows, acc, addend);    \
    break;
      FHE_KIP_CASE(1) FHE_KIP_CASE(2) FHE_KIP_CASE(3) FHE_KIP_CASE(4)
      FHE_KIP_CASE(5) FHE_KIP_CASE(6) FHE_KIP_CASE(7) FHE_KIP_CASE(8)
#undef FHE_KIP_CASE
    }
    return cudaGetLastError();
  }
  note_launch();
  key_inner_product_kernel<<<blocks_for(static_cast<long long>(dp.extended) * n), kThreads, 0, s>>>(
      t, dp, n, moduli_id, ext, key, key_primes, view_offset, acc);
  return cudaGetLastError();
}

cudaError_t launch_mod_down_intt(const PrimeTables &t, int log_n, int moduli_id, int extended,
                                 int64_t *acc, cudaStream_t s, int polys) {
  if (polys < 1 || polys > 2) return cudaErrorInvalidValue;
  const long long stride = static_cast<long long>(extended) << log_n;
  PlainLoad ld{acc, stride};
  EnterExitStore<true> st{acc, stride, t.n_inverse, t.q, t.k, t.exit_shoup};
  // Value-only: the store reduces every word to [0, q).
  return inverse_ntt<PlainLoad, EnterExitStore<true>, kNttValueOnly>(log_n, polys, extended,
                                                                     moduli_id, t, ld, st, acc,
                                                                     stride, s);
}

cudaError_t launch_mod_down_epilogue_ops(const PrimeTables &t, const KeySwitchTables &ks, int n,
                                         int moduli_id, int limbs, const int64_t *acc,
                                         const EpilogueOps &ops, int64_t *out, cudaStream_t s) {
  if ((ops.base_polys > 0 && ops.base == nullptr) || (ops.rescale && ops.signed_perm != nullptr) ||
      ops.polys < 1 || ops.polys > 2 || ops.base_polys > ops.polys)
    return cudaErrorInvalidValue;
  const dim3 grid((n + kEpilogueCoeffs - 1) / kEpilogueCoeffs, ops.polys);
  switch (ks.special_count) {
#define FHE_MD_CASE(K)                                                                      \
  case K:                                                                                   \
    note_launch();                                                                          \
    mod_down_epilogue_kernel<K><<<grid, kThreads, 0, s>>>(t, ks, n, moduli_id, limbs, acc, ops, \
                                                          out);                             \
    break;
    FHE_MD_CASE(1) FHE_MD_CASE(2) FHE_MD_CASE(3) FHE_MD_CASE(4) FHE_MD_CASE(5) FHE_MD_CASE(6)
    FHE_MD_CASE(7) FHE_MD_CASE(8) FHE_MD_CASE(9) FHE_MD_CASE(10) FHE_MD_CASE(11) FHE_MD_CASE(12)
    FHE_MD_CASE(13) FHE_MD_CASE(14) FHE_MD_CASE(15) FHE_MD_CASE(16)
#undef FHE_MD_CASE
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// mode 0: divide only; 1: + base on both polynomials (relinearize); 2: + base and
// rescale (multiply-relinearize-rescale).
cudaError_t launch_mod_down_epilogue(const PrimeTables &t, const KeySwitchTables &ks, int n,
                                     int moduli_id, int limbs, const int64_t *acc,
                                     const int64_t *base, int mode, int64_t *out, cudaStream_t s) {
  EpilogueOps ops;
  ops.base = base;
  ops.base_polys = mode == 0 ? 0 : 2;
  ops.rescale = mode == 2;
  return launch_mod_down_epilogue_ops(t, ks, n, moduli_id, limbs, acc, ops, out, s);
}

cudaError_t launch_to_ntt(const PrimeTables &t, int log_n, int polys, int limbs, int prime_base,
                          const int64_t *x, long long x_stride, int64_t *y, long long y_stride,
                          cudaStream_t s) {
  EnterLoad ld{x, x_stride, t.r_squared, t.q, t.k};
  PlainStore st{y, y_stride};
  return forward_ntt(log_n, polys, limbs, prime_base, t, ld, st, y, y_stride, s);
}

cudaError_t launch_rescale_to_ntt(const PrimeTables &t, const KeySwitchTables &ks, int log_n,
                                  int polys, int limbs, int src_moduli_id, const int64_t *x,
                                  long long x_stride, int64_t *y, long long y_stride,
                                  cudaStream_t s, const ExactLimbs &exact) {
  const long long row = static_cast<long long>(src_moduli_id) * ks.prime_count;
  PlainStore st{y, y_stride};
  if (exact.poly == ExactLimbs::kAllExact) {
    RescaleEnterLoad<false> ld{x, x_stride, ks.rescale_scale + row, ks.rescale_shoup + 2 * row,
                               t.r_squared, t.q, t.k};
    return forward_ntt(log_n, polys, limbs, src_moduli_id + 1, t, ld, st, y, y_stride, s);
  }
  RescaleEnterLoad<true> ld{x, x_stride, ks.rescale_scale + row, ks.rescale_shoup + 2 * row,
                            t.r_squared, t.q, t.k, ks.rescale_enter_shoup + 2 * row, ks.r_mod, exact};
  return forward_ntt<RescaleEnterLoad<true>, PlainStore, kNttMixed>(
      log_n, polys, limbs, src_moduli_id + 1, t, ld, st, y, y_stride, s, nullptr, nullptr, exact);
}

cudaError_t launch_attach_special_ntt(const PrimeTables &t, const KeySwitchTables &ks, int log_n,
                                      int polys, int limbs, int moduli_id, const int64_t *x,
                                      long long x_stride, int64_t *y, long long y_stride,
                                      cudaStream_t s) {
  const long long n = 1LL << log_n;
  const size_t special_bytes = static_cast<size_t>(ks.special_count) * n * sizeof(int64_t);
  for (int p = 0; p < polys; p++) {
    const cudaError_t e = cudaMemsetAsync(y + p * y_stride + limbs * n, 0, special_bytes, s);
    if (e != cudaSuccess) return e;
  }
  ProductEnterLoad ld{x, x_stride, ks.p_product_mult_r, t.r_squared, t.q, t.k};
  PlainStore st{y, y_stride};
  return forward_ntt(log_n, polys, limbs, moduli_id, t, ld, st, y, y_stride, s);
}

cudaError_t launch_to_intt(const PrimeTables &t, int log_n, int polys, int limbs, int prime_base,
                           const int64_t *x, long long x_stride, int64_t *y, long long y_stride,
                           cudaStream_t s) {
  PlainLoad ld{x, x_stride};
  EnterExitStore<false> st{y, y_stride, t.n_inverse, t.q, t.k};
  return inverse_ntt(log_n, polys, limbs, prime_base, t, ld, st, y, y_stride, s);
}

cudaError_t launch_ntt_plain(const PrimeTables &t, int log_n, int polys, int limbs, int prime_base,
                             int64_t *x, long long stride, bool inverse, cudaStream_t s) {
  PlainLoad ld{x, stride};
  PlainStore st{x, stride};
  if (inverse) return inverse_ntt(log_n, polys, limbs, prime_base, t, ld, st, x, stride, s);
  return forward_ntt(log_n, polys, limbs, prime_base, t, ld, st, x, stride, s);
}

cudaError_t launch_tensor_to_intt(const PrimeTables &t, int log_n, int limbs, int prime_base,
                                  const int64_t *a, const int64_t *b, int64_t *y, cudaStream_t s,
                                  int64_t *own_ext, const DevicePartitions *dp,
                                  const ExactLimbs &exact, bool third_only) {
  const long long stride = static_cast<long long>(limbs) << log_n;
  const int polys = third_only ? 1 : 3;
  TensorLoad ld{a, b, stride, t.q, t.k};
  ld.third_only = third_only;
  if (own_ext != nullptr) {
    if (dp == nullptr) return cudaErrorInvalidValue;
    ld.own_ext = own_ext;
    ld.part_start = dp->start;
    ld.part_size = dp->size;
    ld.part_count = dp->count;
    ld.extended = dp->extended;
  }
  if (exact.poly == ExactLimbs::kAllExact) {
    EnterExitStore<false> st{y, stride, t.n_inverse, t.q, t.k};
    return inverse_ntt(log_n, polys, limbs, prime_base, t, ld, st, y, stride, s);
  }
  MixedExitStore st{y, stride, t.n_inverse, t.q, t.k, t.exit_shoup, exact};
  const bool aligned = (reinterpret_cast<uintptr_t>(a) & 15) == 0 &&
                       (reinterpret_cast<uintptr_t>(b) & 15) == 0 &&
                       (reinterpret_cast<uintptr_t>(y) & 15) == 0 &&
                       (own_ext == nullptr || (reinterpret_cast<uintptr_t>(own_ext) & 15) == 0);
  if (third_only && log_n >= 9 && aligned) {
    // d2 first, then a plain mixed inverse transform in place.
    note_launch();
    tensor_third_kernel<<<blocks_for(static_cast<long long>(limbs) << (log_n - 1)), kThreads, 0, s>>>(
        t, ld, log_n, limbs, prime_base, y);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    PlainLoad pl{y, stride};
    return inverse_ntt<PlainLoad, MixedExitStore, kNttMixed>(log_n, 1, limbs, prime_base, t, pl, st, y,
                                                             stride, s, exact);
  }
  return inverse_ntt<TensorLoad, MixedExitStore, kNttMixed>(log_n, polys, limbs, prime_base, t, ld,
                                                            st, y, stride, s, exact);
}

}  // namespace fhe_b200
