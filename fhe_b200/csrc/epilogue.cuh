// The output stage of a ModDown epilogue, shared by the CUDA-core and the
// tensor-core kernels: the divided limbs (the exact division by the special primes,
// make_unsigned_reduce_2q_to_q, canonical in [0, q)) combined with the caller's
// operations (core_key_switch.cpp:110-160 and its callers).
#pragma once

#include "kernels.cuh"
#include "modarith.cuh"

namespace fhe_b200 {

// A CTA owns coefficients [coeff0, coeff0 + valid) of polynomial `poly`; divide(j, c)
// gives the divided limb j of coefficient coeff0 + c.  first_limb holds at least
// `valid` words of shared memory.  Every thread of the CTA calls this.  The rescale's
// product is Shoup's when its operand is in range (rescale_word_shoup, same word);
// LAZY is kept for the callers' signatures and selects nothing else.
template <bool LAZY = false, class Divide>
__device__ __forceinline__ void mod_down_store(const PrimeTables &t, const KeySwitchTables &ks,
                                               int n, int moduli_id, int L, int poly, int coeff0,
                                               int valid, const EpilogueOps &ops, int64_t *out,
                                               int64_t *first_limb, Divide divide) {
  const int P = ks.prime_count;
  const long long in_stride = static_cast<long long>(L) * n;
  const bool add_base = poly < ops.base_polys;  // uniform per CTA
  const int64_t *b = add_base ? ops.base + poly * in_stride + coeff0 : nullptr;
  auto combined = [&](int j, int c) -> int64_t {
    const int64_t qs = static_cast<int64_t>(t.q[moduli_id + j]);
    if (!add_base) return divide(j, c);
    return guard(guard(b[static_cast<long long>(j) * n + c] + divide(j, c), qs << 1), qs);
  };

  if (!ops.rescale) {
    int64_t *o = out + poly * in_stride;
    if (ops.signed_perm == nullptr) {
      for (int w = threadIdx.x; w < L * valid; w += blockDim.x) {
        const int j = w / valid, c = w % valid;
        o[static_cast<long long>(j) * n + coeff0 + c] = combined(j, c);
      }
      return;
    }
    // Permuted store (rotate_ after key_switch_mod_down, core.cpp:939-952).
    for (int w = threadIdx.x; w < L * valid; w += blockDim.x) {
      const int j = w / valid, c = w % valid;
      const int64_t qs = static_cast<int64_t>(t.q[moduli_id + j]);
      const int32_t pc = ops.signed_perm[coeff0 + c];
      int64_t v = combined(j, c);
      if (pc < 0) v = -v;
      v = v < 0 ? v + qs : guard(v, qs);
      o[static_cast<long long>(j) * n + (pc < 0 ? ~pc : pc)] = v;
    }
    return;
  }
  // Rescale of the combined polynomial (core_rescale.cpp:5-25).
  for (int c = threadIdx.x; c < valid; c += blockDim.x) first_limb[c] = combined(0, c);
  __syncthreads();
  const long long out_stride = static_cast<long long>(L - 1) * n;
  int64_t *o = out + poly * out_stride + coeff0;
  const uint64_t q_half = t.q[moduli_id] >> 1;  // unsigned comparison, as get_rounder
  for (int w = threadIdx.x; w < (L - 1) * valid; w += blockDim.x) {
    const int j = 1 + w / valid, c = w % valid;
    const int prime = moduli_id + j;
    const int64_t y0 = first_limb[c];
    o[static_cast<long long>(j - 1) * n + c] =
        rescale_word_shoup(combined(j, c), y0, static_cast<uint64_t>(y0) > q_half ? 1 : 0, t.q[prime],
                           t.k[prime], ks.rescale_scale[static_cast<long long>(moduli_id) * P + prime],
                           ks.rescale_shoup + 2 * (static_cast<long long>(moduli_id) * P + prime));
  }
}

}  // namespace fhe_b200
