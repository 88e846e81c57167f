// Device-side modular arithmetic of the B200 CKKS engine.
//
// Words are int64 holding residues; like the reference (DESILO FHE
// montgomery/unit.h:10-31, montgomery/compound.cpp) every comparison is signed and
// the REDC product is formed from sign-extended operands, so out-of-range
// intermediates evaluate to the same words as on the CPU.  R = 2^62.
#pragma once

#include <cstdint>

namespace fhe_b200 {

constexpr int kMontBits = 62;
constexpr uint64_t kMontMask = (uint64_t(1) << kMontBits) - 1;

// (x < q) ? x : x - q  (unit.h:13)
__device__ __forceinline__ int64_t guard(int64_t x, int64_t q) { return x < q ? x : x - q; }

// REDC(a * b) with R = 2^62: bits [62, 126) of a*b + s*q, s = (a*b*k) mod 2^62
// (unit.h:15-23).  a and b are sign-extended to 128 bits as in the reference.
__device__ __forceinline__ int64_t mont_mult(int64_t a, int64_t b, uint64_t q, uint64_t k) {
  const uint64_t lo = static_cast<uint64_t>(a) * static_cast<uint64_t>(b);
  const uint64_t hi = static_cast<uint64_t>(__mul64hi(a, b));
  const uint64_t s = (lo * k) & kMontMask;
  const uint64_t sq_lo = s * q;
  const uint64_t sq_hi = __umul64hi(s, q);
  const uint64_t sum_lo = lo + sq_lo;
  const uint64_t sum_hi = hi + sq_hi + (sum_lo < lo ? 1 : 0);
  return static_cast<int64_t>((sum_hi << 2) | (sum_lo >> kMontBits));
}

// Montgomery exit (unit.h:25-31): REDC of a single (sign-extended) word.
__device__ __forceinline__ int64_t mont_exit(int64_t x, uint64_t q, uint64_t k) {
  const uint64_t s = (static_cast<uint64_t>(x) * k) & kMontMask;
  const uint64_t sq_lo = s * q;
  const uint64_t sq_hi = __umul64hi(s, q);
  const uint64_t lo = static_cast<uint64_t>(x);
  const uint64_t sum_lo = lo + sq_lo;
  const uint64_t sign = x < 0 ? ~uint64_t(0) : 0;
  const uint64_t sum_hi = sign + sq_hi + (sum_lo < lo ? 1 : 0);
  return static_cast<int64_t>((sum_hi << 2) | (sum_lo >> kMontBits));
}

// Per-prime constants as the kernels read them.
struct PrimeTables {
  const uint64_t *q;
  const uint64_t *k;
  const int64_t *r_squared;
  const int64_t *n_inverse;
  const int64_t *root;          // [prime][N-1]
  const int64_t *root_inverse;  // [prime][N-1]
  int log_n;
};

}  // namespace fhe_b200
