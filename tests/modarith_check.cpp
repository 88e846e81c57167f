// Host check of the device modular arithmetic (fhe_b200/csrc/modarith.cuh compiles
// as plain C++): the short Montgomery product of the NTT's in-range butterflies
// must give the same word as the general sign-extended form, for random odd q
// below 2^61 (k = -q^-1 mod 2^62) and operands below 2^62, edge values included;
// Shoup's product of the value-only butterflies must give W b mod q up to one q,
// for any b below 2^64.
// Usage: modarith_check <iterations> <seed>; prints the mismatch count.
#include <cstdio>
#include <cstdlib>
#include <random>

#include "modarith.cuh"

using namespace fhe_b200;

static uint64_t negated_inverse(uint64_t q) {
  uint64_t x = 1;  // Newton's iteration doubles the correct low bits each step
  for (int i = 0; i < 7; i++) x *= 2 - q * x;
  return (0 - x) & kMontMask;
}

int main(int argc, char **argv) {
  const long iterations = argc > 1 ? std::atol(argv[1]) : 1000000;
  std::mt19937_64 rng(argc > 2 ? std::atoll(argv[2]) : 1);
  const uint64_t top = (uint64_t(1) << 62) - 1;
  long bad = 0;
  for (long it = 0; it < iterations; it++) {
    uint64_t q = (rng() & ((uint64_t(1) << 61) - 1)) | 1;
    if (it % 5 == 0) q = ((uint64_t(1) << 61) - 1) - 2 * (rng() & 0xFF);
    if (it % 5 == 1) q = (rng() & ((uint64_t(1) << 40) - 1)) | (uint64_t(1) << 39) | 1;
    const uint64_t k = negated_inverse(q);
    uint64_t w = rng() & top, b = rng() & top;
    if (it % 3 == 0) w = top - (rng() & 0xFFFF);
    if (it % 7 == 0) b = top - (rng() & 0xFFFF);
    if (it % 13 == 0) b = rng() & 0xFF;
    if (it % 4 == 2) b = rng() % (2 * q);
    if (it % 4 == 3) w = rng() % (2 * q);
    const int64_t want = mont_mult_const(static_cast<int64_t>(w), static_cast<int64_t>(b), q, k);
    if (mont_mult_small(w, b, q, k) != want) bad++;
    const uint64_t plain = w % q, any = (it % 11 == 0) ? ~(rng() & 0xFFFF) : rng();
    const uint64_t shoup = static_cast<uint64_t>((static_cast<unsigned __int128>(plain) << 64) / q);
    const uint64_t r = shoup_mult(plain, shoup, any, q);
    const uint64_t exact = static_cast<uint64_t>(static_cast<unsigned __int128>(plain) * any % q);
    if (!(r < 2 * q && r % q == exact)) bad++;
  }
  std::printf("%ld\n", bad);
  return 0;
}
