// Host check of the device modular arithmetic (fhe_b200/csrc/modarith.cuh compiles
// as plain C++): the short Montgomery product of the NTT's in-range butterflies
// must give the same word as the general sign-extended form, for random odd q
// below 2^61 (k = -q^-1 mod 2^62) and operands below 2^62, edge values included;
// Shoup's product of the value-only butterflies must give W b mod q up to one q,
// for any b below 2^64; and the reduced exit of ModDown's inverse transform (one
// Shoup product by N^-1 R^-1) must give the word of mont_exit(mont_mult(v, N^-1 R))
// reduced to [0, q), for engine primes and v below 2^62; and the rescale word with
// Shoup's product must equal the reference's form for any words.
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
  const uint64_t primes[] = {1152921504598720513ull, 18014398506729473ull, 18014398514987009ull,
                             1099511480321ull};
  for (uint64_t q : primes) {
    using u128 = unsigned __int128;
    auto mulmod = [&](uint64_t a, uint64_t b) { return static_cast<uint64_t>(static_cast<u128>(a) * b % q); };
    auto powmod = [&](uint64_t a, uint64_t e) {
      uint64_t r = 1;
      for (a %= q; e; e >>= 1, a = mulmod(a, a))
        if (e & 1) r = mulmod(r, a);
      return r;
    };
    const uint64_t k = negated_inverse(q);
    const uint64_t r_inverse = powmod((uint64_t(1) << 62) % q, q - 2);
    const uint64_t n_inverse_r = mulmod(powmod(uint64_t(1) << 16, q - 2), (uint64_t(1) << 62) % q);
    const uint64_t c = mulmod(mulmod(n_inverse_r, r_inverse), r_inverse);
    const uint64_t c_shoup = static_cast<uint64_t>((static_cast<u128>(c) << 64) / q);
    for (long it = 0; it < iterations / 8; it++) {
      uint64_t v = rng() & top;
      if (it % 3 == 0) v = rng() % (2 * q);
      if (it % 7 == 0) v = rng() & 3;
      const int64_t want = guard(mont_exit(mont_mult_lazy(static_cast<int64_t>(v), static_cast<int64_t>(n_inverse_r), q, k), q, k),
                                 static_cast<int64_t>(q));
      uint64_t r = shoup_mult(c, c_shoup, v, q);
      r = r >= q ? r - q : r;
      if (static_cast<int64_t>(r) != want) bad++;
    }
  }
  for (size_t a = 0; a < sizeof(primes) / sizeof(primes[0]); a++) {
    for (size_t b = 0; b < sizeof(primes) / sizeof(primes[0]); b++) {
      if (a == b) continue;
      const uint64_t q0 = primes[a], q = primes[b];  // drop q0, rescale limb mod q
      using u128 = unsigned __int128;
      auto mulmod = [&](uint64_t x, uint64_t y) { return static_cast<uint64_t>(static_cast<u128>(x) * y % q); };
      auto powmod = [&](uint64_t x, uint64_t e) {
        uint64_t r = 1;
        for (x %= q; e; e >>= 1, x = mulmod(x, x))
          if (e & 1) r = mulmod(r, x);
        return r;
      };
      const uint64_t k = negated_inverse(q), r_mod = (uint64_t(1) << 62) % q;
      const uint64_t plain = powmod(q0 % q, q - 2);             // q0^-1 mod q
      const int64_t mont = static_cast<int64_t>(mulmod(plain, r_mod));  // q0^-1 R mod q
      const int64_t pair[2] = {static_cast<int64_t>(plain),
                               static_cast<int64_t>((static_cast<u128>(plain) << 64) / q)};
      for (long it = 0; it < iterations / 32; it++) {
        int64_t xj = static_cast<int64_t>(rng() % q), x0 = static_cast<int64_t>(rng() % q0);
        if (it % 5 == 0) xj = static_cast<int64_t>(rng());  // any word, negative ones included
        if (it % 7 == 0) x0 = static_cast<int64_t>(rng() % (2 * q0));
        const int64_t rounder = static_cast<uint64_t>(x0) > (q0 >> 1) ? 1 : 0;
        if (rescale_word_shoup(xj, x0, rounder, q, k, mont, pair) != rescale_word(xj, x0, rounder, q, k, mont))
          bad++;
      }
    }
  }
  std::printf("%ld\n", bad);
  return 0;
}
