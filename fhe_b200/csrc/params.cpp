// Host-side CKKS parameter layer (see params.hpp).
#include "params.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>

namespace fhe_b200 {

namespace {

struct PrimeTable {
  int bits;
  int coeff_count;
  int count;
  const uint64_t *values;
};

#include "prime_tables.inc"

constexpr int kNbits = 62;
constexpr int64_t kR = int64_t(1) << kNbits;
constexpr uint64_t kMask = (uint64_t(1) << kNbits) - 1;

using i128 = __int128;
using u128 = unsigned __int128;

int reverse_bits(int input, int length) {
  int out = 0;
  for (int i = 0; i < length; i++)
    if (input & (1 << i)) out |= 1 << (length - 1 - i);
  return out;
}

uint64_t mulmod_u64(uint64_t a, uint64_t b, uint64_t m) {
  return static_cast<uint64_t>((static_cast<u128>(a) * b) % m);
}

uint64_t powmod_u64(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  b %= m;
  while (e) {
    if (e & 1) r = mulmod_u64(r, b, m);
    b = mulmod_u64(b, b, m);
    e >>= 1;
  }
  return r;
}

// Scaling-prime chain of the given bit length (the reference's cached tables).
std::vector<uint64_t> cached_chain(int bits, int coeff_count, int count) {
  for (const auto &t : kPrimeTables) {
    if (t.bits == bits && t.coeff_count == coeff_count) {
      if (t.count < count) break;
      return std::vector<uint64_t>(t.values, t.values + count);
    }
  }
  throw std::invalid_argument("CKKS Parameters: unsupported config.");
}

// make_decreasing_primes (arithmetic/prime.cpp:891-909): NTT-friendly primes
// q = 1 mod 2N below 2^bits, scanned downwards in steps of 2N.
std::vector<uint64_t> decreasing_primes(int bits, int coeff_count, int count) {
  std::vector<uint64_t> primes;
  const uint64_t step = 2 * static_cast<uint64_t>(coeff_count);
  uint64_t candidate = ((uint64_t(1) << bits) / step) * step + 1;
  while (static_cast<int>(primes.size()) < count) {
    if (is_prime_u64(candidate)) primes.push_back(candidate);
    candidate -= step;
  }
  return primes;
}

}  // namespace

// ---------------------------------------------------------------- helpers --

// Deterministic Miller-Rabin for 64-bit integers (bases 2..37 suffice below 3.3e24).
bool is_prime_u64(uint64_t n) {
  if (n < 2) return false;
  static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  for (uint64_t p : small) {
    if (n % p == 0) return n == p;
  }
  uint64_t d = n - 1;
  int s = 0;
  while ((d & 1) == 0) {
    d >>= 1;
    s++;
  }
  for (uint64_t a : small) {
    uint64_t x = powmod_u64(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool composite = true;
    for (int r = 1; r < s; r++) {
      x = mulmod_u64(x, x, n);
      if (x == n - 1) {
        composite = false;
        break;
      }
    }
    if (composite) return false;
  }
  return true;
}

// Extended Euclid on signed 64-bit values (arithmetic.cpp:9-31 semantics: returns
// 0 when no inverse exists).
int64_t mod_invert(int64_t x, int64_t modulus) {
  int64_t a = x, b = modulus, ra = 1, rb = 0;
  while (b > 0) {
    const int64_t quotient = a / b;
    int64_t t = a;
    a = b;
    b = t - quotient * b;
    t = ra;
    ra = rb;
    rb = t - quotient * rb;
  }
  if (a != 1) return 0;
  return ra >= 0 ? ra : ra + modulus;
}

// Signed 128-bit product remainder (arithmetic.cpp:33-38 semantics).
int64_t mod_mul(int64_t a, int64_t b, int64_t modulus) {
  return static_cast<int64_t>((static_cast<i128>(a) * b) % modulus);
}

int64_t mod_pow(int64_t base, int64_t exponent, int64_t modulus) {
  int64_t r = 1;
  for (; exponent > 0; exponent >>= 1) {
    if (exponent & 1) r = mod_mul(r, base, modulus);
    base = mod_mul(base, base, modulus);
  }
  return r;
}

// k = -q^{-1} mod 2^62 (arithmetic.cpp:159-167).
uint64_t montgomery_k(uint64_t q) {
  const int64_t inverse = mod_invert(kR, static_cast<int64_t>(q));
  const i128 k = (static_cast<i128>(kR) * inverse - 1) / static_cast<i128>(q);
  return static_cast<uint64_t>(k);
}

// REDC with R = 2^62 on sign-extended operands (montgomery/unit.h:15-23).
int64_t host_mont_mult(int64_t a, int64_t b, uint64_t q, uint64_t k) {
  const u128 x = static_cast<u128>(static_cast<i128>(a) * static_cast<i128>(b));
  const uint64_t s = (static_cast<uint64_t>(x) * k) & kMask;
  const u128 sq = static_cast<u128>(s) * q;
  return static_cast<int64_t>(static_cast<uint64_t>((x + sq) >> kNbits));
}

// ----------------------------------------------------------------- config --

PresetInfo preset_info(SchemePreset preset) {
  switch (preset) {
    case SchemePreset::CKKS_40_60_DEFAULT: return {40, 40, 60, false, true, false};
    case SchemePreset::CKKS_54_60_BOOTSTRAP: return {54, 54, 60, true, true, false};
    case SchemePreset::CKKS_40_60_DEFAULT_ENGINE_TEST: return {40, 40, 60, false, true, true};
    case SchemePreset::CKKS_54_60_BOOTSTRAP_ENGINE_TEST: return {54, 54, 60, true, true, true};
    default: throw std::invalid_argument("CKKS Parameters: unsupported config.");
  }
}

int Config::max_log_coeff_count() const {
  const auto p = preset_info(preset);
  if (p.engine_test) return 4;
  if (p.bootstrap) return 16;
  return 17;
}

int Config::min_log_coeff_count() const {
  const auto p = preset_info(preset);
  if (p.engine_test) return 3;
  if (p.bootstrap) return 16;
  return 13;
}

// config.cpp:9-47 (thread/processor checks have no GPU counterpart).
void Config::validate() const {
  if (log_coeff_count < min_log_coeff_count())
    throw std::invalid_argument("The given log coefficient count is too small.");
  if (log_coeff_count > max_log_coeff_count())
    throw std::invalid_argument("The given log coefficient count is too large.");
  if (log_slot_count >= log_coeff_count)
    throw std::invalid_argument("The given log slot count is too large.");
  if (log_slot_count < -1)
    throw std::invalid_argument("The given log slot count is too small.");
  if (special_prime_count < 0)
    throw std::invalid_argument("The given special prime count is too small.");
  if (special_prime_count > 16)
    throw std::invalid_argument("The given special prime count is too large.");
  if (max_level < -1) throw std::invalid_argument("The given max level is too small.");
  if (max_level > 77) throw std::invalid_argument("The given max level is too large.");
}

// config.cpp:49-84: bits available for the scaling primes per ring degree.
int Config::small_prime_count() const {
  int maximum_q_bits;
  switch (log_coeff_count) {
    case 3:
    case 4: maximum_q_bits = 1000; break;
    case 13: maximum_q_bits = 214; break;
    case 14: maximum_q_bits = 430; break;
    case 15: maximum_q_bits = 868; break;
    case 16: maximum_q_bits = 1747; break;
    case 17: maximum_q_bits = 3523; break;
    default: throw std::invalid_argument("CKKS Parameters: unsupported config.");
  }
  maximum_q_bits -= 60 * (1 + special_prime_count);
  return maximum_q_bits / preset_info(preset).small_prime_bits;
}

// ------------------------------------------------------------- parameters --

Parameters::Parameters(const Config &cfg)
    : config(cfg),
      preset(preset_info(cfg.preset)),
      log_n(cfg.log_coeff_count),
      n(1 << cfg.log_coeff_count),
      special_prime_count(cfg.special_prime_count) {
  config.validate();
  small_prime_count = config.small_prime_count();
  if (small_prime_count < 2) throw std::invalid_argument("CKKS Parameters: unsupported config.");
  const int small_bits = preset.small_prime_bits;
  if (!(small_bits == 40 || small_bits == 50 || small_bits == 54))
    throw std::invalid_argument("CKKS Parameters: unsupported config.");

  // Moduli chain: parameters.cpp:9-56.  [one-more-level prime (= first special)],
  // scaling primes, base prime, special primes.
  q = cached_chain(small_bits, n, small_prime_count);
  const auto large = decreasing_primes(preset.large_prime_bits, n, special_prime_count + 1);
  q.insert(q.end(), large.begin(), large.end());
  if (preset.one_more_level) {
    // The one-more-level prime repeats the first special prime, so there must be
    // one (the reference reads past its vector here when special_prime_count == 0).
    if (large.size() < 2) throw std::invalid_argument("CKKS Parameters: unsupported config.");
    q.insert(q.begin(), large[1]);
  }
  for (auto prime : q) {
    // Below 2^61: the lazy [0, 2q) words fit the R = 2^62 Montgomery form (the
    // device's short product, mont_mult_small, relies on it).
    if (!is_prime_u64(prime) || (prime - 1) % (2 * static_cast<uint64_t>(n)) != 0 ||
        prime >= (uint64_t(1) << 61))
      throw std::runtime_error("CKKS Parameters: corrupt prime table.");
  }
  prime_count = static_cast<int>(q.size());
  chain_count = prime_count - special_prime_count;
  full_level = chain_count - 2;
  scale = std::pow(2, preset.scale_bits);
  log_slot_count = config.log_slot_count == -1 ? log_n - 1 : config.log_slot_count;
  slot_count = 1 << log_slot_count;

  // Per-level deviation of the scale from 2^scale_bits: parameters.cpp:64-104.
  {
    std::vector<long double> dev;
    int chain_index = 0;
    for (int level = full_level; level >= 0; level--) {
      if (level == full_level || (preset.one_more_level && level == full_level - 1)) {
        dev.push_back(1.0);
      } else {
        long double level_q_product = static_cast<long double>(q[chain_index - 1]);
        const auto alpha = std::pow(scale / level_q_product, 2);
        const auto deviation = std::pow(dev.back(), 2) * alpha;
        dev.push_back(deviation);
      }
      chain_index += 1;
    }
    std::reverse(dev.begin(), dev.end());
    deviations = dev;
  }

  // Per-prime tables: derived_parameters.cpp:19-50, backward paint precomputed.cpp:15-31.
  k.resize(prime_count);
  r_squared.resize(prime_count);
  n_inverse.resize(prime_count);
  root.resize(static_cast<size_t>(prime_count) * (n - 1));
  root_inverse.resize(static_cast<size_t>(prime_count) * (n - 1));
  psi.resize(prime_count);
  std::map<uint64_t, int> derived;
  for (int i = 0; i < prime_count; i++) {
    const uint64_t qi = q[i];
    auto it = derived.find(qi);
    if (it != derived.end()) {
      const int j = it->second;
      k[i] = k[j];
      r_squared[i] = r_squared[j];
      n_inverse[i] = n_inverse[j];
      psi[i] = psi[j];
      std::copy_n(&root[size_t(j) * (n - 1)], n - 1, &root[size_t(i) * (n - 1)]);
      std::copy_n(&root_inverse[size_t(j) * (n - 1)], n - 1, &root_inverse[size_t(i) * (n - 1)]);
      continue;
    }
    derived[qi] = i;
    const int64_t qs = static_cast<int64_t>(qi);
    r_squared[i] = mod_mul(kR, kR, qs);
    k[i] = montgomery_k(qi);
    n_inverse[i] = mod_mul(mod_invert(n, qs), kR, qs);
    // psi: first base whose ((q-1)/2N)-th power has order 2N (arithmetic.cpp:97-113).
    const int64_t unit_power = (qs - 1) / (2 * static_cast<int64_t>(n));
    int64_t psi = 0;
    for (int64_t base = 2; base < qs; base++) {
      psi = mod_pow(base, unit_power, qs);
      if (mod_pow(psi, n, qs) != 1) break;
    }
    this->psi[i] = psi;
    const int64_t psi_inv = mod_invert(psi, qs);
    std::vector<int64_t> fwd(n), inv(n);
    int64_t a = 1, b = 1;
    for (int j = 0; j < n; j++) {
      fwd[reverse_bits(j, log_n)] = a;
      inv[reverse_bits(j, log_n)] = b;
      a = mod_mul(a, psi, qs);
      b = mod_mul(b, psi_inv, qs);
    }
    int64_t *rt = &root[size_t(i) * (n - 1)];
    int64_t *ri = &root_inverse[size_t(i) * (n - 1)];
    for (int j = 1; j < n; j++) rt[j - 1] = host_mont_mult(fwd[j], r_squared[i], qi, k[i]);
    int o = 0;
    for (int lci = log_n - 1; lci >= 0; lci--) {
      const int groups = 1 << lci;
      for (int g = 0; g < groups; g++)
        ri[o++] = host_mont_mult(inv[groups + g], r_squared[i], qi, k[i]);
    }
  }

  // Key-switching and rescale constants: precomputed.cpp:89-126.
  p_product_mult_r.resize(chain_count);
  for (int qi = 0; qi < chain_count; qi++) {
    int64_t product = kR;
    for (int p = chain_count; p < prime_count; p++)
      product = mod_mul(product, static_cast<int64_t>(q[p]), static_cast<int64_t>(q[qi]));
    p_product_mult_r[qi] = product;
  }
  p_inverse_mult_r.resize(special_prime_count);
  for (int s = 0; s < special_prime_count; s++) {
    const int p_index = prime_count - 1 - s;
    const int64_t p = static_cast<int64_t>(q[p_index]);
    auto &v = p_inverse_mult_r[s];
    v.resize(p_index);
    for (int qi = 0; qi < p_index; qi++) {
      const int64_t qq = static_cast<int64_t>(q[qi]);
      v[qi] = mod_mul(mod_invert(p, qq), kR, qq);
    }
  }
  rescale_scale.resize(prime_count > 0 ? prime_count - 1 : 0);
  for (int from = 0; from + 1 < prime_count; from++) {
    auto &v = rescale_scale[from];
    for (int to = from + 1; to < prime_count; to++) {
      const int64_t qt = static_cast<int64_t>(q[to]);
      v.push_back(mod_mul(mod_invert(static_cast<int64_t>(q[from]), qt), kR, qt));
    }
  }
}

int Parameters::max_level() const {
  return config.max_level == -1 ? full_level : config.max_level;
}

// parameters.cpp:203-212
int Parameters::max_key_switching_level() const {
  if (preset.one_more_level && max_level() == full_level) return full_level - 1;
  return max_level();
}

int Parameters::moduli_id(int level) const {
  if (level < -1 || level > full_level) throw std::out_of_range("level out of range");
  return full_level - level;
}

int Parameters::chains(int moduli_id, bool include_special) const {
  return chain_count - moduli_id + (include_special ? special_prime_count : 0);
}

// data.h:21-32 (limbs = level + 2 before rescale, level + 1 after).
int Parameters::level_of(int moduli_id, bool rescaled) const {
  const int c = chains(moduli_id);
  return rescaled ? c - 1 : c - 2;
}

// parameters.cpp:325-332
int Parameters::partition_count(int moduli_id) const {
  const int K = special_prime_count;
  return (chains(moduli_id) + K - 1) / K;
}

// parameters.cpp:334-360
std::vector<Partition> Parameters::partitions(int moduli_id, int key_moduli_id) const {
  const int K = special_prime_count;
  const int L = chains(moduli_id);
  const int pc = partition_count(moduli_id);
  int index = partition_count(key_moduli_id) - pc;
  std::vector<Partition> out;
  for (int start = L - pc * K; start < L; start += K, index++) {
    const int lo = std::max(0, start);
    const int hi = std::min(L, start + K);
    out.push_back({lo, hi - lo, index});
  }
  return out;
}

// precomputed.cpp:326-382.  The product of the partition's leading primes is
// carried as residues modulo each prime that needs it (the reference uses a BigInt).
PartitionConstants Parameters::partition_constants(int moduli_id, const Partition &p) const {
  PartitionConstants pc;
  pc.size = p.size;
  const int P = chains(moduli_id, true);
  const uint64_t *qq = q.data() + moduli_id;
  const int64_t *r2 = r_squared.data() + moduli_id;
  auto product_mod = [&](int count, int64_t m) {
    int64_t acc = 1;
    for (int z = 0; z < count; z++)
      acc = mod_mul(acc, static_cast<int64_t>(qq[p.start + z] % static_cast<uint64_t>(m)), m);
    return acc;
  };
  pc.product_r_squared.resize(static_cast<size_t>(std::max(p.size - 1, 0)) * P);
  for (int ci = 1; ci < p.size; ci++) {
    const int64_t chain_q = static_cast<int64_t>(qq[p.start + ci]);
    const int64_t inverse = mod_invert(product_mod(ci, chain_q), chain_q);
    pc.inverse_r.push_back((chain_q & 1) == 0 ? inverse : mod_mul(inverse, kR, chain_q));
    if (ci < p.size - 1) {
      std::vector<int64_t> row;
      for (int mi = ci + 1; mi < p.size; mi++) {
        const int64_t mq = static_cast<int64_t>(qq[p.start + mi]);
        const int64_t v = product_mod(ci, mq);
        row.push_back((mq & 1) == 0 ? v : mod_mul(v, kR, mq));
      }
      pc.product_r.push_back(row);
    }
    for (int mi = 0; mi < P; mi++) {
      const int64_t mq = static_cast<int64_t>(qq[mi]);
      const int64_t v = product_mod(ci, mq);
      pc.product_r_squared[static_cast<size_t>(ci - 1) * P + mi] =
          (mq & 1) == 0 ? v : mod_mul(v, r2[mi], mq);
    }
  }
  return pc;
}

// parameters.cpp:178-187
uint64_t Parameters::base_prime() const {
  int index = small_prime_count;
  if (preset.one_more_level) index += 1;
  return q[index];
}

long double Parameters::rescaled_scale(long double s, int moduli_id) const {
  return s / q[moduli_id];
}

}  // namespace fhe_b200

namespace fhe_b200 {

namespace {

// (round(value) * 2^62) mod q for the non-negative double `value`: the
// BigInt::from_double(std::round(value)) * r_ % q of precomputed.cpp:418-462.
int64_t rounded_times_r_mod(double value, uint64_t q) {
  const double r = std::round(value);
  if (!(r >= 0.0) || r >= 18446744073709551616.0)
    throw std::invalid_argument("level down multiplier out of range");
  const unsigned __int128 v = static_cast<unsigned __int128>(static_cast<uint64_t>(r)) << 62;
  return static_cast<int64_t>(v % q);
}

// get_jump: ckks/encode.cpp:44-56.
int64_t rotation_jump(unsigned long shift, unsigned long double_size) {
  if (shift == double_size - 1) return static_cast<int64_t>(shift);
  int64_t jump = 1;
  for (unsigned long power = 0; power < double_size - shift; power++) {
    jump *= 5;
    jump &= static_cast<int64_t>(double_size - 1);
  }
  return jump;
}

int reverse_low_bits(int x, int bits) {
  int y = 0;
  for (int b = 0; b < bits; b++) y |= ((x >> b) & 1) << (bits - 1 - b);
  return y;
}

}  // namespace

std::vector<int32_t> signed_permutation(int n, int delta) {
  const unsigned long double_size = static_cast<unsigned long>(n) * 2;
  const unsigned long shift =
      (static_cast<unsigned long>(static_cast<long>(delta)) + double_size) % double_size;
  const int64_t jump = rotation_jump(shift, double_size);
  std::vector<int32_t> out(n);
  for (int c = 0; c < n; c++) {
    const unsigned long index = static_cast<unsigned long>(jump) * c % double_size;
    const int32_t to = static_cast<int32_t>(index % n);
    out[c] = ((index / n) & 1) ? ~to : to;
  }
  return out;
}

std::vector<int32_t> ntt_permutation(int n, int delta) {
  const int mask = n - 1;
  const uint32_t m2 = static_cast<uint32_t>(n) * 2;
  // modulus_power<uint32_t>(5, delta, 2N): arithmetic/arithmetic.cpp:40-52.
  uint64_t power = 1, base = 5;
  for (uint32_t e = static_cast<uint32_t>(delta); e > 0; e >>= 1) {
    if (e & 1) power = power * base % m2;
    base = base * base % m2;
  }
  const int64_t power_of_five = static_cast<int64_t>(power) & mask;
  const int diff = delta == -1 ? -1 : static_cast<int>(((power - 1) >> 1) & mask);
  const int64_t inverse = delta == -1 ? n - 1 : mod_invert(power_of_five, n);
  int log_n = 0;
  while ((1 << log_n) < n) log_n++;
  std::vector<int32_t> tmp(n), out(n);
  for (int i = 0; i < n; i++) {
    const int64_t index = ((i - diff) % n + n) % n;
    tmp[i] = static_cast<int32_t>(index * inverse % n);
  }
  for (int i = 0; i < n; i++) out[i] = reverse_low_bits(tmp[reverse_low_bits(i, log_n)], log_n);
  return out;
}

std::vector<int64_t> Parameters::level_down_multiplier(int source_level,
                                                       int destination_level) const {
  // CKKSPrecomputed::make_level_down_multiplier (precomputed.cpp:438-462); the
  // deviations are the double copies the precomputed tables hold.
  const int source_moduli_id = moduli_id(source_level);
  const double source_deviation = static_cast<double>(deviations[source_level]);
  const double destination_deviation = static_cast<double>(deviations[destination_level]);
  const double diff = destination_deviation / source_deviation;
  double delta;
  if (preset.one_more_level && source_moduli_id == 0)
    delta = scale * diff;
  else
    delta = static_cast<double>(q[source_moduli_id]) * diff;
  std::vector<int64_t> out;
  for (int i = source_moduli_id; i < chain_count; i++) out.push_back(rounded_times_r_mod(delta, q[i]));
  return out;
}

std::vector<int64_t> Parameters::level_down_multiplier_after_rescale(int source_level,
                                                                     int destination_level) const {
  // make_level_down_multiplier_after_rescale (precomputed.cpp:418-436).
  const double source_deviation = static_cast<double>(deviations[source_level - 1]);
  const double destination_deviation = static_cast<double>(deviations[destination_level]);
  const double diff = destination_deviation / std::sqrt(source_deviation);
  const double delta = scale * diff;
  std::vector<int64_t> out;
  for (int i = moduli_id(destination_level); i < chain_count; i++)
    out.push_back(rounded_times_r_mod(delta, q[i]));
  return out;
}

long double Parameters::level_down_scale(int level) const {
  // core.cpp:743-750: deviation (double) * scale * scale in long double.
  const long double s = scale;
  return static_cast<double>(deviations[level]) * s * s;
}

}  // namespace fhe_b200

// ------------------------------------------------------------ encode/decode --

namespace fhe_b200 {

namespace {

// circular_shift_permutation, fold_canon_permutation, get_permutation_cycles,
// conjugate_permutations and invert_permutation of ckks/encode.cpp:25-154.
std::vector<uint64_t> circular_shift(int size) {
  const int half = size / 2;
  std::vector<uint64_t> out(size);
  out[0] = half - 1;
  for (int i = 1; i < half; i++) out[i] = i - 1;
  for (int i = half; i < size - 1; i++) out[i] = i + 1;
  out[size - 1] = half;
  return out;
}

std::vector<uint64_t> fold_canon(int size) {
  const int double_size = size * 2;
  const int64_t jump = rotation_jump(1, double_size);
  std::vector<uint64_t> out(size);
  int64_t jm = jump;
  for (int i = 0; i < size; i++) {
    out[i] = static_cast<uint64_t>((jm - 1) >> 1);
    jm = (jm + jump * 2) % double_size;
  }
  return out;
}

std::vector<uint64_t> permutation_cycles(const std::vector<uint64_t> &p) {
  const int size = static_cast<int>(p.size());
  std::vector<bool> visited(size, false);
  std::vector<uint64_t> out;
  out.reserve(size);
  int start = 0;
  while (start < size) {
    uint64_t cur = p[start], next = p[cur];
    while (true) {
      out.push_back(cur);
      visited[cur] = true;
      cur = next;
      if (visited[next]) break;
      next = p[cur];
    }
    start++;
    while (start < size && visited[start]) start++;
  }
  return out;
}

}  // namespace

CodecTables Parameters::codec_tables() const {
  CodecTables t;
  const int codec = slot_count * 2;
  t.codec = codec;
  const auto c1 = permutation_cycles(fold_canon(codec));
  const auto c2 = permutation_cycles(circular_shift(codec));
  std::vector<uint64_t> post(codec), pre(codec);
  for (int i = 0; i < codec; i++) post[c1[i]] = c2[i];
  for (int i = 0; i < codec; i++) pre[post[i]] = i;
  t.pre.assign(pre.begin(), pre.end());
  t.post.assign(post.begin(), post.end());
  // precomputed.cpp:67-74 (std::numbers::pi).
  const double pi = 3.141592653589793;
  const double unit_angle = -2 * pi / codec;
  t.fft_cos.resize(codec);
  t.fft_sin.resize(codec);
  t.ifft_cos.resize(codec);
  t.ifft_sin.resize(codec);
  for (int i = 0; i < codec; i++) {
    const double angle = i * unit_angle;
    t.fft_cos[i] = std::cos(angle);
    t.fft_sin[i] = std::sin(angle);
    t.ifft_cos[i] = std::cos(angle);
    t.ifft_sin[i] = std::sin(-angle);
  }
  // apply_twister_ / apply_skewer_ (core_calculate.cpp:539-566, encode.cpp:279-301).
  const int y_count = codec * 2;
  const double twist_step = -pi / y_count;
  const double skew_step = pi / y_count;
  t.twist_cos.resize(codec);
  t.twist_sin.resize(codec);
  t.skew_cos.resize(codec);
  t.skew_sin.resize(codec);
  for (int i = 0; i < codec; i++) {
    const int real_index = 2 * i;
    t.twist_cos[i] = std::cos(real_index * twist_step);
    t.twist_sin[i] = std::sin(real_index * twist_step);
    t.skew_cos[i] = std::cos(real_index * skew_step);
    t.skew_sin[i] = std::sin(real_index * skew_step);
  }
  return t;
}

long double Parameters::ckks_scale(int level) const {
  // precomputed.cpp:144-155.
  const int mid = moduli_id(level);
  const double deviation = static_cast<double>(deviations[level]);
  long double s = static_cast<long double>(deviation) * scale * scale;
  if (preset.one_more_level && mid == 0) s = scale * static_cast<long double>(q[0]);
  return s;
}

EncodeLevel Parameters::encode_level(int level) const {
  // precomputed.cpp:139-215 (no flexible chain: its scale bit is always 0).
  EncodeLevel e;
  int mid = moduli_id(level);
  int chains_here = chains(mid, true);
  const int log_scale = preset.scale_bits;
  const long double ckks = ckks_scale(level);
  e.ckks_scale = ckks;
  const uint64_t p0 = q[mid];
  e.max_level_in_one_more_level = preset.one_more_level && mid == 0 && (ckks >= p0 * scale);
  if (e.max_level_in_one_more_level) {
    e.scale_before_tile = static_cast<double>(ckks / p0);
    chains_here -= 1;
    mid = moduli_id(level - 1);
  } else {
    int exponent = 0;
    const double mantissa = static_cast<double>(std::frexp(ckks, &exponent));
    if (exponent >= log_scale) {
      e.scale_before_tile = mantissa * scale;
      e.log_scale_after_tile = exponent - log_scale;
    } else {
      e.scale_before_tile = static_cast<double>(ckks);
      e.log_scale_after_tile = 0;
    }
  }
  e.first_moduli_id = mid;
  const int64_t r = INT64_C(1) << 62;
  e.r_mult_scale_after_tile.resize(chains_here);
  if (e.max_level_in_one_more_level) {
    for (int j = 0; j < chains_here; j++)
      e.r_mult_scale_after_tile[j] = mod_mul(r, static_cast<int64_t>(p0), static_cast<int64_t>(q[mid + j]));
  } else {
    for (int j = 0; j < chains_here; j++)
      e.r_mult_scale_after_tile[j] = r % static_cast<int64_t>(q[mid + j]);
    for (int64_t ls = e.log_scale_after_tile; ls > 0; ls -= 60) {
      const int64_t partial = INT64_C(1) << std::min<int64_t>(60, ls);
      for (int j = 0; j < chains_here; j++)
        e.r_mult_scale_after_tile[j] =
            mod_mul(e.r_mult_scale_after_tile[j], partial, static_cast<int64_t>(q[mid + j]));
    }
  }
  return e;
}

}  // namespace fhe_b200
