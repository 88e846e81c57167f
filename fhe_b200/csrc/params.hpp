// Host-side CKKS parameter layer of the B200 engine.
//
// Builds the moduli chain, the level <-> moduli-id bookkeeping and every per-prime
// constant the device kernels consume, identically to the reference
// (DESILO FHE: ckks/config.cpp, ckks/parameters.cpp, ckks/precomputed.cpp,
// ckks/derived_parameters.cpp), so that limbs computed on the GPU are bit-exact
// with the reference CPU implementation.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fhe_b200 {

// engine/scheme_preset.h: SchemePreset values and their (scale bits, small-prime
// bits, large-prime bits, bootstrap, one-more-level, engine-test) table.
enum class SchemePreset : int {
  NONE = 0,
  CKKS_40_60_DEFAULT = 1,
  CKKS_54_60_BOOTSTRAP = 2,
  CKKS_40_60_DEFAULT_ENGINE_TEST = 3,
  CKKS_54_60_BOOTSTRAP_ENGINE_TEST = 4,
};

struct PresetInfo {
  int scale_bits;
  int small_prime_bits;
  int large_prime_bits;
  bool bootstrap;
  bool one_more_level;
  bool engine_test;
};

PresetInfo preset_info(SchemePreset preset);

// ckks/config.h: CKKSConfig (processor/thread fields have no meaning on the GPU).
struct Config {
  int log_coeff_count = 14;
  int log_slot_count = -1;
  int special_prime_count = 1;
  int max_level = -1;
  SchemePreset preset = SchemePreset::CKKS_40_60_DEFAULT;

  void validate() const;  // throws std::invalid_argument, messages as config.cpp:9-47
  int small_prime_count() const;
  int max_log_coeff_count() const;
  int min_log_coeff_count() const;
};

struct Partition {
  int start;            // offset from the ciphertext's moduli id
  int size;             // alpha
  int partition_index;  // selects key polynomials 2*index, 2*index+1
};

// Mixed-radix (Garner) constants of one partition: precomputed.cpp:326-382.
struct PartitionConstants {
  int size = 0;
  std::vector<int64_t> inverse_r;                 // [size-1]
  std::vector<std::vector<int64_t>> product_r;    // [size-2][size-ci-1]
  std::vector<int64_t> product_r_squared;         // [(size-1) * prime_count(moduli_id)]
};

// Host tables of the canonical-embedding codec (precomputed.cpp:49-74 and the
// cos/sin factors of apply_twister / apply_skewer), for codec = 2 * slot_count.
struct CodecTables {
  int codec = 0;
  std::vector<int32_t> pre, post;  // pre_permutation_, post_permutation_
  std::vector<double> fft_cos, fft_sin, ifft_cos, ifft_sin;
  std::vector<double> twist_cos, twist_sin, skew_cos, skew_sin;
};

// Per-level encode constants (precomputed.cpp:139-215).
struct EncodeLevel {
  long double ckks_scale = 0;
  double scale_before_tile = 0;
  int64_t log_scale_after_tile = 0;
  bool max_level_in_one_more_level = false;
  int first_moduli_id = 0;  // moduli id of r_mult_scale_after_tile[0]
  std::vector<int64_t> r_mult_scale_after_tile;
};

class Parameters {
 public:
  explicit Parameters(const Config &config);

  const Config config;
  const PresetInfo preset;
  const int log_n;
  const int n;
  const int special_prime_count;  // K
  int small_prime_count = 0;
  int chain_count = 0;  // C: non-special primes at moduli id 0
  int prime_count = 0;  // P = C + K
  int full_level = 0;
  int log_slot_count = 0;
  int slot_count = 0;
  double scale = 0;

  std::vector<uint64_t> q;           // [P]  q_[0] .. q_[P-1], specials last
  std::vector<uint64_t> k;           // [P]  -q^-1 mod 2^62
  std::vector<int64_t> r_squared;    // [P]  2^124 mod q
  std::vector<int64_t> n_inverse;    // [P]  N^-1 * 2^62 mod q
  std::vector<int64_t> root;         // [P][N-1] bit-reversed psi powers, Montgomery form
  std::vector<int64_t> root_inverse; // [P][N-1] backward-paint inverse powers
  std::vector<int64_t> psi;          // [P]  the primitive 2N-th root the tables are built from
  std::vector<int64_t> p_product_mult_r;               // [C]
  std::vector<std::vector<int64_t>> p_inverse_mult_r;  // [K][p_index]
  std::vector<std::vector<int64_t>> rescale_scale;     // [P-1][P-from-1]
  std::vector<long double> deviations;                 // [full_level + 1]

  int max_level() const;
  int max_key_switching_level() const;
  int moduli_id(int level) const;  // throws std::out_of_range for a bad level
  int chains(int moduli_id, bool include_special = false) const;
  int level_of(int moduli_id, bool rescaled) const;
  int partition_count(int moduli_id) const;
  std::vector<Partition> partitions(int moduli_id, int key_moduli_id) const;
  PartitionConstants partition_constants(int moduli_id, const Partition &p) const;
  uint64_t base_prime() const;
  long double rescaled_scale(long double scale, int moduli_id) const;
  // Per-limb Montgomery multipliers of level_down, from the moduli id of the
  // source level (resp. destination level after a rescale) to the last scaling prime.
  std::vector<int64_t> level_down_multiplier(int source_level, int destination_level) const;
  std::vector<int64_t> level_down_multiplier_after_rescale(int source_level,
                                                           int destination_level) const;
  long double level_down_scale(int level) const;
  CodecTables codec_tables() const;
  long double ckks_scale(int level) const;
  EncodeLevel encode_level(int level) const;
};

// get_permutation_and_sign (ckks/encode.cpp:513-526) for a rotation by `delta`
// (-1: conjugation), encoded as perm[c] or ~perm[c] where the sign is -1.
std::vector<int32_t> signed_permutation(int n, int delta);
// get_ntt_permutation (ckks/encode.cpp:528-557): NTT-form rotation gather indices.
std::vector<int32_t> ntt_permutation(int n, int delta);

// Modular helpers shared with the engine (arithmetic/arithmetic.cpp semantics).
int64_t mod_invert(int64_t x, int64_t modulus);
int64_t mod_mul(int64_t a, int64_t b, int64_t modulus);
int64_t mod_pow(int64_t base, int64_t exponent, int64_t modulus);
uint64_t montgomery_k(uint64_t q);
int64_t host_mont_mult(int64_t a, int64_t b, uint64_t q, uint64_t k);
bool is_prime_u64(uint64_t n);

}  // namespace fhe_b200
