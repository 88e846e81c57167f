// Test-side harness around the reference library (compiled from its own sources by
// oracle/Makefile into oracle/_ref/). It exposes a flat C interface over the
// reference's CKKSEngine/CKKSCore so that Python tests and the benchmark's CPU arm
// can feed both implementations the same limbs, keys and seeded randomness.
//
// This file is checker infrastructure only: nothing in the product links it.
// Private members of the reference classes (core_, rng_, allocate_*) are reached with
// the `private -> public` macro trick, confined to this translation unit.

#include <algorithm>
#include <chrono>
#include <complex>
#include <iterator>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <random>
#include <string>
#include <tuple>
#include <vector>

#define private public
#define protected public
#include "arithmetic/prime.h"
#include "ckks/core.h"
#include "ckks/engine.h"
#include "random/gaussian_sampler.h"
#include "operation/ntt.h"
#include "montgomery/unit.h"
#undef private
#undef protected

using namespace desilo::fhe;

namespace {

struct Handle {
  // kind: 1 secret key, 2 public key, 3 relinearization key, 4 unit ciphertext,
  // 5 unit plaintext, 6 fixed rotation key, 7 conjugation key
  int kind = 0;
  Data *data = nullptr;  // the Data carrying limbs (for keys: the key switching key)
  void *owner = nullptr; // the object to delete
};

struct RefEngine {
  std::unique_ptr<CKKSEngine> engine;
  CKKSCore *core() { return engine->core_.get(); }
};

CKKSConfig make_config(int log_n, int log_slot, int special_prime_count,
                       int max_level, int preset, int threads) {
  CKKSConfig config;
  config.log_coeff_count_ = log_n;
  config.log_slot_count_ = log_slot;
  config.special_prime_count_ = special_prime_count;
  config.max_level_ = max_level;
  config.scheme_preset_ = static_cast<SchemePreset>(preset);
  if (threads > 1) {
    config.processor_ = EngineProcessor::CPU_PARALLEL;
    config.thread_count_ = threads;
  }
  return config;
}

template <class T>
T *make_text(CKKSCore *core, int flag, int moduli_id, int polynomial_count,
             long double scale, const int64_t *data) {
  auto text = core->allocate_text<T>(static_cast<DataFlag>(flag), moduli_id,
                                     polynomial_count, scale);
  const int chains = text->chain_count_;
  const int n = core->get_coeff_count();
  for (int p = 0; p < polynomial_count; p++) {
    auto poly = text->get_polynomial(p);
    for (int c = 0; c < chains; c++) {
      std::memcpy(poly->get(c), data + (size_t(p) * chains + c) * n,
                  sizeof(int64_t) * n);
    }
  }
  return text;
}

void dump(Data *data, int64_t *out, int n) {
  const int chains = data->chain_count_;
  const int polys = data->polynomial_count();
  for (int p = 0; p < polys; p++) {
    auto poly = data->get_polynomial(p);
    for (int c = 0; c < chains; c++) {
      std::memcpy(out + (size_t(p) * chains + c) * n, poly->get(c),
                  sizeof(int64_t) * n);
    }
  }
}

thread_local std::string g_ref_error;

// Called inside a catch-all handler: records the message of the exception in flight.
void remember_error() {
  try {
    throw;
  } catch (const std::exception &ex) {
    g_ref_error = ex.what();
  } catch (...) {
    g_ref_error = "unknown exception";
  }
}

Handle *wrap(int kind, Data *data, void *owner) {
  auto h = new Handle();
  h->kind = kind;
  h->data = data;
  h->owner = owner;
  return h;
}

} // namespace

extern "C" {

const char *ref_last_error() { return g_ref_error.c_str(); }

// The discrete-Gaussian CDT tree (sigma 3.2, 128 bits) the sampler walks.
int ref_cdt_tree(uint64_t *out, int capacity) {
  GaussianSamplingTree tree;
  for (int i = 0; i < tree.data_size_ && i < capacity; i++) out[i] = tree.data_[i];
  return tree.data_size_;
}

// The double deviations of the precomputed tables, indexed by level.
int ref_deviations(void *e, double *out, int capacity) {
  auto core = static_cast<RefEngine *>(e)->core();
  const auto &d = core->precomputed_.deviation_;
  const int count = static_cast<int>(d.size());
  for (int i = 0; i < count && i < capacity; i++) out[i] = d[i];
  return count;
}

int ref_cached_primes(int kind, int coeff_count, uint64_t *out, int capacity) {
  std::tuple<uint64_t *, int> cached;
  if (kind == 0) {
    cached = get_cached_small_primes(coeff_count);
  } else if (kind == 1) {
    cached = get_cached_bootstrap_primes(coeff_count);
  } else {
    cached = get_cached_large_primes(coeff_count);
  }
  auto [ptr, count] = cached;
  for (int i = 0; i < count && i < capacity; i++) {
    out[i] = ptr[i];
  }
  return count;
}

void ref_ntt_raw(int64_t *x, int64_t *y, const int64_t *root, uint64_t q,
                 uint64_t k, int coeff_count, int log_coeff_count) {
  ntt(x, y, root, q << 1, q, k, coeff_count, log_coeff_count);
}

void ref_intt_raw(int64_t *x, int64_t *y, const int64_t *root_inverse,
                  uint64_t q, uint64_t k, int coeff_count,
                  int log_coeff_count) {
  intt(x, y, root_inverse, q << 1, q, k, coeff_count, log_coeff_count);
}

void *ref_engine_new(int log_n, int log_slot, int special_prime_count,
                     int max_level, int preset, int threads) {
  try {
    auto config = make_config(log_n, log_slot, special_prime_count, max_level,
                              preset, threads);
    config.validate();
    auto e = new RefEngine();
    e->engine = std::make_unique<CKKSEngine>(config);
    return e;
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void ref_engine_free(void *e) { delete static_cast<RefEngine *>(e); }

void ref_engine_seed(void *e, const uint32_t *seed, const uint8_t *nonce) {
  auto core = static_cast<RefEngine *>(e)->core();
  const int n = core->get_coeff_count();
  core->rng_.~RandomNumberGenerator();
  new (&core->rng_) RandomNumberGenerator(1, n, seed, nonce);
}

// out: [N, chain_count, prime_count, full_level, max_level, max_ks_level,
//       slot_count, special_prime_count, scale_bits, one_more_level]
void ref_engine_info(void *e, int *out) {
  auto core = static_cast<RefEngine *>(e)->core();
  const auto &p = core->parameters_;
  out[0] = p.get_coeff_count();
  out[1] = p.get_chain_count();
  out[2] = p.get_prime_count();
  out[3] = p.get_full_level();
  out[4] = p.get_max_level();
  out[5] = p.get_max_key_switching_level();
  out[6] = p.get_slot_count();
  out[7] = p.get_special_prime_count();
  out[8] = p.get_scale_bit_length();
  out[9] = p.get_use_one_more_level() ? 1 : 0;
}

int ref_moduli_id(void *e, int level) {
  return static_cast<RefEngine *>(e)->core()->parameters_.get_moduli_id(level);
}

int ref_chain_count(void *e, int moduli_id, int include_special) {
  return static_cast<RefEngine *>(e)->core()->parameters_.get_chain_count(
      moduli_id, include_special != 0);
}

int ref_partition_count(void *e, int moduli_id, int key_moduli_id) {
  auto core = static_cast<RefEngine *>(e)->core();
  return static_cast<int>(core->get_partitions(moduli_id, key_moduli_id).size());
}

// All primes (the full chain with specials) and their per-prime tables.
int ref_tables(void *e, uint64_t *q, uint64_t *k, int64_t *r_squared,
               int64_t *n_inverse, int64_t *root, int64_t *root_inverse) {
  auto core = static_cast<RefEngine *>(e)->core();
  const auto &pre = core->precomputed_;
  const int primes = pre.prime_count_;
  const int n = pre.coeff_count_;
  for (int i = 0; i < primes; i++) {
    if (q) q[i] = pre.q_[i];
    if (k) k[i] = pre.k_[i];
    if (r_squared) r_squared[i] = pre.r_squared_[i];
    if (n_inverse) n_inverse[i] = pre.coeff_count_inverse_[i];
  }
  if (root) std::memcpy(root, pre.root_.data(), sizeof(int64_t) * primes * (n - 1));
  if (root_inverse)
    std::memcpy(root_inverse, pre.root_inverse_.data(),
                sizeof(int64_t) * primes * (n - 1));
  return primes;
}

// p_product_mult_r (chain_count entries), p_inverse_mult_r flattened
// [special][q_index < p_index], rescale_scale flattened [from][to>from].
void ref_key_switch_tables(void *e, int64_t *p_product_mult_r,
                           int64_t *p_inverse_mult_r, int64_t *rescale_scale) {
  auto core = static_cast<RefEngine *>(e)->core();
  const auto &pre = core->precomputed_;
  if (p_product_mult_r)
    std::copy(pre.p_product_mult_r_.begin(), pre.p_product_mult_r_.end(),
              p_product_mult_r);
  if (p_inverse_mult_r) {
    size_t o = 0;
    for (auto &v : pre.p_inverse_mult_r_)
      for (auto x : v) p_inverse_mult_r[o++] = x;
  }
  if (rescale_scale) {
    size_t o = 0;
    for (auto &v : pre.rescale_scale_)
      for (auto x : v) rescale_scale[o++] = x;
  }
}

// ---- data handles -------------------------------------------------------------

void *ref_text_new(void *e, int kind, int flag, int moduli_id, int polys,
                   long double scale, const int64_t *data) {
  auto core = static_cast<RefEngine *>(e)->core();
  if (kind == 4) {
    auto t = make_text<UnitCiphertext>(core, flag, moduli_id, polys, scale, data);
    return wrap(4, t, t);
  }
  auto t = make_text<UnitPlaintext>(core, flag, moduli_id, polys, scale, data);
  return wrap(5, t, t);
}

// A relinearization key (kind 3) or a bare key switching key for switch_key
// (kind 8) from limbs laid out [2*dnum][prime_count][N].
void *ref_key_new(void *e, int kind, int moduli_id, int polys,
                  const int64_t *data) {
  auto core = static_cast<RefEngine *>(e)->core();
  auto key = core->allocate_data<KeySwitchingKey>(
      DataFlag::NTT_FORM | DataFlag::INCLUDE_SPECIAL, moduli_id, polys);
  const int chains = key->chain_count_;
  const int n = core->get_coeff_count();
  for (int p = 0; p < polys; p++)
    for (int c = 0; c < chains; c++)
      std::memcpy(key->get_polynomial(p)->get(c),
                  data + (size_t(p) * chains + c) * n, sizeof(int64_t) * n);
  if (kind == 3) {
    auto rk = new RelinearizationKey(key);
    return wrap(3, key, rk);
  }
  return wrap(8, key, key);
}

// A fixed rotation key (kind 6, step delta) or a conjugation key (kind 7) from
// key switching key limbs; permutations as CKKSCore::rotate(key, ...) makes them
// (core_key.cpp:209-236).
void *ref_rotation_key_new(void *e, int kind, int moduli_id, int polys, int delta,
                           const int64_t *data) {
  auto core = static_cast<RefEngine *>(e)->core();
  auto key = core->allocate_data<KeySwitchingKey>(
      DataFlag::NTT_FORM | DataFlag::INCLUDE_SPECIAL, moduli_id, polys);
  const int chains = key->chain_count_;
  const int n = core->get_coeff_count();
  for (int p = 0; p < polys; p++)
    for (int c = 0; c < chains; c++)
      std::memcpy(key->get_polynomial(p)->get(c),
                  data + (size_t(p) * chains + c) * n, sizeof(int64_t) * n);
  auto [perm, sign] = core->precomputed_.make_permutation_parameters(kind == 7 ? -1 : delta);
  if (kind == 7) {
    auto ck = new ConjugationKey(key, perm, sign);
    return wrap(7, key, ck);
  }
  auto fk = new FixedRotationKey(key, perm, sign, delta);
  return wrap(6, key, fk);
}

void ref_handle_free(void *h) {
  auto handle = static_cast<Handle *>(h);
  switch (handle->kind) {
  case 3: delete static_cast<RelinearizationKey *>(handle->owner); break;
  case 6: delete static_cast<FixedRotationKey *>(handle->owner); break;
  case 7: delete static_cast<ConjugationKey *>(handle->owner); break;
  case 9: delete static_cast<RotationKey *>(handle->owner); break;
  case 10: delete static_cast<SmallBootstrapKey *>(handle->owner); break;
  case 12: delete static_cast<BootstrapKey *>(handle->owner); break;
  case 11: break;  // a view into another handle's key
  default: delete static_cast<Data *>(handle->owner); break;
  }
  delete handle;
}

// info: [kind, flag, moduli_id, level, polys, chain_count]; returns scale
long double ref_handle_info(void *h, int *info) {
  auto handle = static_cast<Handle *>(h);
  auto d = handle->data;
  info[0] = handle->kind;
  info[1] = static_cast<int>(d->flag_);
  info[2] = d->moduli_id_;
  info[3] = d->level_;
  info[4] = d->polynomial_count();
  info[5] = d->chain_count_;
  if (handle->kind == 4) return static_cast<UnitCiphertext *>(d)->ckks_scale_;
  if (handle->kind == 5) return static_cast<UnitPlaintext *>(d)->ckks_scale_;
  return 0;
}

void ref_handle_dump(void *e, void *h, int64_t *out) {
  auto core = static_cast<RefEngine *>(e)->core();
  dump(static_cast<Handle *>(h)->data, out, core->get_coeff_count());
}

// ---- keys (seeded through ref_engine_seed) ------------------------------------

void *ref_create_secret_key(void *e, int level) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto sk = level < 0 ? eng->create_secret_key() : eng->create_secret_key(level);
  return wrap(1, sk, sk);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_create_secret_key_from(void *e, const int64_t *secret, int level) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  std::vector<int64_t> s(secret, secret + eng->get_coeff_count());
  auto sk = level < 0 ? eng->create_secret_key(s) : eng->create_secret_key(s, level);
  return wrap(1, sk, sk);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_create_public_key(void *e, void *sk, int level) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto s = static_cast<SecretKey *>(static_cast<Handle *>(sk)->data);
  auto pk = level < 0 ? eng->create_public_key(s) : eng->create_public_key(s, level);
  return wrap(2, pk, pk);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_create_relinearization_key(void *e, void *sk, int level) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto s = static_cast<SecretKey *>(static_cast<Handle *>(sk)->data);
  auto rk = level < 0 ? eng->create_relinearization_key(s)
                      : eng->create_relinearization_key(s, level);
  return wrap(3, rk->key_switching_key_, rk);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_create_fixed_rotation_key(void *e, void *sk, int delta, int level) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto s = static_cast<SecretKey *>(static_cast<Handle *>(sk)->data);
  auto fk = level < 0 ? eng->create_fixed_rotation_key(s, delta)
                      : eng->create_fixed_rotation_key(s, delta, level);
  return wrap(6, fk->key_switching_key_, fk);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_create_conjugation_key(void *e, void *sk, int level) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto s = static_cast<SecretKey *>(static_cast<Handle *>(sk)->data);
  auto ck = level < 0 ? eng->create_conjugation_key(s)
                      : eng->create_conjugation_key(s, level);
  return wrap(7, ck->key_switching_key_, ck);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

// ---- core-level ops on handles --------------------------------------------------

void *ref_core_to_ntt(void *e, void *h) {
  try {
  auto core = static_cast<RefEngine *>(e)->core();
  auto r = core->to_ntt_form(static_cast<UnitCiphertext *>(static_cast<Handle *>(h)->data));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_core_to_intt(void *e, void *h) {
  try {
  auto core = static_cast<RefEngine *>(e)->core();
  auto r = core->to_intt_form(static_cast<UnitCiphertext *>(static_cast<Handle *>(h)->data));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_core_tensor(void *e, void *a, void *b) {
  try {
  auto core = static_cast<RefEngine *>(e)->core();
  auto r = core->multiply(static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data),
                          static_cast<UnitCiphertext *>(static_cast<Handle *>(b)->data));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_core_relinearize(void *e, void *ct, void *rk) {
  try {
  auto core = static_cast<RefEngine *>(e)->core();
  auto r = core->relinearize(
      static_cast<UnitCiphertext *>(static_cast<Handle *>(ct)->data),
      static_cast<RelinearizationKey *>(static_cast<Handle *>(rk)->owner));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_core_rescale(void *e, void *ct) {
  try {
  auto core = static_cast<RefEngine *>(e)->core();
  auto r = core->rescale(static_cast<UnitCiphertext *>(static_cast<Handle *>(ct)->data));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_core_switch_key(void *e, void *ct, void *ksk) {
  try {
  auto core = static_cast<RefEngine *>(e)->core();
  auto r = core->switch_key(
      static_cast<UnitCiphertext *>(static_cast<Handle *>(ct)->data),
      static_cast<KeySwitchingKey *>(static_cast<Handle *>(ksk)->data));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

// ---- engine-level ops ----------------------------------------------------------

void *ref_engine_multiply(void *e, void *a, void *b, void *rk) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto x = static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data);
  auto y = static_cast<UnitCiphertext *>(static_cast<Handle *>(b)->data);
  UnitCiphertext *r;
  if (rk) {
    r = eng->multiply(x, y,
                      static_cast<RelinearizationKey *>(static_cast<Handle *>(rk)->owner));
  } else {
    r = eng->multiply(x, y);
  }
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_relinearize(void *e, void *a, void *rk) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto r = eng->relinearize(
      static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data),
      static_cast<RelinearizationKey *>(static_cast<Handle *>(rk)->owner));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_rescale(void *e, void *a) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto r = eng->rescale(static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_core_rotate(void *e, void *a, void *fk) {
  try {
    auto core = static_cast<RefEngine *>(e)->core();
    auto r = core->rotate(static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data),
                          static_cast<FixedRotationKey *>(static_cast<Handle *>(fk)->owner));
    return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_core_conjugate(void *e, void *a, void *ck) {
  try {
    auto core = static_cast<RefEngine *>(e)->core();
    auto r = core->conjugate(static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data),
                             static_cast<ConjugationKey *>(static_cast<Handle *>(ck)->owner));
    return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_rotate(void *e, void *a, void *fk) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto r = eng->rotate(static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data),
                       static_cast<FixedRotationKey *>(static_cast<Handle *>(fk)->owner));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_conjugate(void *e, void *a, void *ck) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto r = eng->conjugate(static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data),
                          static_cast<ConjugationKey *>(static_cast<Handle *>(ck)->owner));
  return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_level_down(void *e, void *a, int level) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto h = static_cast<Handle *>(a);
    if (h->kind == 5) {
      auto r = eng->level_down(static_cast<UnitPlaintext *>(h->data), level);
      return wrap(5, r, r);
    }
    auto r = eng->level_down(static_cast<UnitCiphertext *>(h->data), level);
    return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_rotate_plain(void *e, void *a, int delta) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto r = eng->rotate(static_cast<UnitPlaintext *>(static_cast<Handle *>(a)->data), delta);
    return wrap(5, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_conjugate_plain(void *e, void *a) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto r = eng->conjugate(static_cast<UnitPlaintext *>(static_cast<Handle *>(a)->data));
    return wrap(5, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

// CKKSEngine::rotate(UnitCiphertext*, RotationKey*, delta, normalize_by_slot_count)
// with a RotationKey that borrows the given fixed rotation keys.
void *ref_engine_rotate_keys(void *e, void *a, void **fks, int count, int delta,
                             int by_slot_count) {
  std::vector<FixedRotationKey *> keys;
  for (int i = 0; i < count; i++)
    keys.push_back(static_cast<FixedRotationKey *>(static_cast<Handle *>(fks[i])->owner));
  RotationKey *rk = nullptr;
  void *out = nullptr;
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    rk = new RotationKey(keys);
    auto r = eng->rotate(static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data), rk, delta,
                         by_slot_count != 0);
    out = wrap(4, r, r);
  } catch (...) {
    remember_error();
    out = nullptr;
  }
  if (rk) {
    rk->fixed_rotation_keys_.clear();
    delete rk;
  }
  return out;
}

// Engine arithmetic (engine_add.cpp, engine_subtract.cpp, engine_multiply.cpp,
// engine_negate.cpp).  op: 0 add, 1 subtract, 2 add plaintext, 3 subtract plaintext,
// 4 plaintext minus ciphertext, 5 multiply plaintext, 6 negate, 7 square, 8 square and
// relinearize (b = key); scalar ops: 0 add, 1 subtract, 2 multiply.
void *ref_engine_arith(void *e, int op, void *a, void *b) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto ct = [](void *h) { return static_cast<UnitCiphertext *>(static_cast<Handle *>(h)->data); };
    auto pt = [](void *h) { return static_cast<UnitPlaintext *>(static_cast<Handle *>(h)->data); };
    UnitCiphertext *r = nullptr;
    switch (op) {
      case 0: r = eng->add(ct(a), ct(b)); break;
      case 1: r = eng->subtract(ct(a), ct(b)); break;
      case 2: r = eng->add(ct(a), pt(b)); break;
      case 3: r = eng->subtract(ct(a), pt(b)); break;
      case 4: r = eng->subtract(pt(b), ct(a)); break;
      case 5: r = eng->multiply(ct(a), pt(b)); break;
      case 6: r = eng->negate(ct(a)); break;
      case 7: r = eng->square(ct(a)); break;
      case 8:
        r = eng->square(ct(a), static_cast<RelinearizationKey *>(static_cast<Handle *>(b)->owner));
        break;
      default: return nullptr;
    }
    return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_scalar(void *e, int op, void *a, double value, long long integer) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto c = static_cast<UnitCiphertext *>(static_cast<Handle *>(a)->data);
    UnitCiphertext *r = nullptr;
    switch (op) {
      case 0: r = eng->add(c, value); break;
      case 1: r = eng->subtract(c, value); break;
      case 2: r = eng->multiply(c, value); break;
      case 3: r = eng->multiply(c, static_cast<int64_t>(integer)); break;
      default: return nullptr;
    }
    return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

// ---- bootstrapping --------------------------------------------------------------

// create_rotation_key(sk[, level]): kind 9 owns the RotationKey; its fixed keys are
// reached with ref_rotation_key_get.
void *ref_create_rotation_key(void *e, void *sk, int level) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto s = static_cast<SecretKey *>(static_cast<Handle *>(sk)->data);
    auto rk = level < 0 ? eng->create_rotation_key(s) : eng->create_rotation_key(s, level);
    return wrap(9, nullptr, rk);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

int ref_rotation_key_count(void *h) {
  return static_cast<int>(
      static_cast<RotationKey *>(static_cast<Handle *>(h)->owner)->fixed_rotation_keys_.size());
}

// A non-owning view (kind 11) of fixed key i: its key switching key limbs and delta.
void *ref_rotation_key_get(void *h, int i, int *delta) {
  auto rk = static_cast<RotationKey *>(static_cast<Handle *>(h)->owner);
  auto fk = rk->fixed_rotation_keys_[i];
  *delta = fk->delta_;
  return wrap(11, fk->key_switching_key_, nullptr);
}

// create_small_bootstrap_key(sk): kind 10; part 0 = to_sparse, 1 = to_dense (views).
void *ref_create_small_bootstrap_key(void *e, void *sk) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto s = static_cast<SecretKey *>(static_cast<Handle *>(sk)->data);
    return wrap(10, nullptr, eng->create_small_bootstrap_key(s));
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_small_bootstrap_key_part(void *h, int part) {
  auto k = static_cast<SmallBootstrapKey *>(static_cast<Handle *>(h)->owner);
  return wrap(11, part == 0 ? k->to_sparse_ : k->to_dense_, nullptr);
}

void *ref_engine_bootstrap(void *e, void *ct, void *rk, void *ck, void *rotk, void *sbk,
                           int stage_count) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto r = eng->bootstrap(
        static_cast<UnitCiphertext *>(static_cast<Handle *>(ct)->data),
        static_cast<RelinearizationKey *>(static_cast<Handle *>(rk)->owner),
        static_cast<ConjugationKey *>(static_cast<Handle *>(ck)->owner),
        static_cast<RotationKey *>(static_cast<Handle *>(rotk)->owner),
        static_cast<SmallBootstrapKey *>(static_cast<Handle *>(sbk)->owner), stage_count);
    return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

// create_bootstrap_key(sk, stage_count, size): kind 12 owns the BootstrapKey.
void *ref_create_bootstrap_key(void *e, void *sk, int stage_count, const char *size) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto s = static_cast<SecretKey *>(static_cast<Handle *>(sk)->data);
    return wrap(12, nullptr, eng->create_bootstrap_key(s, stage_count, size));
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

int ref_bootstrap_key_delta_count(void *h) {
  auto bk = static_cast<BootstrapKey *>(static_cast<Handle *>(h)->owner);
  return static_cast<int>(bk->rotation_contexts_.size());
}

// Rotation context i in ascending delta order: a view of its key switching key.
void *ref_bootstrap_key_get(void *h, int i, int *delta) {
  auto bk = static_cast<BootstrapKey *>(static_cast<Handle *>(h)->owner);
  auto it = bk->rotation_contexts_.begin();
  std::advance(it, i);
  *delta = it->first;
  return wrap(11, it->second.first->key_switching_key_, nullptr);
}

// shape: [level, inner loop count, outer loop count, process order entries].
int ref_bootstrap_key_stage(void *h, int to_slot, int stage, int *shape) {
  auto bk = static_cast<BootstrapKey *>(static_cast<Handle *>(h)->owner);
  auto &stages = to_slot ? bk->coeff_to_slot_stages_ : bk->slot_to_coeff_stages_;
  if (stage < 0 || stage >= static_cast<int>(stages.size())) return -1;
  auto m = stages[stage];
  shape[0] = m->level_;
  shape[1] = m->inner_loop_count_;
  shape[2] = m->outer_loop_count_;
  shape[3] = static_cast<int>(m->outer_loop_process_order_.size());
  return 0;
}

// A view of diagonal (outer, inner) of a stage, or null when the stage has none.
void *ref_bootstrap_key_diagonal(void *h, int to_slot, int stage, int outer, int inner) {
  auto bk = static_cast<BootstrapKey *>(static_cast<Handle *>(h)->owner);
  auto &stages = to_slot ? bk->coeff_to_slot_stages_ : bk->slot_to_coeff_stages_;
  auto &diagonals = stages[stage]->encoded_diagonals_;
  auto o = diagonals.find(outer);
  if (o == diagonals.end()) return nullptr;
  auto i = o->second.find(inner);
  if (i == o->second.end()) return nullptr;
  return wrap(11, i->second, nullptr);
}

void *ref_bootstrap_key_small(void *h, int part) {
  auto bk = static_cast<BootstrapKey *>(static_cast<Handle *>(h)->owner);
  auto k = bk->small_bootstrap_key_;
  return wrap(11, part == 0 ? k->to_sparse_ : k->to_dense_, nullptr);
}

void *ref_engine_bootstrap_with_key(void *e, void *ct, void *rk, void *ck, void *bk) {
  try {
    auto eng = static_cast<RefEngine *>(e)->engine.get();
    auto r = eng->bootstrap(
        static_cast<UnitCiphertext *>(static_cast<Handle *>(ct)->data),
        static_cast<RelinearizationKey *>(static_cast<Handle *>(rk)->owner),
        static_cast<ConjugationKey *>(static_cast<Handle *>(ck)->owner),
        static_cast<BootstrapKey *>(static_cast<Handle *>(bk)->owner));
    return wrap(4, r, r);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_encode(void *e, const double *re, const double *im, int count,
                        int level) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  if (im == nullptr) {  // encode_unit(std::vector<double>&)
    std::vector<double> v(re, re + count);
    auto pt = level < 0 ? eng->encode_unit(v) : eng->encode_unit(v, level);
    return wrap(5, pt, pt);
  }
  std::vector<std::complex<double>> v(count);
  for (int i = 0; i < count; i++) v[i] = {re[i], im[i]};
  auto pt = level < 0 ? eng->encode_unit(v) : eng->encode_unit(v, level);
  return wrap(5, pt, pt);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

int ref_engine_decode_real(void *e, void *pt, double *re) {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto v = eng->decode_unit(static_cast<UnitPlaintext *>(static_cast<Handle *>(pt)->data));
  for (size_t i = 0; i < v.size(); i++) re[i] = v[i];
  return static_cast<int>(v.size());
}

int ref_engine_decode(void *e, void *pt, double *re, double *im) {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto v = eng->decode_complex_unit_plaintext(
      static_cast<UnitPlaintext *>(static_cast<Handle *>(pt)->data));
  for (size_t i = 0; i < v.size(); i++) {
    re[i] = v[i].real();
    im[i] = v[i].imag();
  }
  return static_cast<int>(v.size());
}

void *ref_engine_encrypt(void *e, void *pt, void *key) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto p = static_cast<UnitPlaintext *>(static_cast<Handle *>(pt)->data);
  auto k = static_cast<Handle *>(key);
  UnitCiphertext *ct;
  if (k->kind == 1) {
    ct = eng->encrypt_unit(p, static_cast<SecretKey *>(k->data));
  } else {
    ct = eng->encrypt_unit(p, static_cast<PublicKey *>(k->data));
  }
  return wrap(4, ct, ct);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

void *ref_engine_decrypt(void *e, void *ct, void *sk) {
  try {
  auto eng = static_cast<RefEngine *>(e)->engine.get();
  auto pt = eng->decrypt_to_unit_plaintext(
      static_cast<UnitCiphertext *>(static_cast<Handle *>(ct)->data),
      static_cast<SecretKey *>(static_cast<Handle *>(sk)->data));
  return wrap(5, pt, pt);
  } catch (...) {
    remember_error();
    return nullptr;
  }
}

// ---- CPU timing arm ------------------------------------------------------------
// Times engine.multiply(ct_a, ct_b, rk) followed by engine.rescale on fresh
// ciphertexts encrypted at `level`; keygen and encryption are outside the timing.
// Writes one duration per timed step (milliseconds) and returns the median.
double ref_bench_mult_relin_rescale(int log_n, int special_prime_count, int level,
                                    int threads, int warmup, int steps,
                                    double *step_ms) {
  auto config = make_config(log_n, -1, special_prime_count, -1, 1, threads);
  CKKSEngine engine(config);
  if (level < 0) level = engine.core_->parameters_.get_max_key_switching_level();
  auto sk = engine.create_secret_key();
  auto pk = engine.create_public_key(sk, level);
  auto rk = engine.create_relinearization_key(sk, level);
  const int slots = engine.get_slot_count();
  std::mt19937_64 gen(1);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  std::vector<std::complex<double>> a(slots), b(slots);
  for (auto &z : a) z = {u(gen), u(gen)};
  for (auto &z : b) z = {u(gen), u(gen)};
  auto ca = engine.encrypt_unit(a, pk, level);
  auto cb = engine.encrypt_unit(b, pk, level);
  std::vector<double> times;
  for (int i = 0; i < warmup + steps; i++) {
    auto t0 = std::chrono::steady_clock::now();
    auto m = engine.multiply(ca, cb, rk);
    auto r = engine.rescale(m);
    auto t1 = std::chrono::steady_clock::now();
    delete m;
    delete r;
    if (i >= warmup) {
      times.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
    }
  }
  for (size_t i = 0; i < times.size(); i++) step_ms[i] = times[i];
  delete ca;
  delete cb;
  delete rk;
  delete pk;
  delete sk;
  if (times.empty()) return 0;
  std::sort(times.begin(), times.end());
  return times[times.size() / 2];
}

// Times one engine.bootstrap(ct, rk, ck, rotation key, small bootstrap key, 3) on the
// bootstrap preset at N = 2^16 (keys and encryption outside the timing); returns ms.
double ref_bench_bootstrap(int threads) {
  auto config = make_config(16, -1, 4, -1, 2, threads);
  CKKSEngine engine(config);
  auto sk = engine.create_secret_key();
  auto rk = engine.create_relinearization_key(sk);
  auto ck = engine.create_conjugation_key(sk);
  auto rot = engine.create_rotation_key(sk);
  auto sbk = engine.create_small_bootstrap_key(sk);
  const int slots = engine.get_slot_count();
  std::mt19937_64 gen(1);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  std::vector<std::complex<double>> v(slots);
  for (auto &z : v) z = {u(gen), u(gen)};
  auto pt = engine.encode_unit(v, 3);
  auto ct = engine.encrypt_unit(v, sk, 3);
  auto t0 = std::chrono::steady_clock::now();
  auto out = engine.bootstrap(ct, rk, ck, rot, sbk, 3);
  auto t1 = std::chrono::steady_clock::now();
  delete out;
  delete ct;
  delete pt;
  delete sbk;
  delete rot;
  delete ck;
  delete rk;
  delete sk;
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// Times one engine.bootstrap(ct, rk, ck, bootstrap key) with a "medium" bootstrap key
// of 3 stages on the same workload; returns ms (key generation outside the timing).
double ref_bench_bootstrap_with_key(int threads) {
  auto config = make_config(16, -1, 4, -1, 2, threads);
  CKKSEngine engine(config);
  auto sk = engine.create_secret_key();
  auto rk = engine.create_relinearization_key(sk);
  auto ck = engine.create_conjugation_key(sk);
  auto bk = engine.create_bootstrap_key(sk, 3, "medium");
  const int slots = engine.get_slot_count();
  std::mt19937_64 gen(1);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  std::vector<std::complex<double>> v(slots);
  for (auto &z : v) z = {u(gen), u(gen)};
  auto ct = engine.encrypt_unit(v, sk, 3);
  auto t0 = std::chrono::steady_clock::now();
  auto out = engine.bootstrap(ct, rk, ck, bk);
  auto t1 = std::chrono::steady_clock::now();
  delete out;
  delete ct;
  delete bk;
  delete ck;
  delete rk;
  delete sk;
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

} // extern "C"
