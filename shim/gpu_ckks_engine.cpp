// GpuCKKSEngine: the reference's engine interface (desilo::fhe::AbstractEngine,
// src/engine/abstract_engine.h:12-299) implemented over the fhe_b200 C ABI, so
// programs written against the reference (examples/encrypt_decrypt.cpp,
// examples/multiply_vector.cpp) run on the B200 engine unchanged: link this file
// instead of the reference's src/engine/engine.cpp, which defines the same two
// factories (create_default_engine, create_ckks_engine; engine.cpp:7-20).
//
// Objects stay the reference's own host objects (SecretKey, Ciphertext = LongText of
// UnitCiphertext, ...), with the reference's limb words, so they move freely between
// this engine and the reference's CKKSEngine.  Each call uploads the limbs of its
// operands to the device, runs the operation there and downloads the result into a
// new object the caller owns and deletes, as with the reference.  Long texts (more
// values than slots) are processed unit by unit, as the reference does.
//
// Errors: the C ABI's statuses become the reference's exceptions
// (FHE_ERR_INVALID_ARGUMENT -> std::invalid_argument, the rest ->
// std::runtime_error) carrying its "<Function Name>: <reason>" message.  Members
// outside the accelerated path (matrix products, sums, the polynomial evaluation
// API, power bases, stacking, mod_raise, multiply_imaginary and the BootstrapKey
// form of bootstrapping, whose multi-GB key lives on the device behind the C ABI's
// fhe_bootstrap_key instead of in a host object) throw std::invalid_argument saying
// so.
#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "ckks/config.h"
#include "ckks/encode.h"
#include "engine/engine.h"
#include "fhe_b200.h"

namespace desilo::fhe {
namespace {

void check(int rc) {
  if (rc == FHE_OK) return;
  const std::string message = fhe_last_error();
  if (rc == FHE_ERR_INVALID_ARGUMENT) throw std::invalid_argument(message);
  throw std::runtime_error(message);
}

[[noreturn]] void not_provided(const char *function_name) {
  throw std::invalid_argument(std::string(function_name) +
                              ": not provided by the B200 engine (outside its accelerated path).");
}

// One fhe_data handle, destroyed with the wrapper.
class Handle {
 public:
  Handle() = default;
  Handle(const Handle &) = delete;
  Handle &operator=(const Handle &) = delete;
  Handle(Handle &&o) noexcept : p_(o.p_) { o.p_ = nullptr; }
  ~Handle() { reset(); }
  void reset() {
    if (p_) fhe_data_destroy(p_);
    p_ = nullptr;
  }
  fhe_data *get() const { return p_; }
  fhe_data **out() {
    reset();
    return &p_;
  }

 private:
  fhe_data *p_ = nullptr;
};

int preset_id(SchemePreset p) { return static_cast<int>(p); }

}  // namespace

class GpuCKKSEngine : public AbstractEngine {
 public:
  explicit GpuCKKSEngine(const CKKSConfig &config) : preset_(config.scheme_preset_) {
    fhe_config c;
    fhe_config_default(&c);
    c.log_coeff_count = config.log_coeff_count_;
    c.log_slot_count = config.log_slot_count_;
    c.special_prime_count = config.special_prime_count_;
    c.max_level = config.max_level_;
    c.scheme_preset = preset_id(config.scheme_preset_);
    check(fhe_engine_create(&c, &e_));
    check(fhe_engine_info_get(e_, &info_));
    log_coeff_ = static_cast<uint8_t>(config.log_coeff_count_);
    int log_slot = 0;
    while ((1 << log_slot) < info_.slot_count) log_slot++;
    log_slot_ = static_cast<uint8_t>(log_slot);
  }
  ~GpuCKKSEngine() override { fhe_engine_destroy(e_); }

  // ------------------------------------------------------------------ keys --

  SecretKey *create_secret_key() override { return create_secret_key(-1); }
  SecretKey *create_secret_key(int level) override {
    Handle h;
    check(fhe_create_secret_key(e_, level, h.out()));
    return fetch_data<SecretKey>(h.get());
  }
  SecretKey *create_secret_key(std::vector<int64_t> &secret) override {
    return create_secret_key(secret, -1);
  }
  SecretKey *create_secret_key(std::vector<int64_t> &secret, int level) override {
    Handle h;
    check(fhe_create_secret_key_from(e_, secret.data(), static_cast<int>(secret.size()), level,
                                     h.out()));
    return fetch_data<SecretKey>(h.get());
  }
  PublicKey *create_public_key(SecretKey *secret_key) override {
    return create_public_key(secret_key, -1);
  }
  PublicKey *create_public_key(SecretKey *secret_key, int level) override {
    Handle sk = upload(secret_key, FHE_SECRET_KEY), h;
    check(fhe_create_public_key(e_, sk.get(), level, h.out()));
    return fetch_data<PublicKey>(h.get());
  }
  ConjugationKey *create_conjugation_key(SecretKey *secret_key) override {
    return create_conjugation_key(secret_key, -1);
  }
  ConjugationKey *create_conjugation_key(SecretKey *secret_key, int level) override {
    Handle sk = upload(secret_key, FHE_SECRET_KEY), h;
    check(fhe_create_conjugation_key(e_, sk.get(), level, h.out()));
    auto [permutation, sign] = permutation_parameters(-1);
    return new ConjugationKey(fetch_data<KeySwitchingKey>(h.get()), permutation, sign);
  }
  RelinearizationKey *create_relinearization_key(SecretKey *secret_key) override {
    return create_relinearization_key(secret_key, -1);
  }
  RelinearizationKey *create_relinearization_key(SecretKey *secret_key, int level) override {
    Handle sk = upload(secret_key, FHE_SECRET_KEY), h;
    check(fhe_create_relinearization_key(e_, sk.get(), level, h.out()));
    return new RelinearizationKey(fetch_data<KeySwitchingKey>(h.get()));
  }
  FixedRotationKey *create_fixed_rotation_key(SecretKey *secret_key, int delta) override {
    return create_fixed_rotation_key(secret_key, delta, -1);
  }
  // The reference's CKKSEngine reads this overload's two ints as (delta, level)
  // (ckks/engine.cpp:114-118), whatever the interface names them; so does this one.
  FixedRotationKey *create_fixed_rotation_key(SecretKey *secret_key, int delta,
                                              int level) override {
    Handle sk = upload(secret_key, FHE_SECRET_KEY), h;
    check(fhe_create_fixed_rotation_key(e_, sk.get(), delta, level, 1, h.out()));
    return fetch_fixed_rotation_key(h.get());
  }
  RotationKey *create_rotation_key(SecretKey *secret_key) override {
    return create_rotation_key(secret_key, -1);
  }
  RotationKey *create_rotation_key(SecretKey *secret_key, int level) override {
    Handle sk = upload(secret_key, FHE_SECRET_KEY);
    std::vector<fhe_data *> raw(64, nullptr);
    int count = 0;
    check(fhe_create_rotation_keys(e_, sk.get(), level, raw.data(), static_cast<int>(raw.size()),
                                   &count));
    std::vector<FixedRotationKey *> keys;
    try {
      for (int i = 0; i < count; i++) keys.push_back(fetch_fixed_rotation_key(raw[i]));
    } catch (...) {
      for (auto k : keys) delete k;
      for (int i = 0; i < count; i++) fhe_data_destroy(raw[i]);
      throw;
    }
    for (int i = 0; i < count; i++) fhe_data_destroy(raw[i]);
    return new RotationKey(keys);
  }
  BootstrapKey *create_bootstrap_key(SecretKey *, int, const std::string &) override {
    not_provided("Create Bootstrap Key");
  }
  SmallBootstrapKey *create_small_bootstrap_key(SecretKey *secret_key) override {
    Handle sk = upload(secret_key, FHE_SECRET_KEY), to_sparse, to_dense;
    check(fhe_create_small_bootstrap_key(e_, sk.get(), to_sparse.out(), to_dense.out()));
    auto sparse = fetch_data<KeySwitchingKey>(to_sparse.get());
    return new SmallBootstrapKey(sparse, fetch_data<KeySwitchingKey>(to_dense.get()));
  }

  // ------------------------------------------------------- encode / decode --

  Plaintext *encode(std::vector<double> &input) override { return encode(input, -1); }
  Plaintext *encode(std::vector<double> &input, int level) override {
    return encode_values(input.data(), nullptr, static_cast<int>(input.size()), level);
  }
  Plaintext *encode(std::vector<std::complex<double>> &input) override { return encode(input, -1); }
  Plaintext *encode(std::vector<std::complex<double>> &input, int level) override {
    std::vector<double> re(input.size()), im(input.size());
    for (size_t i = 0; i < input.size(); i++) {
      re[i] = input[i].real();
      im[i] = input[i].imag();
    }
    return encode_values(re.data(), im.data(), static_cast<int>(input.size()), level);
  }
  std::vector<double> decode(Plaintext *plaintext) override {
    std::vector<double> out;
    for (int u = 0; u < plaintext->size(); u++) {
      Handle pt = upload_text(plaintext->get(u), FHE_UNIT_PLAINTEXT);
      std::vector<double> re(info_.slot_count);
      check(fhe_decode(e_, pt.get(), re.data(), nullptr));
      out.insert(out.end(), re.begin(), re.end());
    }
    return out;
  }
  std::vector<std::complex<double>> decode_complex_plaintext(Plaintext *plaintext) override {
    std::vector<std::complex<double>> out;
    for (int u = 0; u < plaintext->size(); u++) {
      Handle pt = upload_text(plaintext->get(u), FHE_UNIT_PLAINTEXT);
      std::vector<double> re(info_.slot_count), im(info_.slot_count);
      check(fhe_decode(e_, pt.get(), re.data(), im.data()));
      for (int i = 0; i < info_.slot_count; i++) out.emplace_back(re[i], im[i]);
    }
    return out;
  }

  // ------------------------------------------------------------- encrypt --

  Ciphertext *encrypt(std::vector<double> &input, PublicKey *public_key) override {
    return encrypt(input, public_key, -1);
  }
  Ciphertext *encrypt(std::vector<double> &input, PublicKey *public_key, int level) override {
    return encrypt_owned(encode(input, level), public_key, FHE_PUBLIC_KEY);
  }
  Ciphertext *encrypt(std::vector<std::complex<double>> &input, PublicKey *public_key) override {
    return encrypt(input, public_key, -1);
  }
  Ciphertext *encrypt(std::vector<std::complex<double>> &input, PublicKey *public_key,
                      int level) override {
    return encrypt_owned(encode(input, level), public_key, FHE_PUBLIC_KEY);
  }
  Ciphertext *encrypt(Plaintext *plaintext, PublicKey *public_key) override {
    return encrypt_plaintext(plaintext, public_key, FHE_PUBLIC_KEY);
  }
  Ciphertext *encrypt(std::vector<double> &input, SecretKey *secret_key) override {
    return encrypt(input, secret_key, -1);
  }
  Ciphertext *encrypt(std::vector<double> &input, SecretKey *secret_key, int level) override {
    return encrypt_owned(encode(input, level), secret_key, FHE_SECRET_KEY);
  }
  Ciphertext *encrypt(std::vector<std::complex<double>> &input, SecretKey *secret_key) override {
    return encrypt(input, secret_key, -1);
  }
  Ciphertext *encrypt(std::vector<std::complex<double>> &input, SecretKey *secret_key,
                      int level) override {
    return encrypt_owned(encode(input, level), secret_key, FHE_SECRET_KEY);
  }
  Ciphertext *encrypt(Plaintext *plaintext, SecretKey *secret_key) override {
    return encrypt_plaintext(plaintext, secret_key, FHE_SECRET_KEY);
  }

  // ------------------------------------------------------------- decrypt --

  std::vector<double> decrypt(Ciphertext *ciphertext, SecretKey *secret_key) override {
    Plaintext *pt = decrypt_to_plaintext(ciphertext, secret_key);
    try {
      auto values = decode(pt);
      delete pt;
      return values;
    } catch (...) {
      delete pt;
      throw;
    }
  }
  std::vector<std::complex<double>> decrypt_complex(Ciphertext *ciphertext,
                                                    SecretKey *secret_key) override {
    Plaintext *pt = decrypt_to_plaintext(ciphertext, secret_key);
    try {
      auto values = decode_complex_plaintext(pt);
      delete pt;
      return values;
    } catch (...) {
      delete pt;
      throw;
    }
  }
  void decrypt_to_buffer(Ciphertext *ciphertext, double *output, SecretKey *secret_key) override {
    const auto values = decrypt(ciphertext, secret_key);
    std::memcpy(output, values.data(), values.size() * sizeof(double));
  }
  void decrypt_to_complex_buffer(Ciphertext *ciphertext, std::complex<double> *output,
                                 SecretKey *secret_key) override {
    const auto values = decrypt_complex(ciphertext, secret_key);
    for (size_t i = 0; i < values.size(); i++) output[i] = values[i];
  }
  Plaintext *decrypt_to_plaintext(Ciphertext *ciphertext, SecretKey *secret_key) override {
    Handle sk = upload(secret_key, FHE_SECRET_KEY);
    std::vector<UnitPlaintext *> units;
    try {
      for (int u = 0; u < ciphertext->size(); u++) {
        Handle ct = upload_text(ciphertext->get(u), FHE_UNIT_CIPHERTEXT), h;
        check(fhe_decrypt(e_, ct.get(), sk.get(), h.out()));
        units.push_back(fetch_text<UnitPlaintext>(h.get()));
      }
    } catch (...) {
      for (auto x : units) delete x;
      throw;
    }
    return new Plaintext(units);
  }

  // ----------------------------------------------------------------- add --

  Ciphertext *add(Ciphertext *a, Ciphertext *b) override { return pair_ct(a, b, fhe_add); }
  Ciphertext *add(Ciphertext *ct, Plaintext *pt) override {
    return pair_ct_pt(ct, pt, fhe_add_plaintext);
  }
  Ciphertext *add(Plaintext *pt, Ciphertext *ct) override { return add(ct, pt); }
  Ciphertext *add(Ciphertext *ct, std::vector<double> &m) override {
    return with_message(ct, encode(m, ct->level()), fhe_add_plaintext);
  }
  Ciphertext *add(std::vector<double> &m, Ciphertext *ct) override { return add(ct, m); }
  Ciphertext *add(Ciphertext *ct, std::vector<std::complex<double>> &m) override {
    return with_message(ct, encode(m, ct->level()), fhe_add_plaintext);
  }
  Ciphertext *add(std::vector<std::complex<double>> &m, Ciphertext *ct) override {
    return add(ct, m);
  }
  Ciphertext *add(Ciphertext *ct, double *m, int size) override {
    std::vector<double> v(m, m + size);
    return add(ct, v);
  }
  Ciphertext *add(double *m, Ciphertext *ct, int size) override { return add(ct, m, size); }
  Ciphertext *add(Ciphertext *ct, std::complex<double> *m, int size) override {
    std::vector<std::complex<double>> v(m, m + size);
    return add(ct, v);
  }
  Ciphertext *add(std::complex<double> *m, Ciphertext *ct, int size) override {
    return add(ct, m, size);
  }
  Ciphertext *add(Ciphertext *ct, double value) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) { return fhe_add_scalar(e_, x, value, out); });
  }
  Ciphertext *add(double value, Ciphertext *ct) override { return add(ct, value); }
  void add_inplace(Ciphertext *a, Ciphertext *b) override { overwrite(a, add(a, b)); }
  void add_inplace(Ciphertext *ct, Plaintext *pt) override { overwrite(ct, add(ct, pt)); }
  void add_inplace(Plaintext *pt, Ciphertext *ct) override { overwrite(ct, add(ct, pt)); }

  // ------------------------------------------------------------ subtract --

  UnitCiphertext *subtract(UnitCiphertext *a, UnitCiphertext *b) override {
    return unit_pair(a, FHE_UNIT_CIPHERTEXT, b, FHE_UNIT_CIPHERTEXT, fhe_subtract);
  }
  UnitCiphertext *subtract(UnitCiphertext *ct, UnitPlaintext *pt) override {
    return unit_pair(ct, FHE_UNIT_CIPHERTEXT, pt, FHE_UNIT_PLAINTEXT, fhe_subtract_plaintext);
  }
  UnitCiphertext *subtract(UnitPlaintext *pt, UnitCiphertext *ct) override {
    return unit_pair(pt, FHE_UNIT_PLAINTEXT, ct, FHE_UNIT_CIPHERTEXT, fhe_subtract_from_plaintext);
  }
  UnitCiphertext *subtract(UnitCiphertext *ct, std::vector<double> &m) override {
    return unit_with_message(ct, m, fhe_subtract_plaintext, false);
  }
  UnitCiphertext *subtract(std::vector<double> &m, UnitCiphertext *ct) override {
    return unit_with_message(ct, m, fhe_subtract_from_plaintext, true);
  }
  UnitCiphertext *subtract(UnitCiphertext *ct, std::vector<std::complex<double>> &m) override {
    return unit_with_message(ct, m, fhe_subtract_plaintext, false);
  }
  UnitCiphertext *subtract(std::vector<std::complex<double>> &m, UnitCiphertext *ct) override {
    return unit_with_message(ct, m, fhe_subtract_from_plaintext, true);
  }
  UnitCiphertext *subtract(UnitCiphertext *ct, double value) override {
    Handle x = upload_text(ct, FHE_UNIT_CIPHERTEXT), h;
    check(fhe_subtract_scalar(e_, x.get(), value, h.out()));
    return fetch_text<UnitCiphertext>(h.get());
  }
  UnitCiphertext *subtract(double value, UnitCiphertext *ct) override {
    Handle x = upload_text(ct, FHE_UNIT_CIPHERTEXT), neg, h;
    check(fhe_negate(e_, x.get(), neg.out()));
    check(fhe_add_scalar(e_, neg.get(), value, h.out()));
    return fetch_text<UnitCiphertext>(h.get());
  }
  Ciphertext *subtract(Ciphertext *a, Ciphertext *b) override {
    return pair_ct(a, b, fhe_subtract);
  }
  Ciphertext *subtract(Ciphertext *ct, Plaintext *pt) override {
    return pair_ct_pt(ct, pt, fhe_subtract_plaintext);
  }
  Ciphertext *subtract(Plaintext *pt, Ciphertext *ct) override {
    return pair_ct_pt(ct, pt, [](fhe_engine *e, const fhe_data *c, const fhe_data *p, fhe_data **o) {
      return fhe_subtract_from_plaintext(e, p, c, o);
    });
  }
  Ciphertext *subtract(Ciphertext *ct, std::vector<double> &m) override {
    return with_message(ct, encode(m, ct->level()), fhe_subtract_plaintext);
  }
  Ciphertext *subtract(std::vector<double> &m, Ciphertext *ct) override {
    Plaintext *pt = encode(m, ct->level());
    return owned_message(pt, subtract(pt, ct));
  }
  Ciphertext *subtract(Ciphertext *ct, std::vector<std::complex<double>> &m) override {
    return with_message(ct, encode(m, ct->level()), fhe_subtract_plaintext);
  }
  Ciphertext *subtract(std::vector<std::complex<double>> &m, Ciphertext *ct) override {
    Plaintext *pt = encode(m, ct->level());
    return owned_message(pt, subtract(pt, ct));
  }
  Ciphertext *subtract(Ciphertext *ct, double *m, int size) override {
    std::vector<double> v(m, m + size);
    return subtract(ct, v);
  }
  Ciphertext *subtract(double *m, Ciphertext *ct, int size) override {
    std::vector<double> v(m, m + size);
    return subtract(v, ct);
  }
  Ciphertext *subtract(Ciphertext *ct, std::complex<double> *m, int size) override {
    std::vector<std::complex<double>> v(m, m + size);
    return subtract(ct, v);
  }
  Ciphertext *subtract(std::complex<double> *m, Ciphertext *ct, int size) override {
    std::vector<std::complex<double>> v(m, m + size);
    return subtract(v, ct);
  }
  Ciphertext *subtract(Ciphertext *ct, double value) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) {
      return fhe_subtract_scalar(e_, x, value, out);
    });
  }
  Ciphertext *subtract(double value, Ciphertext *ct) override {
    return map_units(ct, [&](UnitCiphertext *u) { return subtract(value, u); });
  }
  void subtract_inplace(Ciphertext *a, Ciphertext *b) override { overwrite(a, subtract(a, b)); }

  // ------------------------------------------------------------ multiply --

  Ciphertext *multiply(Ciphertext *a, Ciphertext *b) override { return pair_ct(a, b, fhe_multiply); }
  Ciphertext *multiply(Ciphertext *a, Ciphertext *b, RelinearizationKey *rk) override {
    Handle key = upload_key(rk->key_switching_key_, FHE_RELINEARIZATION_KEY);
    return pair_ct(a, b, [&](fhe_engine *e, const fhe_data *x, const fhe_data *y, fhe_data **o) {
      return fhe_multiply_relinearize(e, x, y, key.get(), o);
    });
  }
  Ciphertext *square(Ciphertext *ct) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) { return fhe_square(e_, x, nullptr, out); });
  }
  Ciphertext *square(Ciphertext *ct, RelinearizationKey *rk) override {
    Handle key = upload_key(rk->key_switching_key_, FHE_RELINEARIZATION_KEY);
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) { return fhe_square(e_, x, key.get(), out); });
  }
  Ciphertext *multiply(Ciphertext *ct, Plaintext *pt) override {
    return pair_ct_pt(ct, pt, fhe_multiply_plaintext);
  }
  Ciphertext *multiply(Plaintext *pt, Ciphertext *ct) override { return multiply(ct, pt); }
  Ciphertext *multiply(Ciphertext *ct, std::vector<double> &m) override {
    return with_message(ct, encode(m, ct->level()), fhe_multiply_plaintext);
  }
  Ciphertext *multiply(std::vector<double> &m, Ciphertext *ct) override { return multiply(ct, m); }
  Ciphertext *multiply(Ciphertext *ct, std::vector<std::complex<double>> &m) override {
    return with_message(ct, encode(m, ct->level()), fhe_multiply_plaintext);
  }
  Ciphertext *multiply(std::vector<std::complex<double>> &m, Ciphertext *ct) override {
    return multiply(ct, m);
  }
  Ciphertext *multiply(Ciphertext *ct, double *m, int size) override {
    std::vector<double> v(m, m + size);
    return multiply(ct, v);
  }
  Ciphertext *multiply(double *m, Ciphertext *ct, int size) override { return multiply(ct, m, size); }
  Ciphertext *multiply(Ciphertext *ct, std::complex<double> *m, int size) override {
    std::vector<std::complex<double>> v(m, m + size);
    return multiply(ct, v);
  }
  Ciphertext *multiply(std::complex<double> *m, Ciphertext *ct, int size) override {
    return multiply(ct, m, size);
  }
  Ciphertext *multiply(Ciphertext *ct, double value) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) {
      return fhe_multiply_scalar(e_, x, value, out);
    });
  }
  Ciphertext *multiply(double value, Ciphertext *ct) override { return multiply(ct, value); }
  Ciphertext *multiply(Ciphertext *ct, int64_t value) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) {
      return fhe_multiply_integer(e_, x, static_cast<long long>(value), out);
    });
  }
  Ciphertext *multiply(int64_t value, Ciphertext *ct) override { return multiply(ct, value); }
  Ciphertext *multiply_imaginary(Ciphertext *, int64_t) override {
    not_provided("Multiply Imaginary");
  }
  Ciphertext *multiply_imaginary(int64_t, Ciphertext *) override {
    not_provided("Multiply Imaginary");
  }
  Ciphertext *multiply_matrix(double *, Ciphertext *, RotationKey *) override {
    not_provided("Multiply Matrix");
  }
  Ciphertext *multiply_matrix(std::complex<double> *, Ciphertext *, RotationKey *) override {
    not_provided("Multiply Matrix");
  }
  Ciphertext *multiply_matrix(std::vector<double> &, Ciphertext *, RotationKey *) override {
    not_provided("Multiply Matrix");
  }
  Ciphertext *multiply_matrix(std::vector<std::complex<double>> &, Ciphertext *,
                              RotationKey *) override {
    not_provided("Multiply Matrix");
  }
  Ciphertext *relinearize(Ciphertext *ct, RelinearizationKey *rk) override {
    Handle key = upload_key(rk->key_switching_key_, FHE_RELINEARIZATION_KEY);
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) {
      return fhe_relinearize(e_, x, key.get(), out);
    });
  }

  // ---------------------------------------------------- conjugate, rotate --

  UnitPlaintext *conjugate(UnitPlaintext *pt) override {
    Handle x = upload_text(pt, FHE_UNIT_PLAINTEXT), h;
    check(fhe_conjugate_plaintext(e_, x.get(), h.out()));
    return fetch_text<UnitPlaintext>(h.get());
  }
  UnitCiphertext *conjugate(UnitCiphertext *ct, ConjugationKey *ck) override {
    Handle key = upload_key(ck->key_switching_key_, FHE_CONJUGATION_KEY);
    Handle x = upload_text(ct, FHE_UNIT_CIPHERTEXT), h;
    check(fhe_conjugate(e_, x.get(), key.get(), h.out()));
    return fetch_text<UnitCiphertext>(h.get());
  }
  Plaintext *conjugate(Plaintext *pt) override {
    return map_pt(pt, [&](fhe_data *x, fhe_data **out) { return fhe_conjugate_plaintext(e_, x, out); });
  }
  Ciphertext *conjugate(Ciphertext *ct, ConjugationKey *ck) override {
    Handle key = upload_key(ck->key_switching_key_, FHE_CONJUGATION_KEY);
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) {
      return fhe_conjugate(e_, x, key.get(), out);
    });
  }
  Plaintext *rotate(Plaintext *pt, int delta) override {
    return map_pt(pt, [&](fhe_data *x, fhe_data **out) {
      return fhe_rotate_plaintext(e_, x, delta, out);
    });
  }
  Ciphertext *rotate(Ciphertext *ct, FixedRotationKey *key) override {
    Handle k = upload_fixed_key(key);
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) { return fhe_rotate(e_, x, k.get(), out); });
  }
  Ciphertext *rotate(Ciphertext *ct, RotationKey *rotation_key, int delta) override {
    std::vector<Handle> keys = upload_rotation_key(rotation_key);
    std::vector<const fhe_data *> raw;
    for (auto &k : keys) raw.push_back(k.get());
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) {
      return fhe_rotate_with_keys(e_, x, raw.data(), static_cast<int>(raw.size()), delta, 1, out);
    });
  }
  std::vector<Ciphertext *> rotate_batch(Ciphertext *ct,
                                         std::vector<FixedRotationKey *> fixed_keys) override {
    std::vector<Handle> keys;
    std::vector<const fhe_data *> raw;
    for (auto k : fixed_keys) {
      keys.push_back(upload_fixed_key(k));
      raw.push_back(keys.back().get());
    }
    const int count = static_cast<int>(raw.size());
    std::vector<std::vector<UnitCiphertext *>> per_key(count);
    try {
      for (int u = 0; u < ct->size(); u++) {
        Handle x = upload_text(ct->get(u), FHE_UNIT_CIPHERTEXT);
        std::vector<fhe_data *> outs(count, nullptr);
        check(fhe_rotate_batch(e_, x.get(), raw.data(), count, outs.data()));
        for (int i = 0; i < count; i++) {
          Handle h;
          *h.out() = outs[i];
          per_key[i].push_back(fetch_text<UnitCiphertext>(h.get()));
        }
      }
    } catch (...) {
      for (auto &v : per_key)
        for (auto x : v) delete x;
      throw;
    }
    std::vector<Ciphertext *> result;
    for (auto &v : per_key) result.push_back(new Ciphertext(v));
    return result;
  }
  std::vector<Ciphertext *> rotate_batch(Ciphertext *ct, RotationKey *rotation_key,
                                         std::vector<int> deltas) override {
    std::vector<Ciphertext *> result;
    try {
      for (int d : deltas) result.push_back(rotate(ct, rotation_key, d));
    } catch (...) {
      for (auto x : result) delete x;
      throw;
    }
    return result;
  }

  // --------------------------------------------- forms, levels, utilities --

  Plaintext *ntt(Plaintext *pt) override {
    return map_pt(pt, [&](fhe_data *x, fhe_data **out) { return fhe_to_ntt(e_, x, out); });
  }
  Ciphertext *ntt(Ciphertext *ct) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) { return fhe_to_ntt(e_, x, out); });
  }
  Plaintext *intt(Plaintext *pt) override {
    return map_pt(pt, [&](fhe_data *x, fhe_data **out) { return fhe_to_intt(e_, x, out); });
  }
  Ciphertext *intt(Ciphertext *ct) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) { return fhe_to_intt(e_, x, out); });
  }
  Plaintext *rescale(Plaintext *pt) override {
    return map_pt(pt, [&](fhe_data *x, fhe_data **out) { return fhe_rescale(e_, x, out); });
  }
  Ciphertext *rescale(Ciphertext *ct) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) { return fhe_rescale(e_, x, out); });
  }
  Plaintext *level_down(Plaintext *pt, int level) override {
    return map_pt(pt, [&](fhe_data *x, fhe_data **out) { return fhe_level_down(e_, x, level, out); });
  }
  Ciphertext *level_down(Ciphertext *ct, int level) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) { return fhe_level_down(e_, x, level, out); });
  }
  Ciphertext *negate(Ciphertext *ct) override {
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) { return fhe_negate(e_, x, out); });
  }
  Plaintext *clone(Plaintext *pt) override {
    std::vector<UnitPlaintext *> units;
    for (int u = 0; u < pt->size(); u++) units.push_back(copy_text(pt->get(u)));
    return new Plaintext(units);
  }
  Ciphertext *clone(Ciphertext *ct) override {
    std::vector<UnitCiphertext *> units;
    for (int u = 0; u < ct->size(); u++) units.push_back(copy_text(ct->get(u)));
    return new Ciphertext(units);
  }

  // -------------------------------------------------------- bootstrapping --

  Ciphertext *bootstrap(Ciphertext *ct, RelinearizationKey *rk, ConjugationKey *ck,
                        RotationKey *rotation_key, SmallBootstrapKey *sbk,
                        int stage_count) override {
    Handle r = upload_key(rk->key_switching_key_, FHE_RELINEARIZATION_KEY);
    Handle c = upload_key(ck->key_switching_key_, FHE_CONJUGATION_KEY);
    Handle sparse = upload_key(sbk->to_sparse_, FHE_KEY_SWITCHING_KEY);
    Handle dense = upload_key(sbk->to_dense_, FHE_KEY_SWITCHING_KEY);
    std::vector<Handle> keys = upload_rotation_key(rotation_key);
    std::vector<const fhe_data *> raw;
    for (auto &k : keys) raw.push_back(k.get());
    return map_ct(ct, [&](fhe_data *x, fhe_data **out) {
      return fhe_bootstrap(e_, x, r.get(), c.get(), raw.data(), static_cast<int>(raw.size()),
                           sparse.get(), dense.get(), stage_count, out);
    });
  }
  Ciphertext *bootstrap(Ciphertext *, RelinearizationKey *, ConjugationKey *,
                        BootstrapKey *) override {
    not_provided("Bootstrap With Bootstrap Key");
  }
  Ciphertext *mod_raise(Ciphertext *, SmallBootstrapKey *) override { not_provided("Mod Raise"); }
  Ciphertext *mod_raise(Ciphertext *, BootstrapKey *) override { not_provided("Mod Raise"); }

  // ------------------------------------- outside the accelerated path --

  std::vector<Ciphertext *> make_power_basis(Ciphertext *, int, RelinearizationKey *) override {
    not_provided("Make Power Basis");
  }
  std::vector<Ciphertext *> make_chebyshev_basis(Ciphertext *, int,
                                                 RelinearizationKey *) override {
    not_provided("Make Chebyshev Basis");
  }
  Ciphertext *weighted_sum(std::vector<Ciphertext *> &, std::vector<int64_t> &) override {
    not_provided("Weighted Sum");
  }
  Ciphertext *weighted_sum(std::vector<Ciphertext *> &, std::vector<double> &) override {
    not_provided("Weighted Sum");
  }
  Ciphertext *evaluate_polynomial(Ciphertext *, std::vector<int64_t> &,
                                  RelinearizationKey *) override {
    not_provided("Evaluate Polynomial");
  }
  Ciphertext *evaluate_polynomial(Ciphertext *, std::vector<double> &,
                                  RelinearizationKey *) override {
    not_provided("Evaluate Polynomial");
  }
  Ciphertext *evaluate_chebyshev_polynomial(Ciphertext *, std::vector<int64_t> &,
                                            RelinearizationKey *) override {
    not_provided("Evaluate Chebyshev Polynomial");
  }
  Ciphertext *evaluate_chebyshev_polynomial(Ciphertext *, std::vector<double> &,
                                            RelinearizationKey *) override {
    not_provided("Evaluate Chebyshev Polynomial");
  }
  Ciphertext *sum_1d_by_row(Ciphertext *, RotationKey *) override { not_provided("Sum 1D By Row"); }
  Ciphertext *sum_1d_by_column(Ciphertext *) override { not_provided("Sum 1D By Column"); }
  Ciphertext *sum_2d(Ciphertext *, RotationKey *) override { not_provided("Sum 2D"); }
  Ciphertext *stack_by_row(std::vector<Ciphertext *> &) override { not_provided("Stack By Row"); }

  int get_slot_count() const override { return info_.slot_count; }
  int get_max_level() const override { return info_.max_level; }
  std::string get_mode() const override { return "gpu"; }

 private:
  fhe_engine *e_ = nullptr;
  fhe_engine_info info_{};
  SchemePreset preset_;
  uint8_t log_coeff_ = 0;
  uint8_t log_slot_ = 0;

  using PairFn = int (*)(fhe_engine *, const fhe_data *, const fhe_data *, fhe_data **);

  // ---- host object <-> device handle

  Handle upload_limbs(Data *x, int type, long double scale) {
    const int polys = static_cast<int>(x->polynomial_count());
    const int chains = x->chain_count_;
    const size_t n = x->coeff_count_;
    std::vector<int64_t> buf(static_cast<size_t>(polys) * chains * n);
    for (int p = 0; p < polys; p++)
      for (int j = 0; j < chains; j++)
        std::memcpy(&buf[(static_cast<size_t>(p) * chains + j) * n], x->get_polynomial(p)->get(j),
                    n * sizeof(int64_t));
    Handle h;
    check(fhe_data_upload(e_, type, static_cast<int>(x->flag_), x->moduli_id_, polys, scale,
                          buf.data(), h.out()));
    return h;
  }
  Handle upload(Data *x, int type) { return upload_limbs(x, type, 1.0L); }
  template <class T>
  Handle upload_text(T *x, int type) { return upload_limbs(x, type, x->ckks_scale_); }
  Handle upload_key(KeySwitchingKey *k, int type) { return upload_limbs(k, type, 1.0L); }
  Handle upload_fixed_key(FixedRotationKey *k) {
    Handle h = upload_limbs(k->key_switching_key_, FHE_FIXED_ROTATION_KEY, 1.0L);
    check(fhe_data_set_delta(h.get(), k->delta_));
    return h;
  }
  std::vector<Handle> upload_rotation_key(RotationKey *rk) {
    std::vector<Handle> keys;
    for (auto k : rk->fixed_rotation_keys_) keys.push_back(upload_fixed_key(k));
    return keys;
  }

  std::vector<Polynomial *> fetch_polynomials(fhe_data *d, fhe_data_info &info) {
    check(fhe_data_info_get(d, &info));
    const size_t n = info_.coeff_count;
    std::vector<int64_t> buf(static_cast<size_t>(info.polys) * info.chains * n);
    check(fhe_data_download(d, buf.data()));
    std::vector<Polynomial *> polys;
    for (int p = 0; p < info.polys; p++) {
      auto poly = new Polynomial(static_cast<DataFlag>(info.flag), info.moduli_id, info.chains,
                                 static_cast<int>(n));
      for (int j = 0; j < info.chains; j++)
        std::memcpy(poly->get(j), &buf[(static_cast<size_t>(p) * info.chains + j) * n],
                    n * sizeof(int64_t));
      polys.push_back(poly);
    }
    return polys;
  }
  template <class T>
  T *fetch_data(fhe_data *d) {
    fhe_data_info info;
    auto polys = fetch_polynomials(d, info);
    return new T(polys, static_cast<DataFlag>(info.flag), preset_, log_slot_, log_coeff_,
                 static_cast<uint8_t>(info_.special_prime_count), info.moduli_id, info.level,
                 info.chains, info_.coeff_count);
  }
  template <class T>
  T *fetch_text(fhe_data *d) {
    fhe_data_info info;
    auto polys = fetch_polynomials(d, info);
    return new T(polys, static_cast<DataFlag>(info.flag), preset_, log_slot_, log_coeff_,
                 static_cast<uint8_t>(info_.special_prime_count), info.moduli_id, info.level,
                 info.chains, info_.coeff_count, info.ckks_scale);
  }
  // The slot permutation and signs a rotation by `delta` applies, as the reference
  // keeps them beside each rotation key (CKKSPrecomputed::make_permutation_parameters,
  // ckks/precomputed.cpp:395-406).
  std::pair<PermutationParameters *, PermutationParameters *> permutation_parameters(int delta) {
    auto permutation = new PermutationParameters();
    auto sign = new PermutationParameters();
    permutation->values_.resize(info_.coeff_count);
    sign->values_.resize(info_.coeff_count);
    get_permutation_and_sign(permutation->values_.data(), sign->values_.data(), info_.coeff_count,
                             delta);
    return {permutation, sign};
  }
  FixedRotationKey *fetch_fixed_rotation_key(fhe_data *d) {
    fhe_data_info info;
    check(fhe_data_info_get(d, &info));
    auto [permutation, sign] = permutation_parameters(info.delta);
    return new FixedRotationKey(fetch_data<KeySwitchingKey>(d), permutation, sign, info.delta);
  }
  template <class T>
  T *copy_text(T *x) {
    std::vector<Polynomial *> polys;
    for (uint32_t p = 0; p < x->polynomial_count(); p++) {
      auto poly = new Polynomial(x->flag_, x->moduli_id_, x->chain_count_, x->coeff_count_);
      for (int j = 0; j < x->chain_count_; j++)
        std::memcpy(poly->get(j), x->get_polynomial(p)->get(j), x->coeff_count_ * sizeof(int64_t));
      polys.push_back(poly);
    }
    return new T(polys, x->flag_, x->scheme_preset_, x->log_slot_count_, x->log_coeff_count_,
                 x->special_prime_count_, x->moduli_id_, x->level_, x->chain_count_,
                 x->coeff_count_, x->ckks_scale_);
  }

  // ---- long texts, unit by unit

  Plaintext *encode_values(const double *re, const double *im, int count, int level) {
    if (level < 0) level = info_.max_level;  // the reference's get_max_level() default
    std::vector<UnitPlaintext *> units;
    try {
      for (int start = 0; start < count || (count == 0 && units.empty()); start += info_.slot_count) {
        const int chunk = std::max(0, std::min(info_.slot_count, count - start));
        Handle h;
        check(fhe_encode(e_, re ? re + start : nullptr, im ? im + start : nullptr, chunk, level, 0,
                         h.out()));
        units.push_back(fetch_text<UnitPlaintext>(h.get()));
        if (count == 0) break;
      }
    } catch (...) {
      for (auto x : units) delete x;
      throw;
    }
    return new Plaintext(units);
  }
  Ciphertext *encrypt_plaintext(Plaintext *pt, Data *key, int key_type) {
    Handle k = upload(key, key_type);
    std::vector<UnitCiphertext *> units;
    try {
      for (int u = 0; u < pt->size(); u++) {
        Handle x = upload_text(pt->get(u), FHE_UNIT_PLAINTEXT), h;
        check(fhe_encrypt(e_, x.get(), k.get(), h.out()));
        units.push_back(fetch_text<UnitCiphertext>(h.get()));
      }
    } catch (...) {
      for (auto x : units) delete x;
      throw;
    }
    return new Ciphertext(units);
  }
  Ciphertext *encrypt_owned(Plaintext *pt, Data *key, int key_type) {
    return owned_message(pt, encrypt_plaintext(pt, key, key_type));
  }
  template <class R>
  R *owned_message(Plaintext *pt, R *result) {
    delete pt;
    return result;
  }
  template <class F>
  Ciphertext *map_units(Ciphertext *ct, F f) {
    std::vector<UnitCiphertext *> units;
    try {
      for (int u = 0; u < ct->size(); u++) units.push_back(f(ct->get(u)));
    } catch (...) {
      for (auto x : units) delete x;
      throw;
    }
    return new Ciphertext(units);
  }
  template <class F>
  Ciphertext *map_ct(Ciphertext *ct, F f) {
    return map_units(ct, [&](UnitCiphertext *u) {
      Handle x = upload_text(u, FHE_UNIT_CIPHERTEXT), h;
      check(f(x.get(), h.out()));
      return fetch_text<UnitCiphertext>(h.get());
    });
  }
  template <class F>
  Plaintext *map_pt(Plaintext *pt, F f) {
    std::vector<UnitPlaintext *> units;
    try {
      for (int u = 0; u < pt->size(); u++) {
        Handle x = upload_text(pt->get(u), FHE_UNIT_PLAINTEXT), h;
        check(f(x.get(), h.out()));
        units.push_back(fetch_text<UnitPlaintext>(h.get()));
      }
    } catch (...) {
      for (auto x : units) delete x;
      throw;
    }
    return new Plaintext(units);
  }
  static int partner(int count, int u, const char *what) {
    if (count == 1) return 0;
    if (u >= count) throw std::invalid_argument(std::string(what) + ": the texts have different sizes.");
    return u;
  }
  template <class F>
  Ciphertext *pair_ct(Ciphertext *a, Ciphertext *b, F f) {
    if (a->size() != b->size() && b->size() != 1)
      throw std::invalid_argument("Ciphertext Operation: the ciphertexts have different sizes.");
    int u = 0;
    return map_units(a, [&](UnitCiphertext *x) {
      Handle ha = upload_text(x, FHE_UNIT_CIPHERTEXT);
      Handle hb = upload_text(b->get(partner(b->size(), u++, "Ciphertext Operation")),
                              FHE_UNIT_CIPHERTEXT);
      Handle h;
      check(f(e_, ha.get(), hb.get(), h.out()));
      return fetch_text<UnitCiphertext>(h.get());
    });
  }
  template <class F>
  Ciphertext *pair_ct_pt(Ciphertext *ct, Plaintext *pt, F f) {
    if (ct->size() != pt->size() && pt->size() != 1)
      throw std::invalid_argument("Ciphertext And Plaintext Operation: the texts have different sizes.");
    int u = 0;
    return map_units(ct, [&](UnitCiphertext *x) {
      Handle hc = upload_text(x, FHE_UNIT_CIPHERTEXT);
      Handle hp = upload_text(pt->get(partner(pt->size(), u++, "Ciphertext And Plaintext Operation")),
                              FHE_UNIT_PLAINTEXT);
      Handle h;
      check(f(e_, hc.get(), hp.get(), h.out()));
      return fetch_text<UnitCiphertext>(h.get());
    });
  }
  Ciphertext *with_message(Ciphertext *ct, Plaintext *pt, PairFn f) {
    try {
      return owned_message(pt, pair_ct_pt(ct, pt, f));
    } catch (...) {
      delete pt;
      throw;
    }
  }
  template <class A, class B>
  UnitCiphertext *unit_pair(A *a, int type_a, B *b, int type_b, PairFn f) {
    Handle ha = upload_text(a, type_a), hb = upload_text(b, type_b), h;
    check(f(e_, ha.get(), hb.get(), h.out()));
    return fetch_text<UnitCiphertext>(h.get());
  }
  template <class V>
  UnitCiphertext *unit_with_message(UnitCiphertext *ct, std::vector<V> &m, PairFn f,
                                    bool message_first) {
    Plaintext *pt = encode(m, ct->level_);
    try {
      Handle hc = upload_text(ct, FHE_UNIT_CIPHERTEXT);
      Handle hp = upload_text(pt->get(0), FHE_UNIT_PLAINTEXT), h;
      check(message_first ? f(e_, hp.get(), hc.get(), h.out()) : f(e_, hc.get(), hp.get(), h.out()));
      delete pt;
      return fetch_text<UnitCiphertext>(h.get());
    } catch (...) {
      delete pt;
      throw;
    }
  }
  // The in-place forms: the result's words replace the destination's, which keeps
  // its shape (the reference's in-place operations require matching operands).
  void overwrite(Ciphertext *dst, Ciphertext *result) {
    try {
      if (result->size() != dst->size())
        throw std::invalid_argument("Add Inplace: the result has another size.");
      for (int u = 0; u < dst->size(); u++) {
        UnitCiphertext *d = dst->get(u), *r = result->get(u);
        if (d->flag_ != r->flag_ || d->moduli_id_ != r->moduli_id_ ||
            d->polynomial_count() != r->polynomial_count())
          throw std::invalid_argument(
              "Add Inplace: the result's form, level or size differs from the destination's.");
        for (uint32_t p = 0; p < d->polynomial_count(); p++)
          for (int j = 0; j < d->chain_count_; j++)
            std::memcpy(d->get_polynomial(p)->get(j), r->get_polynomial(p)->get(j),
                        d->coeff_count_ * sizeof(int64_t));
      }
    } catch (...) {
      delete result;
      throw;
    }
    delete result;
  }
};

AbstractEngine *create_default_engine(const std::string &scheme_preset) {
  std::string lower = scheme_preset;
  for (auto &c : lower) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  if (lower == "ckks") return create_ckks_engine(CKKSConfig{});
  throw std::invalid_argument("The given scheme is not supported.");
}

AbstractEngine *create_ckks_engine(CKKSConfig config) { return new GpuCKKSEngine(config); }

}  // namespace desilo::fhe
