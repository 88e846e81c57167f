// C ABI of the B200 CKKS engine (include/fhe_b200.h): handle wrappers, status
// codes and the thread-local last-error message.  No function lets a C++
// exception or a CUDA error escape.
#include <cstring>
#include <new>
#include <string>

#include "../../include/fhe_b200.h"
#include "engine.hpp"

using fhe_b200::Data;
using fhe_b200::Engine;

struct fhe_engine {
  Engine *impl;
};

struct fhe_data {
  Data *impl;
};

struct fhe_bootstrap_key {
  fhe_b200::BootstrapKey *impl;
};

namespace fhe_b200 {
namespace {
thread_local std::string g_last_error;
}
void set_last_error(const std::string &message) { g_last_error = message; }
}  // namespace fhe_b200

namespace {

// Every call runs inside an NVTX range named after the C-ABI function, so Nsight
// tools show the reference-level operations around their kernels.
template <class F>
int guarded(const char *name, F &&f) {
  const fhe_b200::NvtxRange range(name);
  try {
    f();
    fhe_b200::set_last_error("");
    return FHE_OK;
  } catch (const std::invalid_argument &e) {
    fhe_b200::set_last_error(e.what());
    return FHE_ERR_INVALID_ARGUMENT;
  } catch (const std::out_of_range &e) {
    fhe_b200::set_last_error(e.what());
    return FHE_ERR_INVALID_ARGUMENT;
  } catch (const fhe_b200::CudaError &e) {
    fhe_b200::set_last_error(e.what());
    return FHE_ERR_CUDA;
  } catch (const std::bad_alloc &) {
    fhe_b200::set_last_error("out of device or host memory");
    return FHE_ERR_OUT_OF_MEMORY;
  } catch (const std::runtime_error &e) {
    fhe_b200::set_last_error(e.what());
    return FHE_ERR_RUNTIME;
  } catch (...) {
    fhe_b200::set_last_error("unknown error");
    return FHE_ERR_RUNTIME;
  }
}

#define REQUIRE_HANDLE(h)                                  \
  do {                                                     \
    if (!(h) || !(h)->impl) {                              \
      fhe_b200::set_last_error("null handle: " #h);        \
      return FHE_ERR_NULL_HANDLE;                          \
    }                                                      \
  } while (0)

#define REQUIRE_OUT(p)                                     \
  do {                                                     \
    if (!(p)) {                                            \
      fhe_b200::set_last_error("null output pointer: " #p); \
      return FHE_ERR_NULL_HANDLE;                          \
    }                                                      \
  } while (0)

// The object behind a handle, checked to be alive and owned by `engine`
// (is_compatible, engine_require.cpp:15-22).
const Data &live(const fhe_engine *engine, const fhe_data *d) {
  if (!d->impl->engine) throw std::runtime_error("the engine of the input object was destroyed.");
  if (engine && d->impl->engine != engine->impl)
    throw std::runtime_error("the input object is not compatible with this engine.");
  return *d->impl;
}

fhe_data *wrap(std::unique_ptr<Data> d) {
  auto h = new fhe_data;
  h->impl = d.release();
  return h;
}

}  // namespace

extern "C" {

const char *fhe_last_error(void) { return fhe_b200::g_last_error.c_str(); }

void fhe_config_default(fhe_config *config) {
  if (!config) return;
  config->log_coeff_count = 14;
  config->log_slot_count = -1;
  config->special_prime_count = 1;
  config->max_level = -1;
  config->scheme_preset = FHE_PRESET_CKKS_40_60_DEFAULT;
}

static fhe_b200::Config to_config(const fhe_config *config) {
  fhe_b200::Config c;
  c.log_coeff_count = config->log_coeff_count;
  c.log_slot_count = config->log_slot_count;
  c.special_prime_count = config->special_prime_count;
  c.max_level = config->max_level;
  c.preset = static_cast<fhe_b200::SchemePreset>(config->scheme_preset);
  return c;
}

static void fill_info(const fhe_b200::Parameters &p, fhe_engine_info *info) {
  info->coeff_count = p.n;
  info->slot_count = p.slot_count;
  info->chain_count = p.chain_count;
  info->prime_count = p.prime_count;
  info->special_prime_count = p.special_prime_count;
  info->full_level = p.full_level;
  info->max_level = p.max_level();
  info->max_key_switching_level = p.max_key_switching_level();
  info->scale_bit_length = p.preset.scale_bits;
}

int fhe_parameters_query(const fhe_config *config, fhe_engine_info *info, uint64_t *moduli,
                         int capacity) {
  REQUIRE_OUT(config);
  return guarded(__func__, [&] {
    fhe_b200::Parameters p(to_config(config));
    if (info) fill_info(p, info);
    if (moduli)
      for (int i = 0; i < capacity && i < p.prime_count; i++) moduli[i] = p.q[i];
  });
}

int fhe_parameters_tables(const fhe_config *config, uint64_t *k, int64_t *r_squared,
                          int64_t *n_inverse, int64_t *root, int64_t *root_inverse) {
  REQUIRE_OUT(config);
  return guarded(__func__, [&] {
    fhe_b200::Parameters p(to_config(config));
    if (k) std::memcpy(k, p.k.data(), sizeof(uint64_t) * p.k.size());
    if (r_squared) std::memcpy(r_squared, p.r_squared.data(), sizeof(int64_t) * p.r_squared.size());
    if (n_inverse) std::memcpy(n_inverse, p.n_inverse.data(), sizeof(int64_t) * p.n_inverse.size());
    if (root) std::memcpy(root, p.root.data(), sizeof(int64_t) * p.root.size());
    if (root_inverse)
      std::memcpy(root_inverse, p.root_inverse.data(), sizeof(int64_t) * p.root_inverse.size());
  });
}

int fhe_engine_create(const fhe_config *config, fhe_engine **engine) {
  REQUIRE_OUT(config);
  REQUIRE_OUT(engine);
  *engine = nullptr;
  return guarded(__func__, [&] {
    auto e = new Engine(to_config(config));
    *engine = new fhe_engine{e};
  });
}

int fhe_engine_destroy(fhe_engine *engine) {
  if (!engine) return FHE_OK;
  int rc = guarded(__func__, [&] { delete engine->impl; });
  delete engine;
  return rc;
}

int fhe_engine_info_get(const fhe_engine *engine, fhe_engine_info *info) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(info);
  return guarded(__func__, [&] {
    fill_info(engine->impl->params, info);
  });
}

int fhe_engine_moduli(const fhe_engine *engine, uint64_t *moduli, int capacity) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(moduli);
  return guarded(__func__, [&] {
    const auto &q = engine->impl->params.q;
    for (int i = 0; i < capacity && i < static_cast<int>(q.size()); i++) moduli[i] = q[i];
  });
}

int fhe_engine_moduli_id(const fhe_engine *engine, int level, int *moduli_id) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(moduli_id);
  return guarded(__func__, [&] { *moduli_id = engine->impl->params.moduli_id(level); });
}

int fhe_engine_synchronize(fhe_engine *engine) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->synchronize(); });
}

int fhe_engine_set_stream(fhe_engine *engine, void *cuda_stream) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->set_stream(static_cast<cudaStream_t>(cuda_stream)); });
}

int fhe_engine_set_profiling(fhe_engine *engine, int enable) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->set_profiling(enable != 0); });
}

int fhe_engine_profile_report(fhe_engine *engine, char *buffer, int capacity) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(buffer);
  return guarded(__func__, [&] {
    const std::string r = engine->impl->profile_report();
    if (capacity <= 0) throw std::invalid_argument("the report buffer is empty.");
    const size_t n = std::min(r.size(), static_cast<size_t>(capacity - 1));
    std::memcpy(buffer, r.data(), n);
    buffer[n] = '\0';
  });
}

int fhe_engine_profile_reset(fhe_engine *engine) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->profile_reset(); });
}

unsigned long long fhe_kernel_launch_count(void) { return fhe_b200::kernel_launch_count(); }

int fhe_data_upload(fhe_engine *engine, int type, int flag, int moduli_id, int polys,
                    long double ckks_scale, const int64_t *host_limbs, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    *out = wrap(engine->impl->upload(type, flag, moduli_id, polys, ckks_scale, host_limbs));
  });
}

int fhe_data_download(const fhe_data *data, int64_t *host_limbs) {
  REQUIRE_HANDLE(data);
  return guarded(__func__, [&] { live(nullptr, data).engine->download(*data->impl, host_limbs); });
}

int fhe_data_download_async(const fhe_data *data, int64_t *host_limbs) {
  REQUIRE_HANDLE(data);
  return guarded(__func__, [&] { live(nullptr, data).engine->download_async(*data->impl, host_limbs); });
}

int fhe_data_serialized_size(const fhe_data *data, uint64_t *size) {
  REQUIRE_HANDLE(data);
  REQUIRE_OUT(size);
  return guarded(__func__, [&] { *size = live(nullptr, data).engine->serialized_size(*data->impl); });
}

int fhe_data_serialize(const fhe_data *data, void *buffer, uint64_t capacity) {
  REQUIRE_HANDLE(data);
  REQUIRE_OUT(buffer);
  return guarded(__func__, [&] {
    live(nullptr, data).engine->serialize(*data->impl, buffer, static_cast<size_t>(capacity));
  });
}

int fhe_data_deserialize(fhe_engine *engine, const void *buffer, uint64_t size, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(buffer);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->deserialize(buffer, static_cast<size_t>(size))); });
}

int fhe_data_info_get(const fhe_data *data, fhe_data_info *info) {
  REQUIRE_HANDLE(data);
  REQUIRE_OUT(info);
  return guarded(__func__, [&] {
    const Data &d = live(nullptr, data);
    info->type = d.type;
    info->flag = d.flag;
    info->moduli_id = d.moduli_id;
    info->level = d.level();
    info->polys = d.polys;
    info->chains = d.chains;
    info->delta = d.delta;
    info->ckks_scale = d.scale;
  });
}

int fhe_data_set_delta(fhe_data *data, int delta) {
  REQUIRE_HANDLE(data);
  data->impl->delta = delta;
  return FHE_OK;
}

int fhe_data_device_pointer(const fhe_data *data, int64_t **device_limbs) {
  REQUIRE_HANDLE(data);
  REQUIRE_OUT(device_limbs);
  *device_limbs = data->impl->d;
  return FHE_OK;
}

int fhe_data_destroy(fhe_data *data) {
  if (!data) return FHE_OK;
  int rc = guarded(__func__, [&] { delete data->impl; });
  delete data;
  return rc;
}

#define UNARY_OP(name, call)                                                  \
  int name(fhe_engine *engine, const fhe_data *x, fhe_data **out) {           \
    REQUIRE_HANDLE(engine);                                                   \
    REQUIRE_HANDLE(x);                                                        \
    REQUIRE_OUT(out);                                                         \
    *out = nullptr;                                                           \
    return guarded(__func__, [&] { *out = wrap(engine->impl->call(live(engine, x))); }); \
  }

UNARY_OP(fhe_rescale, rescale)
UNARY_OP(fhe_to_ntt, to_ntt)
UNARY_OP(fhe_to_intt, to_intt)

int fhe_multiply(fhe_engine *engine, const fhe_data *a, const fhe_data *b, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(a);
  REQUIRE_HANDLE(b);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->multiply(live(engine, a), live(engine, b))); });
}

int fhe_multiply_relinearize(fhe_engine *engine, const fhe_data *a, const fhe_data *b,
                             const fhe_data *rk, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(a);
  REQUIRE_HANDLE(b);
  REQUIRE_HANDLE(rk);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__,
                 [&] { *out = wrap(engine->impl->multiply_relinearize(live(engine, a), live(engine, b), live(engine, rk))); });
}

int fhe_multiply_relinearize_rescale(fhe_engine *engine, const fhe_data *a, const fhe_data *b,
                                     const fhe_data *rk, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(a);
  REQUIRE_HANDLE(b);
  REQUIRE_HANDLE(rk);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    *out = wrap(engine->impl->multiply_relinearize_rescale(live(engine, a), live(engine, b), live(engine, rk)));
  });
}

int fhe_relinearize(fhe_engine *engine, const fhe_data *ct, const fhe_data *rk, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_HANDLE(rk);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->relinearize(live(engine, ct), live(engine, rk))); });
}

int fhe_ntt_limbs(fhe_engine *engine, int64_t *device_limbs, int moduli_id, int chains, int polys,
                  long long poly_stride, int inverse) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] {
    engine->impl->ntt_limbs(device_limbs, moduli_id, chains, polys, poly_stride, inverse != 0);
  });
}

int fhe_mont_mult_limbs(fhe_engine *engine, const int64_t *a, const int64_t *b, int64_t *y,
                        int moduli_id, int chains, int polys, long long poly_stride) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] {
    engine->impl->mont_mult_limbs(a, b, y, moduli_id, chains, polys, poly_stride);
  });
}

}  // extern "C"

extern "C" {

int fhe_level_down(fhe_engine *engine, const fhe_data *text, int level, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(text);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->level_down(live(engine, text), level)); });
}

int fhe_rotate(fhe_engine *engine, const fhe_data *ct, const fhe_data *key, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_HANDLE(key);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->rotate(live(engine, ct), live(engine, key))); });
}

int fhe_rotate_with_keys(fhe_engine *engine, const fhe_data *ct, const fhe_data *const *keys,
                         int key_count, int delta, int normalize_by_slot_count, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_OUT(out);
  *out = nullptr;
  if (key_count < 1 || keys == nullptr) {
    fhe_b200::set_last_error(
        "Rotate Unit Ciphertext With Rotation Key: the input fixed rotation key vector is empty.");
    return FHE_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < key_count; i++) REQUIRE_HANDLE(keys[i]);
  return guarded(__func__, [&] {
    std::vector<const fhe_b200::Data *> list;
    for (int i = 0; i < key_count; i++) list.push_back(&live(engine, keys[i]));
    *out = wrap(engine->impl->rotate(live(engine, ct), list, delta, normalize_by_slot_count != 0));
  });
}

int fhe_rotate_plaintext(fhe_engine *engine, const fhe_data *pt, int delta, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(pt);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->rotate_plain(live(engine, pt), delta)); });
}

int fhe_conjugate(fhe_engine *engine, const fhe_data *ct, const fhe_data *key, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_HANDLE(key);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->conjugate(live(engine, ct), live(engine, key))); });
}

int fhe_conjugate_plaintext(fhe_engine *engine, const fhe_data *pt, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(pt);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->conjugate_plain(live(engine, pt))); });
}

int fhe_switch_key(fhe_engine *engine, const fhe_data *ct, const fhe_data *key, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_HANDLE(key);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->switch_key(live(engine, ct), live(engine, key))); });
}

}  // extern "C"

extern "C" {

int fhe_encode(fhe_engine *engine, const double *re, const double *im, int count, int level,
               int include_special, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__,
                 [&] { *out = wrap(engine->impl->encode(re, im, count, level, include_special != 0)); });
}

int fhe_decode(fhe_engine *engine, const fhe_data *pt, double *re, double *im) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(pt);
  return guarded(__func__, [&] { engine->impl->decode(live(engine, pt), re, im); });
}

}  // extern "C"

extern "C" {

int fhe_engine_seed(fhe_engine *engine, const uint32_t *seed, const uint8_t *nonce) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->seed(seed, nonce); });
}

int fhe_create_secret_key(fhe_engine *engine, int level, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    auto &e = *engine->impl;
    *out = wrap(e.create_secret_key(level < 0 ? e.params.max_level() : level));
  });
}

int fhe_create_secret_key_from(fhe_engine *engine, const int64_t *secret, int count, int level,
                               fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    auto &e = *engine->impl;
    *out = wrap(e.create_secret_key(secret, count, level < 0 ? e.params.max_level() : level));
  });
}

int fhe_create_sparse_secret_key(fhe_engine *engine, int hamming_weight, int level,
                                 fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    auto &e = *engine->impl;
    *out = wrap(e.create_sparse_secret_key(hamming_weight, level < 0 ? e.params.max_level() : level));
  });
}

int fhe_create_public_key(fhe_engine *engine, const fhe_data *sk, int level, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(sk);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    auto &e = *engine->impl;
    *out = wrap(e.create_public_key(live(engine, sk), level < 0 ? e.params.max_level() : level));
  });
}

int fhe_create_relinearization_key(fhe_engine *engine, const fhe_data *sk, int level,
                                   fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(sk);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    auto &e = *engine->impl;
    *out = wrap(e.create_relinearization_key(
        live(engine, sk), level < 0 ? e.params.max_key_switching_level() : level));
  });
}

int fhe_create_fixed_rotation_key(fhe_engine *engine, const fhe_data *sk, int delta, int level,
                                  int normalize_by_slot_count, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(sk);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    auto &e = *engine->impl;
    const int nd = e.normalized_delta(delta, normalize_by_slot_count != 0);
    *out = wrap(e.create_fixed_rotation_key(
        live(engine, sk), nd, level < 0 ? e.params.max_key_switching_level() : level));
  });
}

int fhe_create_rotation_keys(fhe_engine *engine, const fhe_data *sk, int level, fhe_data **keys,
                             int capacity, int *count) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(sk);
  REQUIRE_OUT(keys);
  REQUIRE_OUT(count);
  *count = 0;
  return guarded(__func__, [&] {
    auto &e = *engine->impl;
    int needed = 0;
    for (int d = 1; d < e.params.n / 2; d <<= 1) needed++;
    if (capacity < needed)
      throw std::invalid_argument("Create Rotation Key: the output array holds fewer than " +
                                  std::to_string(needed) + " keys.");
    auto made = e.create_rotation_keys(live(engine, sk),
                                       level < 0 ? e.params.max_key_switching_level() : level);
    for (auto &k : made) keys[(*count)++] = wrap(std::move(k));
  });
}

int fhe_create_conjugation_key(fhe_engine *engine, const fhe_data *sk, int level, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(sk);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    auto &e = *engine->impl;
    *out = wrap(e.create_conjugation_key(live(engine, sk),
                                         level < 0 ? e.params.max_key_switching_level() : level));
  });
}

int fhe_encrypt(fhe_engine *engine, const fhe_data *pt, const fhe_data *key, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(pt);
  REQUIRE_HANDLE(key);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->encrypt(live(engine, pt), live(engine, key))); });
}

int fhe_decrypt(fhe_engine *engine, const fhe_data *ct, const fhe_data *sk, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_HANDLE(sk);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->decrypt(live(engine, ct), live(engine, sk))); });
}

}  // extern "C"

extern "C" {

#define FHE_BINARY_OP(name, call)                                                      \
  int name(fhe_engine *engine, const fhe_data *a, const fhe_data *b, fhe_data **out) { \
    REQUIRE_HANDLE(engine);                                                            \
    REQUIRE_HANDLE(a);                                                                 \
    REQUIRE_HANDLE(b);                                                                 \
    REQUIRE_OUT(out);                                                                  \
    *out = nullptr;                                                                    \
    return guarded(__func__, [&] {                                                               \
      auto &e = *engine->impl;                                                         \
      const Data &x = live(engine, a);                                                 \
      const Data &y = live(engine, b);                                                 \
      *out = wrap(call);                                                               \
    });                                                                                \
  }
FHE_BINARY_OP(fhe_add, e.add(x, y))
FHE_BINARY_OP(fhe_subtract, e.subtract(x, y))
FHE_BINARY_OP(fhe_add_plaintext, e.add_plain(x, y))
FHE_BINARY_OP(fhe_subtract_plaintext, e.subtract_plain(x, y))
FHE_BINARY_OP(fhe_subtract_from_plaintext, e.subtract_from_plain(x, y))
FHE_BINARY_OP(fhe_multiply_plaintext, e.multiply_plain(x, y))
#undef FHE_BINARY_OP

#define FHE_SCALAR_OP(name, type, call)                                            \
  int name(fhe_engine *engine, const fhe_data *a, type value, fhe_data **out) {    \
    REQUIRE_HANDLE(engine);                                                        \
    REQUIRE_HANDLE(a);                                                             \
    REQUIRE_OUT(out);                                                              \
    *out = nullptr;                                                                \
    return guarded(__func__, [&] {                                                           \
      auto &e = *engine->impl;                                                     \
      const Data &x = live(engine, a);                                             \
      *out = wrap(call);                                                           \
    });                                                                            \
  }
FHE_SCALAR_OP(fhe_add_scalar, double, e.add_scalar(x, value))
FHE_SCALAR_OP(fhe_subtract_scalar, double, e.subtract_scalar(x, value))
FHE_SCALAR_OP(fhe_multiply_scalar, double, e.multiply_scalar(x, value))
FHE_SCALAR_OP(fhe_multiply_integer, long long, e.multiply_integer(x, value))
#undef FHE_SCALAR_OP

int fhe_negate(fhe_engine *engine, const fhe_data *ct, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] { *out = wrap(engine->impl->negate(live(engine, ct))); });
}

int fhe_square(fhe_engine *engine, const fhe_data *ct, const fhe_data *rk, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    const Data *key = rk ? &live(engine, rk) : nullptr;
    *out = wrap(engine->impl->square(live(engine, ct), key));
  });
}

}  // extern "C"

extern "C" {

int fhe_create_small_bootstrap_key(fhe_engine *engine, const fhe_data *sk, fhe_data **to_sparse,
                                   fhe_data **to_dense) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(sk);
  REQUIRE_OUT(to_sparse);
  REQUIRE_OUT(to_dense);
  *to_sparse = nullptr;
  *to_dense = nullptr;
  return guarded(__func__, [&] {
    auto keys = engine->impl->create_small_bootstrap_key(live(engine, sk));
    *to_sparse = wrap(std::move(keys.first));
    *to_dense = wrap(std::move(keys.second));
  });
}

int fhe_bootstrap(fhe_engine *engine, const fhe_data *ct, const fhe_data *rk, const fhe_data *ck,
                  const fhe_data *const *rotation_keys, int rotation_key_count,
                  const fhe_data *to_sparse, const fhe_data *to_dense, int stage_count,
                  fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_HANDLE(rk);
  REQUIRE_HANDLE(ck);
  REQUIRE_HANDLE(to_sparse);
  REQUIRE_HANDLE(to_dense);
  REQUIRE_OUT(out);
  *out = nullptr;
  if (rotation_keys == nullptr || rotation_key_count < 1) {
    fhe_b200::set_last_error("Bootstrap Unit Ciphertext With Rotation Key: the rotation key is empty.");
    return FHE_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < rotation_key_count; i++) REQUIRE_HANDLE(rotation_keys[i]);
  return guarded(__func__, [&] {
    std::vector<const Data *> keys;
    for (int i = 0; i < rotation_key_count; i++) keys.push_back(&live(engine, rotation_keys[i]));
    *out = wrap(engine->impl->bootstrap(live(engine, ct), live(engine, rk), live(engine, ck), keys,
                                        live(engine, to_sparse), live(engine, to_dense),
                                        stage_count));
  });
}

// The bootstrap key behind a handle, checked to belong to `engine`.
static const fhe_b200::BootstrapKey &live_key(const fhe_engine *engine,
                                              const fhe_bootstrap_key *key) {
  const Data *part = key->impl->to_sparse.get();
  if (!part || !part->engine) throw std::runtime_error("the engine of the bootstrap key was destroyed.");
  if (engine && part->engine != engine->impl)
    throw std::runtime_error("the bootstrap key is not compatible with this engine.");
  return *key->impl;
}

int fhe_rotate_batch(fhe_engine *engine, const fhe_data *ct, const fhe_data *const *keys,
                     int key_count, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_OUT(keys);
  REQUIRE_OUT(out);
  if (key_count < 1) {
    fhe_b200::set_last_error("Batch Rotate Ciphertext With Fixed Rotation Keys: no keys.");
    return FHE_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < key_count; i++) {
    REQUIRE_HANDLE(keys[i]);
    out[i] = nullptr;
  }
  return guarded(__func__, [&] {
    std::vector<const Data *> ks;
    for (int i = 0; i < key_count; i++) ks.push_back(&live(engine, keys[i]));
    auto r = engine->impl->rotate_batch(live(engine, ct), ks);
    for (int i = 0; i < key_count; i++) out[i] = wrap(std::move(r[i]));
  });
}

int fhe_ntt_tuning_set(int log_n, int s_second, int first_columns_log, int second_tile_log) {
  fhe_b200::NttTuning t;
  t.s_second = s_second;
  t.first_columns_log = first_columns_log;
  t.second_tile_log = second_tile_log;
  if (!fhe_b200::set_ntt_tuning(log_n, t)) {
    fhe_b200::set_last_error("NTT tuning: the shape is not valid for this transform size.");
    return FHE_ERR_INVALID_ARGUMENT;
  }
  fhe_b200::set_last_error("");
  return FHE_OK;
}

int fhe_ntt_tuning_get(int log_n, int *s_second, int *first_columns_log, int *second_tile_log) {
  REQUIRE_OUT(s_second);
  REQUIRE_OUT(first_columns_log);
  REQUIRE_OUT(second_tile_log);
  const fhe_b200::NttTuning t = fhe_b200::ntt_tuning(log_n);
  *s_second = t.s_second;
  *first_columns_log = t.first_columns_log;
  *second_tile_log = t.second_tile_log;
  return FHE_OK;
}

int fhe_engine_set_tensor_cores(fhe_engine *engine, int mode) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->set_tensor_cores(mode); });
}

int fhe_engine_set_tensor_core_wait_limit(fhe_engine *engine, long long limit) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->set_tensor_core_wait_limit(limit); });
}

int fhe_engine_set_graphs(fhe_engine *engine, int enable) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->set_graphs(enable != 0); });
}

int fhe_engine_set_fused_bsgs(fhe_engine *engine, int enable) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->set_fused_bsgs(enable != 0); });
}

int fhe_engine_set_value_transforms(fhe_engine *engine, int enable) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->set_value_transforms(enable != 0); });
}

int fhe_multiply_rotate_batch(fhe_engine *engine, int count, const fhe_data *const *a,
                              const fhe_data *const *b, const fhe_data *relinearization_key,
                              const fhe_data *const *rotation_keys, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(relinearization_key);
  REQUIRE_OUT(a);
  REQUIRE_OUT(b);
  REQUIRE_OUT(rotation_keys);
  REQUIRE_OUT(out);
  if (count < 1) {
    fhe_b200::set_last_error("Multiply Rotate Batch: the batch is empty.");
    return FHE_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < count; i++) {
    REQUIRE_HANDLE(a[i]);
    REQUIRE_HANDLE(b[i]);
    REQUIRE_HANDLE(rotation_keys[i]);
    out[i] = nullptr;
  }
  return guarded(__func__, [&] {
    std::vector<const Data *> va, vb, vk;
    for (int i = 0; i < count; i++) {
      va.push_back(&live(engine, a[i]));
      vb.push_back(&live(engine, b[i]));
      vk.push_back(&live(engine, rotation_keys[i]));
    }
    auto r = engine->impl->multiply_rotate_batch(va, vb, live(engine, relinearization_key), vk);
    for (int i = 0; i < count; i++) out[i] = wrap(std::move(r[i]));
  });
}

int fhe_multiply_relinearize_rescale_batch(fhe_engine *engine, int count,
                                           const fhe_data *const *a, const fhe_data *const *b,
                                           const fhe_data *relinearization_key, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(relinearization_key);
  REQUIRE_OUT(a);
  REQUIRE_OUT(b);
  REQUIRE_OUT(out);
  if (count < 1) {
    fhe_b200::set_last_error("Multiply Relinearize Rescale Batch: the batch is empty.");
    return FHE_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < count; i++) {
    REQUIRE_HANDLE(a[i]);
    REQUIRE_HANDLE(b[i]);
    out[i] = nullptr;
  }
  return guarded(__func__, [&] {
    std::vector<const Data *> va, vb;
    for (int i = 0; i < count; i++) {
      va.push_back(&live(engine, a[i]));
      vb.push_back(&live(engine, b[i]));
    }
    auto r = engine->impl->multiply_relinearize_rescale_batch(va, vb,
                                                              live(engine, relinearization_key));
    for (int i = 0; i < count; i++) out[i] = wrap(std::move(r[i]));
  });
}

int fhe_bootstrap_batch(fhe_engine *engine, int count, const fhe_data *const *cts,
                        const fhe_data *relinearization_key, const fhe_data *conjugation_key,
                        const fhe_bootstrap_key *bootstrap_key, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(relinearization_key);
  REQUIRE_HANDLE(conjugation_key);
  REQUIRE_HANDLE(bootstrap_key);
  REQUIRE_OUT(cts);
  REQUIRE_OUT(out);
  if (count < 1) {
    fhe_b200::set_last_error("Bootstrap Batch: the batch is empty.");
    return FHE_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < count; i++) {
    REQUIRE_HANDLE(cts[i]);
    out[i] = nullptr;
  }
  return guarded(__func__, [&] {
    std::vector<const Data *> v;
    for (int i = 0; i < count; i++) v.push_back(&live(engine, cts[i]));
    auto r = engine->impl->bootstrap_batch(v, live(engine, relinearization_key),
                                           live(engine, conjugation_key),
                                           live_key(engine, bootstrap_key));
    for (int i = 0; i < count; i++) out[i] = wrap(std::move(r[i]));
  });
}

int fhe_engine_set_concurrency(fhe_engine *engine, int streams) {
  REQUIRE_HANDLE(engine);
  return guarded(__func__, [&] { engine->impl->set_concurrency(streams); });
}

int fhe_engine_graph_counts(const fhe_engine *engine, int *captured, int *failed) {
  REQUIRE_HANDLE(engine);
  REQUIRE_OUT(captured);
  REQUIRE_OUT(failed);
  return guarded(__func__, [&] {
    const auto c = engine->impl->graph_counts();
    *captured = c.first;
    *failed = c.second;
  });
}

int fhe_create_bootstrap_key(fhe_engine *engine, const fhe_data *secret_key, int stage_count,
                             const char *size, fhe_bootstrap_key **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(secret_key);
  REQUIRE_OUT(size);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    auto bk = engine->impl->create_bootstrap_key(live(engine, secret_key), stage_count, size);
    auto h = new fhe_bootstrap_key;
    h->impl = bk.release();
    *out = h;
  });
}

int fhe_bootstrap_key_destroy(fhe_bootstrap_key *key) {
  if (!key) return FHE_OK;
  delete key->impl;
  delete key;
  return FHE_OK;
}

int fhe_bootstrap_key_info(const fhe_bootstrap_key *key, int *stage_count, int *inner_loop_shift,
                           int *rotation_key_count, uint64_t *bytes) {
  REQUIRE_HANDLE(key);
  return guarded(__func__, [&] {
    const auto &bk = live_key(nullptr, key);
    if (stage_count) *stage_count = bk.stage_count;
    if (inner_loop_shift) *inner_loop_shift = bk.inner_loop_shift;
    if (rotation_key_count) *rotation_key_count = static_cast<int>(bk.rotation_keys.size());
    if (bytes) *bytes = bk.bytes();
  });
}

int fhe_bootstrap_key_deltas(const fhe_bootstrap_key *key, int *deltas, int capacity, int *count) {
  REQUIRE_HANDLE(key);
  REQUIRE_OUT(count);
  return guarded(__func__, [&] {
    const auto &bk = live_key(nullptr, key);
    int i = 0;
    for (const auto &kv : bk.rotation_keys) {
      if (deltas && i < capacity) deltas[i] = kv.first;
      i++;
    }
    *count = i;
  });
}

int fhe_bootstrap_key_rotation_key(fhe_engine *engine, const fhe_bootstrap_key *key, int delta,
                                   fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(key);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    const auto &bk = live_key(engine, key);
    auto it = bk.rotation_keys.find(delta);
    if (it == bk.rotation_keys.end())
      throw std::invalid_argument("the bootstrap key does not contain a rotation context for delta " +
                                  std::to_string(delta) + ".");
    *out = wrap(engine->impl->clone(*it->second));
  });
}

static const fhe_b200::BootstrapStage &key_stage(const fhe_b200::BootstrapKey &bk, int to_slot,
                                                 int stage) {
  const auto &stages = to_slot ? bk.coeff_to_slot : bk.slot_to_coeff;
  if (stage < 0 || stage >= static_cast<int>(stages.size()))
    throw std::invalid_argument("the stage index is out of range.");
  return stages[stage];
}

int fhe_bootstrap_key_stage(const fhe_bootstrap_key *key, int to_slot, int stage, int *level,
                            int *inner_loop_count, int *outer_loop_count) {
  REQUIRE_HANDLE(key);
  return guarded(__func__, [&] {
    const auto &st = key_stage(live_key(nullptr, key), to_slot, stage);
    if (level) *level = st.level;
    if (inner_loop_count) *inner_loop_count = st.inner;
    if (outer_loop_count) *outer_loop_count = st.outer;
  });
}

int fhe_bootstrap_key_diagonal(fhe_engine *engine, const fhe_bootstrap_key *key, int to_slot,
                               int stage, int outer, int inner, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(key);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    const auto &st = key_stage(live_key(engine, key), to_slot, stage);
    auto row = st.diagonals.find(outer);
    if (row == st.diagonals.end()) return;
    auto entry = row->second.find(inner);
    if (entry == row->second.end()) return;
    *out = wrap(engine->impl->clone(*entry->second));
  });
}

int fhe_bootstrap_key_small(fhe_engine *engine, const fhe_bootstrap_key *key,
                            fhe_data **to_sparse, fhe_data **to_dense) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(key);
  REQUIRE_OUT(to_sparse);
  REQUIRE_OUT(to_dense);
  *to_sparse = nullptr;
  *to_dense = nullptr;
  return guarded(__func__, [&] {
    const auto &bk = live_key(engine, key);
    auto a = engine->impl->clone(*bk.to_sparse);
    auto b = engine->impl->clone(*bk.to_dense);
    *to_sparse = wrap(std::move(a));
    *to_dense = wrap(std::move(b));
  });
}

int fhe_bootstrap_with_key(fhe_engine *engine, const fhe_data *ct,
                           const fhe_data *relinearization_key, const fhe_data *conjugation_key,
                           const fhe_bootstrap_key *bootstrap_key, fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_HANDLE(relinearization_key);
  REQUIRE_HANDLE(conjugation_key);
  REQUIRE_HANDLE(bootstrap_key);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    *out = wrap(engine->impl->bootstrap(live(engine, ct), live(engine, relinearization_key),
                                        live(engine, conjugation_key),
                                        live_key(engine, bootstrap_key)));
  });
}

int fhe_rotate_with_bootstrap_key(fhe_engine *engine, const fhe_data *ct,
                                  const fhe_bootstrap_key *bootstrap_key, int delta,
                                  fhe_data **out) {
  REQUIRE_HANDLE(engine);
  REQUIRE_HANDLE(ct);
  REQUIRE_HANDLE(bootstrap_key);
  REQUIRE_OUT(out);
  *out = nullptr;
  return guarded(__func__, [&] {
    *out = wrap(engine->impl->rotate(live(engine, ct), live_key(engine, bootstrap_key), delta));
  });
}

}  // extern "C"
