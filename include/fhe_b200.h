/*
 * fhe_b200 -- C ABI of the B200-native CKKS engine.
 *
 * The drop-in boundary for the reference's CKKS hot path (DESILO FHE,
 * open-source variant).  The reference exposes a C++ pure-virtual engine
 * (src/engine/abstract_engine.h:12-299, implemented by CKKSEngine in
 * src/ckks/engine.h:19-897) and no C ABI; every function below replaces one of
 * its members, cited beside it.  Objects live in HBM behind opaque handles; limbs
 * cross the boundary as plain int64 arrays laid out [poly][limb][N] in the
 * reference's own representation (Montgomery domain with R = 2^62 in NTT form,
 * bit-reversed NTT order), so keys and ciphertexts move between the reference and
 * this engine unchanged.
 *
 * Conventions
 *  - Every function returns FHE_OK (0) or a negative fhe_status; the message of
 *    the last failure on the calling thread is fhe_last_error().  The reference
 *    throws std::invalid_argument / std::runtime_error with
 *    "<Function Name>: <reason>" (src/ckks/engine_require.cpp); the same text is
 *    reported here and the exception class maps to FHE_ERR_INVALID_ARGUMENT /
 *    FHE_ERR_RUNTIME.
 *  - Operations return new objects owned by the caller (fhe_data_destroy), as the
 *    reference returns new heap objects the caller deletes.
 *  - Work is queued on the engine's CUDA stream; fhe_data_download and
 *    fhe_engine_synchronize wait for it.  One engine per thread, or external
 *    locking (the reference engine is not thread-safe either).
 *  - No function aborts the process or traps the GPU.
 */
#ifndef FHE_B200_H
#define FHE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fhe_status {
  FHE_OK = 0,
  FHE_ERR_INVALID_ARGUMENT = -1, /* std::invalid_argument in the reference */
  FHE_ERR_RUNTIME = -2,          /* std::runtime_error in the reference */
  FHE_ERR_CUDA = -3,             /* a CUDA call failed */
  FHE_ERR_OUT_OF_MEMORY = -4,
  FHE_ERR_NULL_HANDLE = -5,
  FHE_ERR_UNSUPPORTED = -6
} fhe_status;

/* SchemePreset, src/engine/scheme_preset.h:9-15 */
enum {
  FHE_PRESET_CKKS_40_60_DEFAULT = 1,
  FHE_PRESET_CKKS_54_60_BOOTSTRAP = 2,
  FHE_PRESET_CKKS_40_60_DEFAULT_ENGINE_TEST = 3,
  FHE_PRESET_CKKS_54_60_BOOTSTRAP_ENGINE_TEST = 4
};

/* DataFlag bits, src/data/flag.h:7-13 */
enum {
  FHE_FLAG_NONE = 0,
  FHE_FLAG_COMPLEX = 1,
  FHE_FLAG_NTT_FORM = 2,
  FHE_FLAG_RESCALED = 4,
  FHE_FLAG_SPARSE = 8,
  FHE_FLAG_INCLUDE_SPECIAL = 16
};

/* Object kinds: SecretKey, PublicKey, RelinearizationKey, UnitCiphertext,
 * UnitPlaintext, FixedRotationKey, ConjugationKey, KeySwitchingKey
 * (src/data/data.h:94-300). */
enum {
  FHE_SECRET_KEY = 1,
  FHE_PUBLIC_KEY = 2,
  FHE_RELINEARIZATION_KEY = 3,
  FHE_UNIT_CIPHERTEXT = 4,
  FHE_UNIT_PLAINTEXT = 5,
  FHE_FIXED_ROTATION_KEY = 6,
  FHE_CONJUGATION_KEY = 7,
  FHE_KEY_SWITCHING_KEY = 8
};

typedef struct fhe_engine fhe_engine;
typedef struct fhe_data fhe_data;
/* BootstrapKey (data/bootstrap.h:24-44), resident on the device. */
typedef struct fhe_bootstrap_key fhe_bootstrap_key;

/* CKKSConfig, src/ckks/config.h:11-34 (processor/stream/thread fields have no
 * GPU meaning and are absent). */
typedef struct fhe_config {
  int log_coeff_count;     /* default 14 */
  int log_slot_count;      /* -1: log_coeff_count - 1 */
  int special_prime_count; /* default 1 */
  int max_level;           /* -1: full level */
  int scheme_preset;       /* FHE_PRESET_* */
} fhe_config;

typedef struct fhe_engine_info {
  int coeff_count;         /* N */
  int slot_count;
  int chain_count;         /* non-special primes at moduli id 0 */
  int prime_count;         /* chain_count + special_prime_count */
  int special_prime_count;
  int full_level;
  int max_level;
  int max_key_switching_level;
  int scale_bit_length;
} fhe_engine_info;

typedef struct fhe_data_info {
  int type;       /* FHE_SECRET_KEY ... */
  int flag;       /* FHE_FLAG_* bits */
  int moduli_id;  /* first prime of the object's chain */
  int level;      /* to_level, src/data/data.h:21-32 */
  int polys;      /* polynomial count */
  int chains;     /* limbs per polynomial (with specials when INCLUDE_SPECIAL) */
  int delta;      /* rotation step of a fixed rotation key, else 0 */
  long double ckks_scale;
} fhe_data_info;

/* ---- library / engine ------------------------------------------------------ */

/* Message of the last failure on this thread ("" when none). */
const char *fhe_last_error(void);
/* fhe_config with the reference's defaults (CKKSConfig{}). */
void fhe_config_default(fhe_config *config);

/* create_ckks_engine(CKKSConfig), src/engine/engine.cpp:17-20 (validates the
 * config like CKKSConfig::validate, src/ckks/config.cpp:9-47). */
int fhe_engine_create(const fhe_config *config, fhe_engine **engine);
/* delete engine */
int fhe_engine_destroy(fhe_engine *engine);
/* get_coeff_count/get_slot_count/... , src/ckks/engine.h:505-515 */
int fhe_engine_info_get(const fhe_engine *engine, fhe_engine_info *info);
/* The full moduli chain q_0..q_{P-1} (CKKSParameters::get_moduli(0),
 * src/ckks/parameters.cpp:219-238).  Writes min(capacity, P) values. */
int fhe_engine_moduli(const fhe_engine *engine, uint64_t *moduli, int capacity);
/* CKKSParameters::get_moduli_id(level), src/ckks/parameters.cpp:246-248 */
int fhe_engine_moduli_id(const fhe_engine *engine, int level, int *moduli_id);
/* Wait for all queued work. */
int fhe_engine_synchronize(fhe_engine *engine);
/* Queue subsequent work on a caller-owned cudaStream_t (NULL: the engine's own). */
int fhe_engine_set_stream(fhe_engine *engine, void *cuda_stream);

/* Diagnostics (no reference counterpart; the reference has no tracing).  While
 * profiling is on, each kernel family launched on the engine's stream is timed with
 * CUDA events; the report is "name launches total_ms" lines.  The launch count is
 * the number of kernels this library has launched in the process. */
int fhe_engine_set_profiling(fhe_engine *engine, int enable);
int fhe_engine_profile_report(fhe_engine *engine, char *buffer, int capacity);
int fhe_engine_profile_reset(fhe_engine *engine);
unsigned long long fhe_kernel_launch_count(void);

/* Host-only parameter queries (no GPU needed).  The moduli chain and per-prime
 * tables a config produces: CKKSParameters (src/ckks/parameters.cpp:9-105) and
 * CKKSPrecomputed / CKKSDerivedParameters (src/ckks/precomputed.cpp:33-217,
 * src/ckks/derived_parameters.cpp:19-50).  `moduli` receives up to `capacity`
 * primes; each table pointer may be NULL, and root tables hold
 * prime_count * (N - 1) entries. */
int fhe_parameters_query(const fhe_config *config, fhe_engine_info *info, uint64_t *moduli,
                         int capacity);
int fhe_parameters_tables(const fhe_config *config, uint64_t *k, int64_t *r_squared,
                          int64_t *n_inverse, int64_t *root, int64_t *root_inverse);

/* ---- objects ------------------------------------------------------------------ */

/* Build an object from host limbs [polys][chains][N] (chains implied by
 * moduli_id and FHE_FLAG_INCLUDE_SPECIAL).  Replaces constructing Data
 * (src/data/data.cpp:9-48) around the reference's per-limb arrays.  The copy runs on
 * the engine's upload stream and later work waits for it; from pinned host memory the
 * call returns at once and the copy overlaps kernels already queued. */
int fhe_data_upload(fhe_engine *engine, int type, int flag, int moduli_id, int polys,
                    long double ckks_scale, const int64_t *host_limbs, fhe_data **out);
/* Copy all limbs to host memory [polys][chains][N] (waits for queued work). */
int fhe_data_download(const fhe_data *data, int64_t *host_limbs);
/* Queue the same copy without waiting: it runs on the engine's download stream after
 * the work queued so far, overlapping later kernels (the host buffer should be
 * pinned; completion is observed with fhe_engine_synchronize).  Objects are never
 * modified after they are made, so the copy reads the object's final words. */
int fhe_data_download_async(const fhe_data *data, int64_t *host_limbs);
int fhe_data_info_get(const fhe_data *data, fhe_data_info *info);
/* A wire format for any object (the reference declares Data::write and Bytearray,
 * data/data.h:66 and data/bytearray.h, but defines no format): an 80-byte
 * little-endian header (magic "FHEB200D", format version, the reference's
 * DATA_VERSION, the engine's N, prime counts and a hash of its prime chain, the
 * object's type, flags, moduli id, shape, delta and scale) followed by the limbs
 * [polys][chains][N].  serialize waits for queued work; deserialize rejects objects
 * of an engine with other parameters. */
int fhe_data_serialized_size(const fhe_data *data, uint64_t *size);
int fhe_data_serialize(const fhe_data *data, void *buffer, uint64_t capacity);
int fhe_data_deserialize(fhe_engine *engine, const void *buffer, uint64_t size, fhe_data **out);
/* Set the rotation step carried by a fixed rotation key (FixedRotationKey::delta_). */
int fhe_data_set_delta(fhe_data *data, int delta);
/* Device address of the limbs (valid until fhe_data_destroy). */
int fhe_data_device_pointer(const fhe_data *data, int64_t **device_limbs);
int fhe_data_destroy(fhe_data *data);

/* ---- CKKS operations (engine level, src/ckks/engine.h) ---------------------------- */

/* CKKSEngine::multiply(UnitCiphertext*, UnitCiphertext*), engine_multiply.cpp:40-57:
 * lazy rescale of both inputs (prepare_for_multiply, :13-28), then the tensor. */
int fhe_multiply(fhe_engine *engine, const fhe_data *a, const fhe_data *b, fhe_data **out);
/* CKKSEngine::multiply(ct, ct, RelinearizationKey*), engine_multiply.cpp:132-147 */
int fhe_multiply_relinearize(fhe_engine *engine, const fhe_data *a, const fhe_data *b,
                             const fhe_data *relinearization_key, fhe_data **out);
/* CKKSEngine::relinearize, engine_relinearize.cpp:14-29 */
int fhe_relinearize(fhe_engine *engine, const fhe_data *ct, const fhe_data *relinearization_key,
                    fhe_data **out);
/* CKKSEngine::rescale, engine_rescale.cpp:45-55 */
int fhe_rescale(fhe_engine *engine, const fhe_data *ct, fhe_data **out);
/* engine.multiply(a, b, rk) followed by engine.rescale(.) in one call: the same
 * output words as the two reference calls, with the relinearized intermediate
 * never leaving the chip. */
int fhe_multiply_relinearize_rescale(fhe_engine *engine, const fhe_data *a, const fhe_data *b,
                                     const fhe_data *relinearization_key, fhe_data **out);
/* CKKSEngine::ntt / intt (engine_ntt.cpp:35-42, engine_intt.cpp) */
int fhe_to_ntt(fhe_engine *engine, const fhe_data *text, fhe_data **out);
int fhe_to_intt(fhe_engine *engine, const fhe_data *text, fhe_data **out);

/* CKKSEngine::level_down (engine.h:387-388, engine_level_down.cpp:44-70): the text
 * moved to `level` (level_down_multiplier, then a rescale unless the text was
 * rescaled); form is kept. */
int fhe_level_down(fhe_engine *engine, const fhe_data *text, int level, fhe_data **out);

/* CKKSEngine::rotate(UnitCiphertext*, FixedRotationKey*) (engine.h:341-342,
 * engine_rotate.cpp:52-74).  The key is an object of kind FHE_FIXED_ROTATION_KEY whose
 * delta (fhe_data_set_delta) is the key's normalised rotation step; the result is in
 * coefficient form. */
int fhe_rotate(fhe_engine *engine, const fhe_data *ct, const fhe_data *fixed_rotation_key,
               fhe_data **out);
/* CKKSEngine::rotate(UnitCiphertext*, RotationKey*, int delta, bool) (engine.h:343-345,
 * engine_rotate.cpp:106-139): a RotationKey is the list of its fixed rotation keys;
 * the keys whose delta shares a bit with the normalised delta are applied in list
 * order.  A zero normalised delta returns the coefficient form of the input. */
int fhe_rotate_with_keys(fhe_engine *engine, const fhe_data *ct,
                         const fhe_data *const *fixed_rotation_keys, int key_count, int delta,
                         int normalize_by_slot_count, fhe_data **out);
/* CKKSEngine::rotate(UnitPlaintext*, int) (engine.h:340, engine_rotate.cpp:10-24):
 * keyless rotation of a plaintext in either form. */
int fhe_rotate_plaintext(fhe_engine *engine, const fhe_data *pt, int delta, fhe_data **out);
/* CKKSEngine::conjugate(UnitCiphertext*, ConjugationKey*) (engine.h:334-335,
 * engine_conjugate.cpp:53-73); the key is of kind FHE_CONJUGATION_KEY. */
int fhe_conjugate(fhe_engine *engine, const fhe_data *ct, const fhe_data *conjugation_key,
                  fhe_data **out);
/* CKKSEngine::conjugate(UnitPlaintext*) (engine.h:333, engine_conjugate.cpp:10-24). */
int fhe_conjugate_plaintext(fhe_engine *engine, const fhe_data *pt, fhe_data **out);
/* CKKSEngine::encode_unit (engine.h:50-54, engine_encode.cpp:6-36; CKKSCore::encode,
 * core_encode.cpp:33-150): `count` slot values (im NULL: real input; fewer than the
 * slot count are zero-padded, more are ignored) encoded at `level` into a plaintext
 * in coefficient form.  The FFT, twist and rounding run on the device in IEEE
 * double with the reference's operation order, so the limbs are bit-identical. */
int fhe_encode(fhe_engine *engine, const double *re, const double *im, int count, int level,
               int include_special, fhe_data **out);
/* CKKSEngine::decode_unit / decode_complex_unit_plaintext (engine.h:75-77,
 * engine_decode.cpp:6-19; core_decode.cpp:11-124): slot_count values into re (and
 * im unless NULL).  CRT reconstruction, skew, FFT and permutation run on the device. */
int fhe_decode(fhe_engine *engine, const fhe_data *pt, double *re, double *im);

/* ---- arithmetic (engine_add.cpp, engine_subtract.cpp, engine_multiply.cpp,
 *      engine_negate.cpp): operands are brought to a common level, rescale state and
 *      form first, as the reference's match_form / prepare_for_multiply do ---------- */

/* CKKSEngine::add / subtract(UnitCiphertext*, UnitCiphertext*) (engine.h:158-159,
 * engine_add.cpp:82-104, engine_subtract.cpp:5-30); 2- and 3-polynomial operands. */
int fhe_add(fhe_engine *engine, const fhe_data *a, const fhe_data *b, fhe_data **out);
int fhe_subtract(fhe_engine *engine, const fhe_data *a, const fhe_data *b, fhe_data **out);
/* add(ct, pt) / subtract(ct, pt) / subtract(pt, ct) (engine_add.cpp:221-234,
 * engine_subtract.cpp:91-157). */
int fhe_add_plaintext(fhe_engine *engine, const fhe_data *ct, const fhe_data *pt, fhe_data **out);
int fhe_subtract_plaintext(fhe_engine *engine, const fhe_data *ct, const fhe_data *pt,
                           fhe_data **out);
int fhe_subtract_from_plaintext(fhe_engine *engine, const fhe_data *pt, const fhe_data *ct,
                                fhe_data **out);
/* multiply(ct, pt) (engine_multiply.cpp:210-227): the tensor with a plaintext. */
int fhe_multiply_plaintext(fhe_engine *engine, const fhe_data *ct, const fhe_data *pt,
                           fhe_data **out);
/* add / subtract(ct, double) (engine_add.cpp:518-536, engine_subtract.cpp:319-325). */
int fhe_add_scalar(fhe_engine *engine, const fhe_data *ct, double value, fhe_data **out);
int fhe_subtract_scalar(fhe_engine *engine, const fhe_data *ct, double value, fhe_data **out);
/* multiply(ct, double) with its rescale (engine_multiply.cpp:418-432) and
 * multiply(ct, int64_t) (:443-457). */
int fhe_multiply_scalar(fhe_engine *engine, const fhe_data *ct, double value, fhe_data **out);
int fhe_multiply_integer(fhe_engine *engine, const fhe_data *ct, long long value, fhe_data **out);
/* negate (engine_negate.cpp:5-12); square([relinearization key]) (engine_multiply.cpp:
 * 86-101, 175-188; relinearization_key may be NULL). */
int fhe_negate(fhe_engine *engine, const fhe_data *ct, fhe_data **out);
int fhe_square(fhe_engine *engine, const fhe_data *ct, const fhe_data *relinearization_key,
               fhe_data **out);

/* ---- randomness, keys, encryption ------------------------------------------------ */

/* RandomNumberGenerator(1, N, seed, nonce) (src/random/random_number_generator.cpp:9-55)
 * for the engine's ChaCha20 stream: 8 seed words and 2 nonce bytes; NULL draws them
 * from the system random device.  The block counter restarts at zero.  With the
 * reference engine reseeded the same way, keys and ciphertexts made afterwards by
 * the same sequence of calls are bit-identical. */
int fhe_engine_seed(fhe_engine *engine, const uint32_t *seed, const uint8_t *nonce);
/* CKKSEngine::create_secret_key([level]) (engine.h:23-24, core_key.cpp:9-28);
 * level -1: the maximum level. */
int fhe_create_secret_key(fhe_engine *engine, int level, fhe_data **out);
/* create_secret_key(std::vector<int64_t>&, level) (engine.h:25-26, core_key.cpp:30-50):
 * `count` signed coefficients, zero-padded to N. */
int fhe_create_secret_key_from(fhe_engine *engine, const int64_t *secret, int count, int level,
                               fhe_data **out);
/* create_sparse_secret_key (engine.cpp:41-48, core_key.cpp:52-77): ternary with
 * `hamming_weight` nonzero coefficients (the engine's default is 128). */
int fhe_create_sparse_secret_key(fhe_engine *engine, int hamming_weight, int level,
                                 fhe_data **out);
/* create_public_key(sk[, level]) (engine.h:27-28, core_key.cpp:79-109). */
int fhe_create_public_key(fhe_engine *engine, const fhe_data *secret_key, int level,
                          fhe_data **out);
/* create_relinearization_key(sk[, level]) (engine.h:33-35, core_key.cpp:168-190);
 * level -1: the maximum key-switching level. */
int fhe_create_relinearization_key(fhe_engine *engine, const fhe_data *secret_key, int level,
                                   fhe_data **out);
/* create_fixed_rotation_key(sk, delta[, level, normalize_by_slot_count]) (engine.h:37-42,
 * engine.cpp:98-124, core_key.cpp:229-242). */
int fhe_create_fixed_rotation_key(fhe_engine *engine, const fhe_data *secret_key, int delta,
                                  int level, int normalize_by_slot_count, fhe_data **out);
/* create_rotation_key(sk[, level]) (engine.h:44-45, core_key.cpp:258-268): one fixed
 * rotation key per power of two below N/2, written to keys[0..*count). */
int fhe_create_rotation_keys(fhe_engine *engine, const fhe_data *secret_key, int level,
                             fhe_data **keys, int capacity, int *count);
/* create_conjugation_key(sk[, level]) (engine.h:30-31, core_key.cpp:244-256). */
int fhe_create_conjugation_key(fhe_engine *engine, const fhe_data *secret_key, int level,
                               fhe_data **out);
/* CKKSCore::encrypt(UnitPlaintext*, PublicKey* | SecretKey*) (core.cpp:35-122), as
 * CKKSEngine::encrypt_unit uses it after encoding (engine_encrypt.cpp:104-112). */
int fhe_encrypt(fhe_engine *engine, const fhe_data *plaintext, const fhe_data *key,
                fhe_data **out);
/* CKKSEngine::decrypt_to_unit_plaintext (engine_decrypt.cpp:99-126): a plaintext in
 * coefficient form (fhe_decode gives the slots). */
int fhe_decrypt(fhe_engine *engine, const fhe_data *ciphertext, const fhe_data *secret_key,
                fhe_data **out);

/* ---- bootstrapping ---------------------------------------------------------------- */

/* CKKSEngine::create_small_bootstrap_key (engine.h, engine.cpp:141-160): key switching
 * keys to a sparse secret (Hamming weight 128) at level 0 and back at the maximum
 * key-switching level.  Needs a bootstrapping preset. */
int fhe_create_small_bootstrap_key(fhe_engine *engine, const fhe_data *secret_key,
                                   fhe_data **to_sparse, fhe_data **to_dense);
/* CKKSEngine::rotate_batch(Ciphertext*, std::vector<FixedRotationKey*>)
 * (engine_rotate.cpp:262-300), per unit ciphertext: the input is decomposed once and
 * every fixed key reuses the decomposition (hoisted rotations).  out receives
 * key_count new handles, out[i] rotated by keys[i]. */
int fhe_rotate_batch(fhe_engine *engine, const fhe_data *ct, const fhe_data *const *keys,
                     int key_count, fhe_data **out);
/* CKKSEngine::bootstrap(UnitCiphertext*, RelinearizationKey*, ConjugationKey*,
 * RotationKey*, SmallBootstrapKey*, int stage_count) (engine_bootstrap.cpp:712-754):
 * level down to 0, mod raise, coefficients-to-slots, EvalRound, slots-to-coefficients
 * and the correction, on a coefficient-form ciphertext.  The rotation key is the list
 * of fixed rotation keys fhe_create_rotation_keys made. */
int fhe_bootstrap(fhe_engine *engine, const fhe_data *ct, const fhe_data *relinearization_key,
                  const fhe_data *conjugation_key, const fhe_data *const *rotation_keys,
                  int rotation_key_count, const fhe_data *to_sparse, const fhe_data *to_dense,
                  int stage_count, fhe_data **out);

/* CKKSEngine::create_bootstrap_key(SecretKey*, int stage_count, const std::string &size)
 * (engine.h:47, engine.cpp:162-215): the baby-step giant-step stages of
 * coefficients-to-slots and slots-to-coefficients (every twiddle diagonal encoded with
 * the special primes, rescaled, NTT form), a fixed rotation key per step at the first
 * level that needs it, and the small bootstrap key.  size is "medium" or "large"
 * (inner loop shift 0 or 1, case-insensitive).  Keys are drawn from the engine's
 * random stream in the reference's order. */
int fhe_create_bootstrap_key(fhe_engine *engine, const fhe_data *secret_key, int stage_count,
                             const char *size, fhe_bootstrap_key **out);
/* Releases a bootstrap key (~BootstrapKey, data/bootstrap.cpp). */
int fhe_bootstrap_key_destroy(fhe_bootstrap_key *key);
/* stage_count_, inner_loop_shift_, rotation_contexts_.size() and the device bytes
 * held (BootstrapKey::nbytes).  Any output pointer may be null. */
int fhe_bootstrap_key_info(const fhe_bootstrap_key *key, int *stage_count, int *inner_loop_shift,
                           int *rotation_key_count, uint64_t *bytes);
/* The normalised deltas of the rotation contexts in ascending order; *count gets
 * their number (at most capacity are written). */
int fhe_bootstrap_key_deltas(const fhe_bootstrap_key *key, int *deltas, int capacity, int *count);
/* A copy of the fixed rotation key of a normalised delta (rotation_contexts_[delta]). */
int fhe_bootstrap_key_rotation_key(fhe_engine *engine, const fhe_bootstrap_key *key, int delta,
                                   fhe_data **out);
/* PlainMatrix level_, inner_loop_count_, outer_loop_count_ of a stage (to_slot 1:
 * coefficients-to-slots, 0: slots-to-coefficients). */
int fhe_bootstrap_key_stage(const fhe_bootstrap_key *key, int to_slot, int stage, int *level,
                            int *inner_loop_count, int *outer_loop_count);
/* A copy of encoded_diagonals_[outer][inner] of a stage; *out is null when the stage
 * has no such diagonal. */
int fhe_bootstrap_key_diagonal(fhe_engine *engine, const fhe_bootstrap_key *key, int to_slot,
                               int stage, int outer, int inner, fhe_data **out);
/* Copies of the small bootstrap key's two key switching keys. */
int fhe_bootstrap_key_small(fhe_engine *engine, const fhe_bootstrap_key *key,
                            fhe_data **to_sparse, fhe_data **to_dense);
/* CKKSEngine::bootstrap(UnitCiphertext*, RelinearizationKey*, ConjugationKey*,
 * BootstrapKey*) (engine_bootstrap.cpp:804-838): as fhe_bootstrap, with the hoisted
 * baby-step giant-step transforms of the bootstrap key. */
int fhe_bootstrap_with_key(fhe_engine *engine, const fhe_data *ct,
                           const fhe_data *relinearization_key, const fhe_data *conjugation_key,
                           const fhe_bootstrap_key *bootstrap_key, fhe_data **out);
/* CKKSEngine::rotate(UnitCiphertext*, BootstrapKey*, int delta) (engine_rotate.cpp:
 * 192-206): rotation by a delta (normalised by the slot count) whose fixed key the
 * bootstrap key holds. */
int fhe_rotate_with_bootstrap_key(fhe_engine *engine, const fhe_data *ct,
                                  const fhe_bootstrap_key *bootstrap_key, int delta,
                                  fhe_data **out);

/* CKKSCore::switch_key (core.h, core.cpp:1058-1083): c0 + KS(c1) with a key
 * switching key (FHE_KEY_SWITCHING_KEY); NTT-form input is brought to coefficient
 * form first. */
int fhe_switch_key(fhe_engine *engine, const fhe_data *ct, const fhe_data *key_switching_key,
                   fhe_data **out);

/* Relinearize without allocating (no counterpart in the reference, which has no
 * device memory).  For callers that cannot call cudaMalloc while they run: an
 * application whose own allocator owns the GPU's memory and gives libraries a fixed
 * budget, a real-time loop that cannot take cudaMalloc's implicit device
 * synchronisation or an out-of-memory failure in mid-run, or code running where
 * CUDA allocation calls are not allowed (stream callbacks).  Same words as
 * fhe_relinearize; inputs and output are caller-owned device buffers on the
 * engine's device: ct [3][L][N] in NTT form at moduli_id, the key switching key
 * [key_polys][prime_count(key_moduli_id)][N] at key_moduli_id, out [2][L][N].
 * All temporaries, the partition constants included (computed on the device), come
 * from one fixed 32 MiB device array per GPU, held until the process exits; a call
 * whose temporaries would not fit (N = 2^16 with many limbs) is rejected with
 * FHE_ERR_INVALID_ARGUMENT.  The first call on a device resolves that array's
 * address (cudaGetSymbolAddress) and should come before any stream capture.  All
 * calls share the array and it keeps the last call's contents: calls that overlap
 * on the GPU race and must be serialised by the caller. */
int fhe_relinearize_noalloc(fhe_engine *engine, const int64_t *ct_device, int moduli_id,
                            const int64_t *key_device, int key_moduli_id, int key_polys,
                            int64_t *out_device);

/* ---- B200 options (no reference counterpart) ---------------------------------------- */

/* Selects where the base conversions run (ModUp's digit contraction,
 * core_key_switch.cpp:92-108, and ModDown's exact division by the special primes,
 * :123-160): FHE_TENSOR_CORES_OFF on the CUDA cores, FHE_TENSOR_CORES_ON on the INT8
 * tensor pipe (tcgen05.mma kind::i8) wherever the shape allows it, together with
 * ModUp's forward and ModDown's inverse NTT at N = 2^16 (a radix-16 four-step
 * transform as INT8 contractions), FHE_TENSOR_CORES_AUTO (the default) on the
 * tensor pipe where it measured faster (both base conversions from 4 special
 * primes; the NTTs stay on the CUDA cores).  Every mode gives the same words. */
enum {
  FHE_TENSOR_CORES_OFF = 0,
  FHE_TENSOR_CORES_ON = 1,
  FHE_TENSOR_CORES_AUTO = 2
};
int fhe_engine_set_tensor_cores(fhe_engine *engine, int mode);
/* Diagnostics (no reference counterpart): how many times each tensor-core kernel
 * polls for an MMA round to complete before it gives up (0: at once; negative: the
 * default, about 4 M polls).  A kernel that gives up still waits, with the default
 * limit, for its MMAs to finish before it frees its tensor memory, leaves its
 * outputs unspecified and sets the engine's error flag, which the next
 * fhe_engine_synchronize reports as FHE_ERR_CUDA.  Applies to kernels launched
 * afterwards (a CUDA graph captured earlier keeps its limit). */
int fhe_engine_set_tensor_core_wait_limit(fhe_engine *engine, long long limit);
/* A serving step with no reference counterpart: for every i, multiply a[i] by b[i]
 * with the relinearization key and rescale (fhe_multiply_relinearize_rescale), then
 * rotate the product with rotation_keys[i] (fhe_rotate).  out receives count new
 * handles.  After its first run a batch of the same shapes and keys is replayed as
 * one CUDA graph. */
int fhe_multiply_rotate_batch(fhe_engine *engine, int count, const fhe_data *const *a,
                              const fhe_data *const *b, const fhe_data *relinearization_key,
                              const fhe_data *const *rotation_keys, fhe_data **out);
/* Batches with no reference counterpart: the same words as one call per item
 * (fhe_multiply_relinearize_rescale for every pair a[i], b[i]; fhe_bootstrap_with_key
 * for every cts[i]), the items run concurrently on the engine's worker streams.  out
 * receives count new handles. */
int fhe_multiply_relinearize_rescale_batch(fhe_engine *engine, int count,
                                           const fhe_data *const *a, const fhe_data *const *b,
                                           const fhe_data *relinearization_key, fhe_data **out);
int fhe_bootstrap_batch(fhe_engine *engine, int count, const fhe_data *const *cts,
                        const fhe_data *relinearization_key, const fhe_data *conjugation_key,
                        const fhe_bootstrap_key *bootstrap_key, fhe_data **out);
/* How many streams the items of a batch share (1 to 8, default 4; 1 runs them in
 * order on the engine's stream).  Same words for every count. */
int fhe_engine_set_concurrency(fhe_engine *engine, int streams);
/* CUDA graphs (default on): after one direct run of an input shape,
 * fhe_bootstrap_with_key and fhe_multiply_rotate_batch capture the whole operation
 * once and replay it.  Graphs are not used while profiling.  Same words either way. */
int fhe_engine_set_graphs(fhe_engine *engine, int enable);
/* The inner loop of a bootstrap key's linear transforms (engine_bootstrap.cpp:218-262:
 * the inner rotations through one decomposition and every outer group's diagonal
 * sums) as one fused kernel (default on) or as per-rotation kernels.  Same words
 * either way. */
int fhe_engine_set_fused_bsgs(fhe_engine *engine, int enable);
/* Multiply-then-relinearize (fhe_multiply_relinearize[_rescale] and the batches over
 * them) transforms its rescaled inputs and its tensor value-only on the limbs whose
 * words relinearization reads only modulo q (default on), or every limb with the
 * reference's butterflies.  Same words either way; no reference counterpart. */
int fhe_engine_set_value_transforms(fhe_engine *engine, int enable);
/* The number of captured bootstrap graphs the engine holds, and of input shapes
 * whose capture failed and which therefore run directly. */
int fhe_engine_graph_counts(const fhe_engine *engine, int *captured, int *failed);

/* Shapes of the two-pass NTT of 2^log_n words (12 <= log_n <= 17, process-wide): the
 * contiguous pass covers s_second stages, the strided pass log_n - s_second;
 * 2^first_columns_log sub-transforms share a CTA in the strided pass and
 * 2^second_tile_log words make a CTA tile in the contiguous one.  Every shape gives
 * the same words; fhe_b200/autotune.py measures them on the device and writes the
 * fastest to fhe_b200/ntt_tuning.json, which the Python package installs on load.
 * set returns FHE_ERR_INVALID_ARGUMENT for a shape the kernels cannot run. */
int fhe_ntt_tuning_set(int log_n, int s_second, int first_columns_log, int second_tile_log);
int fhe_ntt_tuning_get(int log_n, int *s_second, int *first_columns_log, int *second_tile_log);

/* ---- processor-level kernels on device limbs (src/processor/single.h) --------------- */

/* SingleProcessor::ntt / intt (single.cpp:420-454) on `polys` x `chains` device limbs
 * at moduli_id, in place, [poly][chain][N] with the given poly stride (words). */
int fhe_ntt_limbs(fhe_engine *engine, int64_t *device_limbs, int moduli_id, int chains,
                  int polys, long long poly_stride, int inverse);
/* SingleProcessor::mont_mult (single.h:27, unit.cpp): y = REDC(a * b) word by word on
 * `polys` x `chains` device limbs at moduli_id ([poly][chain][N], the given stride);
 * y may alias a or b. */
int fhe_mont_mult_limbs(fhe_engine *engine, const int64_t *a, const int64_t *b, int64_t *y,
                        int moduli_id, int chains, int polys, long long poly_stride);

#ifdef __cplusplus
}
#endif

#endif /* FHE_B200_H */
