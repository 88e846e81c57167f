/*
 * CPU oracle for the B200 CKKS engine's parity tests -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference (DESILO FHE, open-source variant) CKKS
 * arithmetic on the hot path: R = 2^62 Montgomery REDC with lazy [0, 2q) ranges,
 * the per-limb negacyclic NTT/iNTT, the derived per-prime tables, tensoring,
 * hybrid key switching (Garner mixed-radix ModUp, key inner product, sequential
 * ModDown), rescale and the slot-rotation permutations.  Each function cites the
 * reference file:line it follows.  Only tests/, __graft_entry__.smoke() and the
 * benchmark's CPU-baseline leg may load this library; the product never does.
 *
 * Pinning: the oracle is checked against the reference's own known-answer tests
 * (test/operation/ntt.cpp, test/montgomery/{unit,compound}.cpp, test/ckks/precomputed/default.cpp)
 * through fixtures in tests/golden/, and against the reference library itself
 * compiled from its sources into oracle/_ref/ (see oracle/Makefile).
 *
 * Layout: a polynomial is [limb][N] int64; a multi-polynomial object is
 * [poly][limb][N].  Limb j of an object at moduli id m is modulo prime q[m + j].
 */
#ifndef CKKS_ORACLE_H
#define CKKS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

/* Scalar kernels (montgomery/unit.h:13-31). */
int64_t oracle_mont_mult(int64_t x1, int64_t x2, uint64_t q, uint64_t k);
int64_t oracle_mont_exit(int64_t x, uint64_t q, uint64_t k);
uint64_t oracle_calculate_k(uint64_t q);
int64_t oracle_find_root(int64_t q, int coeff_count);

/* One-limb transforms with explicit tables (operation/ntt.cpp:46,177). */
void oracle_ntt_limb(const int64_t *x, int64_t *y, const int64_t *root,
                     uint64_t q, uint64_t k, int coeff_count, int log_coeff_count);
void oracle_intt_limb(const int64_t *x, int64_t *y, const int64_t *root_inverse,
                      uint64_t q, uint64_t k, int coeff_count, int log_coeff_count);

/* Context: the full prime chain q[0..prime_count) whose last special_prime_count
 * entries are the special primes.  All derived tables are computed here. */
oracle_ctx *oracle_ctx_new(int log_coeff_count, int prime_count,
                           int special_prime_count, const uint64_t *q);
void oracle_ctx_free(oracle_ctx *ctx);
/* Per-prime tables: k, r^2, N^-1*R, roots (prime_count*(N-1)) and inverse roots. */
void oracle_ctx_tables(const oracle_ctx *ctx, uint64_t *k, int64_t *r_squared,
                       int64_t *n_inverse, int64_t *root, int64_t *root_inverse);
int oracle_chain_count(const oracle_ctx *ctx, int moduli_id);     /* without specials */
int oracle_partition_count(const oracle_ctx *ctx, int moduli_id); /* dnum at moduli_id */

/* to_ntt_ / to_intt_ over `polys` polynomials of `chains` limbs at moduli_id
 * (core_ntt.cpp:91,131).  In place allowed (x == y). */
void oracle_to_ntt(const oracle_ctx *ctx, int moduli_id, int chains, int polys,
                   const int64_t *x, int64_t *y);
void oracle_to_intt(const oracle_ctx *ctx, int moduli_id, int chains, int polys,
                    const int64_t *x, int64_t *y);

/* CKKSCore::multiply tensor (core.cpp:284-314): a, b are [2][L][N] NTT form,
 * out is [3][L][N]. */
void oracle_tensor(const oracle_ctx *ctx, int moduli_id, const int64_t *a,
                   const int64_t *b, int64_t *out);

/* CKKSCore::relinearize (core.cpp:713-741).  ct is [3][L][N] in NTT form at
 * moduli_id; key is [2*dnum_key][prime_count(key_moduli_id)][N] (NTT form) at
 * key_moduli_id; out is [2][L][N] coefficient form. */
void oracle_relinearize(const oracle_ctx *ctx, int moduli_id, const int64_t *ct,
                        int key_moduli_id, const int64_t *key, int64_t *out);

/* rns_to_mrs (core_key_switch.cpp:21-56) of every key-switching partition of the
 * coefficient-form polynomial x (L limbs at moduli_id, partitions for a key at
 * key_moduli_id, K > 1): out[limb] holds the digit of the limb's partition at the
 * limb's position, [L][N]. */
void oracle_mixed_radix(const oracle_ctx *ctx, int moduli_id, int key_moduli_id,
                        const int64_t *x, int64_t *out);

/* mod_down (core_key_switch.cpp:110-160) of one NTT-form polynomial x of
 * prime_count(moduli_id) limbs (copied, not modified); out is its L canonical
 * coefficient-form limbs. */
void oracle_mod_down(const oracle_ctx *ctx, int moduli_id, const int64_t *x, int64_t *out);

/* Key switch of one coefficient-form polynomial x (L limbs at moduli_id) with a
 * key switching key: create_key_switcher_from_intt (core_key_switch.cpp:410);
 * out is [2][L][N]. */
void oracle_key_switch(const oracle_ctx *ctx, int moduli_id, const int64_t *x,
                       int key_moduli_id, const int64_t *key, int64_t *out);

/* CKKSCore::rescale_ on coefficient-form polys (core_rescale.cpp:5-25):
 * x is [polys][L][N] at moduli_id, y is [polys][L-1][N]. */
void oracle_rescale(const oracle_ctx *ctx, int moduli_id, int polys,
                    const int64_t *x, int64_t *y);

/* Engine HMult+relinearize+rescale on two fresh (not rescaled, coefficient form)
 * ciphertexts at the same moduli_id (engine_multiply.cpp:13-28,149;
 * engine_rescale.cpp).  a, b: [2][L][N]; out: [2][L-2][N]. */
void oracle_mult_relin_rescale(const oracle_ctx *ctx, int moduli_id,
                               const int64_t *a, const int64_t *b,
                               int key_moduli_id, const int64_t *key,
                               int64_t *out);

/* CKKSCore::switch_key (core.cpp:1058): ct [2][L][N] coefficient form -> out. */
void oracle_switch_key(const oracle_ctx *ctx, int moduli_id, const int64_t *ct,
                       int key_moduli_id, const int64_t *key, int64_t *out);
/* CKKSCore::conjugate (core.cpp:1035): ct [2][L][N] coefficient form -> out. */
void oracle_conjugate(const oracle_ctx *ctx, int moduli_id, const int64_t *ct,
                      int key_moduli_id, const int64_t *key, int64_t *out);
/* CKKSCore::rotate(ct, fixed key) (core.cpp:939-963); delta = the key's step. */
void oracle_rotate(const oracle_ctx *ctx, int moduli_id, const int64_t *ct,
                   int key_moduli_id, const int64_t *key, int delta, int64_t *out);

/* Rotation permutations (ckks/encode.cpp:513-557). */
void oracle_permutation_and_sign(int32_t *permutation, int32_t *sign,
                                 int coeff_count, int delta);
void oracle_ntt_permutation(int32_t *permutation, int coeff_count, int delta);

/* Level down (core.cpp:743-838) and its multipliers (precomputed.cpp:418-462). */
void oracle_deviations(const oracle_ctx *ctx, double scale, int one_more_level, double *out);
int oracle_level_down_multiplier(const oracle_ctx *ctx, double scale, int one_more_level,
                                 int source_level, int destination_level, int rescaled,
                                 int64_t *out);
void oracle_level_down(const oracle_ctx *ctx, int src_moduli_id, int polys, int rescaled,
                       int dst_moduli_id, const int64_t *multiplier, const int64_t *x,
                       int64_t *y);
/* Keyless rotation of a text (core.cpp:871-910), coefficient and NTT form. */
void oracle_rotate_plain(const oracle_ctx *ctx, int moduli_id, int polys, int delta,
                         const int64_t *x, int64_t *y);
void oracle_rotate_plain_ntt(const oracle_ctx *ctx, int moduli_id, int polys, int delta,
                             const int64_t *x, int64_t *y);

/* Encode / decode (core_encode.cpp:33-150, core_decode.cpp:11-124). */
void oracle_encode_level(const oracle_ctx *ctx, double scale, int scale_bits, int one_more_level,
                         int level, long double *ckks_scale, double *scale_before_tile,
                         int *max_level_flag, int *first_moduli_id, int64_t *r_mult);
void oracle_encode(const oracle_ctx *ctx, const double *re, const double *im, int log_slot,
                   double scale_before_tile, int max_level_flag, int first_moduli_id,
                   const int64_t *r_mult, int limbs, int64_t *out);
void oracle_decode(const oracle_ctx *ctx, const int64_t *x, int moduli_id, int limbs,
                   int log_slot, long double output_scale, double *re, double *im);
void oracle_decode_plaintext(const oracle_ctx *ctx, const int64_t *x, int moduli_id, int log_slot,
                             const long double *scale, double engine_scale, double *re,
                             double *im);

/* ChaCha20 stream and samplers (random.cpp:76-170). */
void oracle_chacha_block(const uint32_t *seed, const uint32_t *nonce, uint64_t counter,
                         uint32_t *out);
void oracle_rand_int(const uint32_t *seed, const uint32_t *nonce, uint64_t counter0, int count,
                     uint64_t max_value, int64_t shift, int64_t *out);
void oracle_discrete_gaussian(const uint32_t *seed, const uint32_t *nonce, uint64_t counter0,
                              int count, const uint64_t *tree, int size, int depth, int64_t *out);

#ifdef __cplusplus
}
#endif

#endif
