/*
 * CPU oracle -- TEST INFRASTRUCTURE ONLY (see ckks_oracle.h).
 *
 * Integer semantics follow the reference exactly: words are int64_t, every
 * comparison is signed, and a product inside REDC is formed from sign-extended
 * 128-bit operands, so that even out-of-range intermediate values (negative
 * differences in a rescale from a large first prime, for instance) evaluate to the
 * same words as the reference produces.
 */
#include "ckks_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef __int128 i128;
typedef unsigned __int128 u128;

#define NBITS 62
#define FB_MASK ((UINT64_C(1) << NBITS) - 1)
#define R_VALUE ((int64_t)1 << NBITS)

/* ---------------------------------------------------------------- scalars -- */

/* guard: montgomery/unit.h:13 */
static inline int64_t guard(int64_t x, int64_t q) { return (x < q) ? x : x - q; }

/* mont_mult_scalar: montgomery/unit.h:15-23 */
int64_t oracle_mont_mult(int64_t x1, int64_t x2, uint64_t q, uint64_t k) {
  const u128 x = (u128)(i128)x1 * (u128)(i128)x2;
  const uint64_t s = ((uint64_t)x * k) & FB_MASK;
  const u128 sq = (u128)s * (u128)q;
  return (int64_t)(uint64_t)((x + sq) >> NBITS);
}

/* mont_exit_scalar: montgomery/unit.h:25-31 */
int64_t oracle_mont_exit(int64_t x, uint64_t q, uint64_t k) {
  const uint64_t s = ((uint64_t)x * k) & FB_MASK;
  const u128 sq = (u128)s * (u128)q;
  return (int64_t)(uint64_t)(((u128)(i128)x + sq) >> NBITS);
}

#define MM oracle_mont_mult

/* ------------------------------------------------------- modular helpers -- */

/* modulus_invert: arithmetic/arithmetic.cpp:9-31 (extended Euclid). */
static int64_t mod_invert(int64_t x, int64_t modulus) {
  int64_t dividend = x, divisor = modulus;
  int64_t dividend_reverse = 1, divisor_reverse = 0;
  while (divisor > 0) {
    int64_t quotient = dividend / divisor;
    int64_t t = dividend;
    dividend = divisor;
    divisor = t - quotient * divisor;
    t = dividend_reverse;
    dividend_reverse = divisor_reverse;
    divisor_reverse = t - quotient * divisor_reverse;
  }
  if (dividend != 1) return 0;
  return dividend_reverse >= 0 ? dividend_reverse : dividend_reverse + modulus;
}

/* modulus_multiply: arithmetic.cpp:33-38 (signed 128-bit remainder). */
static int64_t mod_mul(int64_t a, int64_t b, int64_t m) {
  i128 p = (i128)a * (i128)b;
  p %= (i128)m;
  return (int64_t)p;
}

static int64_t mod_pow(int64_t base, int64_t exponent, int64_t modulus) {
  int64_t current = 1;
  for (; exponent > 0; exponent >>= 1) {
    if (exponent & 1) current = mod_mul(current, base, modulus);
    base = mod_mul(base, base, modulus);
  }
  return current;
}

/* calculate_k with r = 2^62: arithmetic.cpp:159-167, k = -q^{-1} mod 2^62. */
uint64_t oracle_calculate_k(uint64_t q) {
  const int64_t inv = mod_invert(R_VALUE, (int64_t)q);
  i128 k = (i128)R_VALUE * (i128)inv - 1;
  k /= (i128)q;
  return (uint64_t)k;
}

/* find_root: arithmetic.cpp:97-113, first base whose ((q-1)/2N)-th power is a
 * primitive 2N-th root of unity. */
int64_t oracle_find_root(int64_t q, int coeff_count) {
  const int64_t unit_power = (q - 1) / (2 * (int64_t)coeff_count);
  int64_t exp_unit = 0;
  for (int64_t base = 2; base < q; base++) {
    exp_unit = mod_pow(base, unit_power, q);
    if (mod_pow(exp_unit, coeff_count, q) != 1) break;
  }
  return exp_unit;
}

/* reverse_integer_bits: ckks/encode.cpp:11-23 */
static int reverse_bits(int input, int length) {
  int out = 0;
  for (int i = 0; i < length; i++)
    if (input & (1 << i)) out |= 1 << (length - 1 - i);
  return out;
}

/* ------------------------------------------------------------------ NTT -- */

/* ntt: operation/ntt.cpp:46-134.  Cooley-Tukey, natural order in, bit-reversed
 * out, root table consumed stage by stage; every butterfly leaves [0, 2q). */
void oracle_ntt_limb(const int64_t *x, int64_t *y, const int64_t *root,
                     uint64_t q, uint64_t k, int n, int log_n) {
  const int64_t q2 = (int64_t)(q << 1);
  if (x != y) memcpy(y, x, sizeof(int64_t) * n);
  int jump = n;
  for (int s = 0; s < log_n - 1; s++) {
    const int groups = 1 << s;
    jump >>= 1;
    int64_t *a = y;
    for (int g = 0; g < groups; g++) {
      int64_t *b = a + jump;
      const int64_t w = *root++;
      for (int c = 0; c < jump; c++) {
        const int64_t u = a[c];
        const int64_t p = MM(w, b[c], q, k);
        a[c] = guard(u + p, q2);
        b[c] = guard(u + q2 - p, q2);
      }
      a = b + jump;
    }
  }
  for (int c = 0; c < (n >> 1); c++) {
    const int64_t w = *root++;
    const int64_t u = y[2 * c], v = y[2 * c + 1];
    const int64_t p = MM(w, v, q, k);
    y[2 * c] = guard(u + p, q2);
    y[2 * c + 1] = guard(u + q2 - p, q2);
  }
}

/* intt: operation/ntt.cpp:177-272.  Gentleman-Sande, bit-reversed in, natural out. */
void oracle_intt_limb(const int64_t *x, int64_t *y, const int64_t *root_inverse,
                      uint64_t q, uint64_t k, int n, int log_n) {
  const int64_t q2 = (int64_t)(q << 1);
  if (x != y) memcpy(y, x, sizeof(int64_t) * n);
  for (int c = 0; c < (n >> 1); c++) {
    const int64_t w = *root_inverse++;
    const int64_t u = y[2 * c], v = y[2 * c + 1];
    y[2 * c] = guard(u + v, q2);
    y[2 * c + 1] = MM(w, guard(u + q2 - v, q2), q, k);
  }
  int jump = 2;
  for (int s = log_n - 2; s >= 0; s--) {
    const int groups = 1 << s;
    int64_t *a = y;
    for (int g = 0; g < groups; g++) {
      int64_t *b = a + jump;
      const int64_t w = *root_inverse++;
      for (int c = 0; c < jump; c++) {
        const int64_t u = a[c], v = b[c];
        a[c] = guard(u + v, q2);
        b[c] = MM(w, guard(u + q2 - v, q2), q, k);
      }
      a = b + jump;
    }
    jump <<= 1;
  }
}

/* -------------------------------------------------------------- context -- */

struct oracle_ctx {
  int log_n, n;
  int prime_count, special_count, chain_count; /* chain_count: non-special at id 0 */
  uint64_t *q, *k;
  int64_t *r_squared, *n_inverse;
  int64_t *root, *root_inverse;       /* prime_count * (n-1) */
  int64_t *p_product_mult_r;          /* chain_count */
  int64_t **p_inverse_mult_r;         /* [special s][q_index < p_index(s)] */
  int64_t **rescale_scale;            /* [from][to - from - 1] */
};

/* CKKSDerivedParameters: ckks/derived_parameters.cpp:19-50 and
 * get_backward_paint: ckks/precomputed.cpp:15-31. */
static void derive_prime(oracle_ctx *c, int i) {
  const int n = c->n, log_n = c->log_n;
  const uint64_t q = c->q[i];
  const int64_t qi = (int64_t)q;
  c->r_squared[i] = mod_mul(R_VALUE, R_VALUE, qi);
  c->k[i] = oracle_calculate_k(q);
  c->n_inverse[i] = mod_mul(mod_invert(n, qi), R_VALUE, qi);

  const int64_t psi = oracle_find_root(qi, n);
  const int64_t psi_inv = mod_invert(psi, qi);
  int64_t *pw = malloc(sizeof(int64_t) * n), *pwi = malloc(sizeof(int64_t) * n);
  int64_t *sh = malloc(sizeof(int64_t) * n), *shi = malloc(sizeof(int64_t) * n);
  pw[0] = 1;
  pwi[0] = 1;
  for (int j = 1; j < n; j++) {
    pw[j] = mod_mul(pw[j - 1], psi, qi);
    pwi[j] = mod_mul(pwi[j - 1], psi_inv, qi);
  }
  for (int j = 0; j < n; j++) {
    sh[reverse_bits(j, log_n)] = pw[j];
    shi[reverse_bits(j, log_n)] = pwi[j];
  }
  int64_t *root = c->root + (size_t)i * (n - 1);
  int64_t *rinv = c->root_inverse + (size_t)i * (n - 1);
  for (int j = 1; j < n; j++) root[j - 1] = sh[j];
  /* backward paint: groups of size n/2, n/4, ..., 1 with root indices
   * [n/2, n), [n/4, n/2), ..., [1, 2). */
  int o = 0;
  for (int lci = log_n - 1; lci >= 0; lci--) {
    const int groups = 1 << lci;
    for (int g = 0; g < groups; g++) rinv[o++] = shi[groups + g];
  }
  for (int j = 0; j < n - 1; j++) {
    root[j] = MM(root[j], c->r_squared[i], q, c->k[i]);
    rinv[j] = MM(rinv[j], c->r_squared[i], q, c->k[i]);
  }
  free(pw);
  free(pwi);
  free(sh);
  free(shi);
}

oracle_ctx *oracle_ctx_new(int log_n, int prime_count, int special_count,
                           const uint64_t *q) {
  oracle_ctx *c = calloc(1, sizeof(*c));
  c->log_n = log_n;
  c->n = 1 << log_n;
  c->prime_count = prime_count;
  c->special_count = special_count;
  c->chain_count = prime_count - special_count;
  c->q = malloc(sizeof(uint64_t) * prime_count);
  c->k = malloc(sizeof(uint64_t) * prime_count);
  c->r_squared = malloc(sizeof(int64_t) * prime_count);
  c->n_inverse = malloc(sizeof(int64_t) * prime_count);
  c->root = malloc(sizeof(int64_t) * prime_count * (c->n - 1));
  c->root_inverse = malloc(sizeof(int64_t) * prime_count * (c->n - 1));
  memcpy(c->q, q, sizeof(uint64_t) * prime_count);
  for (int i = 0; i < prime_count; i++) {
    int dup = -1;
    for (int j = 0; j < i; j++)
      if (c->q[j] == c->q[i]) dup = j;
    if (dup >= 0) { /* the one-more-level prime repeats a special prime */
      c->k[i] = c->k[dup];
      c->r_squared[i] = c->r_squared[dup];
      c->n_inverse[i] = c->n_inverse[dup];
      memcpy(c->root + (size_t)i * (c->n - 1), c->root + (size_t)dup * (c->n - 1),
             sizeof(int64_t) * (c->n - 1));
      memcpy(c->root_inverse + (size_t)i * (c->n - 1),
             c->root_inverse + (size_t)dup * (c->n - 1), sizeof(int64_t) * (c->n - 1));
    } else {
      derive_prime(c, i);
    }
  }
  /* p_product_mult_r: precomputed.cpp:89-98 */
  const int C = c->chain_count;
  c->p_product_mult_r = malloc(sizeof(int64_t) * (C > 0 ? C : 1));
  for (int qi = 0; qi < C; qi++) {
    int64_t prod = R_VALUE;
    for (int p = C; p < prime_count; p++) prod = mod_mul(prod, (int64_t)c->q[p], (int64_t)c->q[qi]);
    c->p_product_mult_r[qi] = prod;
  }
  /* p_inverse_mult_r: precomputed.cpp:100-112, last special prime first. */
  c->p_inverse_mult_r = malloc(sizeof(int64_t *) * (special_count > 0 ? special_count : 1));
  for (int s = 0; s < special_count; s++) {
    const int p_index = prime_count - 1 - s;
    const int64_t p = (int64_t)c->q[p_index];
    c->p_inverse_mult_r[s] = malloc(sizeof(int64_t) * (p_index > 0 ? p_index : 1));
    for (int qi = 0; qi < p_index; qi++) {
      const int64_t qq = (int64_t)c->q[qi];
      c->p_inverse_mult_r[s][qi] = mod_mul(mod_invert(p, qq), R_VALUE, qq);
    }
  }
  /* rescale_scale: precomputed.cpp:114-126 */
  c->rescale_scale = malloc(sizeof(int64_t *) * prime_count);
  for (int from = 0; from < prime_count - 1; from++) {
    c->rescale_scale[from] = malloc(sizeof(int64_t) * (prime_count - from));
    for (int to = from + 1; to < prime_count; to++) {
      const int64_t qt = (int64_t)c->q[to];
      c->rescale_scale[from][to - from - 1] =
          mod_mul(mod_invert((int64_t)c->q[from], qt), R_VALUE, qt);
    }
  }
  c->rescale_scale[prime_count - 1] = NULL;
  return c;
}

void oracle_ctx_free(oracle_ctx *c) {
  if (!c) return;
  for (int s = 0; s < c->special_count; s++) free(c->p_inverse_mult_r[s]);
  for (int i = 0; i < c->prime_count; i++) free(c->rescale_scale[i]);
  free(c->p_inverse_mult_r);
  free(c->rescale_scale);
  free(c->p_product_mult_r);
  free(c->q);
  free(c->k);
  free(c->r_squared);
  free(c->n_inverse);
  free(c->root);
  free(c->root_inverse);
  free(c);
}

void oracle_ctx_tables(const oracle_ctx *c, uint64_t *k, int64_t *r_squared,
                       int64_t *n_inverse, int64_t *root, int64_t *root_inverse) {
  const size_t P = (size_t)c->prime_count;
  if (k) memcpy(k, c->k, sizeof(uint64_t) * P);
  if (r_squared) memcpy(r_squared, c->r_squared, sizeof(int64_t) * P);
  if (n_inverse) memcpy(n_inverse, c->n_inverse, sizeof(int64_t) * P);
  if (root) memcpy(root, c->root, sizeof(int64_t) * P * (c->n - 1));
  if (root_inverse) memcpy(root_inverse, c->root_inverse, sizeof(int64_t) * P * (c->n - 1));
}

int oracle_chain_count(const oracle_ctx *c, int moduli_id) {
  return c->chain_count - moduli_id;
}

/* get_partition_count_: ckks/parameters.cpp:325-332 */
int oracle_partition_count(const oracle_ctx *c, int moduli_id) {
  const int K = c->special_count;
  return (oracle_chain_count(c, moduli_id) + K - 1) / K;
}

/* ------------------------------------------------------- limb-wise ops -- */

#define LIMB(ptr, j) ((ptr) + (size_t)(j) * n)

/* mont_enter(x, r^2) then ntt: core_ntt.cpp:91-100 */
static void to_ntt_poly(const oracle_ctx *c, int mid, int chains, const int64_t *x, int64_t *y) {
  const int n = c->n;
  for (int j = 0; j < chains; j++) {
    const int p = mid + j;
    const int64_t *xs = LIMB(x, j);
    int64_t *ys = LIMB(y, j);
    for (int t = 0; t < n; t++) ys[t] = MM(xs[t], c->r_squared[p], c->q[p], c->k[p]);
    oracle_ntt_limb(ys, ys, c->root + (size_t)p * (n - 1), c->q[p], c->k[p], n, c->log_n);
  }
}

/* intt then mont_enter_exit(N^-1 R): core_ntt.cpp:131-148, compound.cpp:54-61 */
static void to_intt_poly(const oracle_ctx *c, int mid, int chains, const int64_t *x, int64_t *y) {
  const int n = c->n;
  for (int j = 0; j < chains; j++) {
    const int p = mid + j;
    int64_t *ys = LIMB(y, j);
    oracle_intt_limb(LIMB(x, j), ys, c->root_inverse + (size_t)p * (n - 1), c->q[p], c->k[p],
                     n, c->log_n);
    for (int t = 0; t < n; t++) {
      const int64_t entered = MM(ys[t], c->n_inverse[p], c->q[p], c->k[p]);
      ys[t] = oracle_mont_exit(entered, c->q[p], c->k[p]);
    }
  }
}

void oracle_to_ntt(const oracle_ctx *c, int mid, int chains, int polys, const int64_t *x,
                   int64_t *y) {
  const size_t stride = (size_t)chains * c->n;
  for (int p = 0; p < polys; p++) to_ntt_poly(c, mid, chains, x + p * stride, y + p * stride);
}

void oracle_to_intt(const oracle_ctx *c, int mid, int chains, int polys, const int64_t *x,
                    int64_t *y) {
  const size_t stride = (size_t)chains * c->n;
  for (int p = 0; p < polys; p++) to_intt_poly(c, mid, chains, x + p * stride, y + p * stride);
}

/* CKKSCore::multiply: core.cpp:284-314 */
void oracle_tensor(const oracle_ctx *c, int mid, const int64_t *a, const int64_t *b,
                   int64_t *out) {
  const int n = c->n, L = oracle_chain_count(c, mid);
  const size_t P = (size_t)L * n;
  const int64_t *x0 = a, *x1 = a + P, *y0 = b, *y1 = b + P;
  int64_t *z0 = out, *z1 = out + P, *z2 = out + 2 * P;
  for (int j = 0; j < L; j++) {
    const int p = mid + j;
    const uint64_t q = c->q[p], k = c->k[p];
    const int64_t q2 = (int64_t)(q << 1), qs = (int64_t)q;
    for (int t = 0; t < n; t++) {
      const size_t i = (size_t)j * n + t;
      const int64_t m0 = MM(x0[i], y0[i], q, k);
      const int64_t m1 = MM(x0[i], y1[i], q, k);
      const int64_t m3 = MM(x1[i], y0[i], q, k);
      const int64_t m2 = MM(x1[i], y1[i], q, k);
      z0[i] = m0;
      z1[i] = guard(guard(m1 + m3, q2), qs); /* mont_add_reduce_2q_to_q */
      z2[i] = m2;
    }
  }
}

/* ------------------------------------------------------- key switching -- */

typedef struct {
  int start, size, partition_index;
} partition_t;

/* CKKSParameters::get_partitions: ckks/parameters.cpp:334-360.  Indices are
 * offsets from the ciphertext's moduli id. */
static int make_partitions(const oracle_ctx *c, int mid, int key_mid, partition_t *out) {
  const int K = c->special_count;
  const int L = oracle_chain_count(c, mid);
  const int pc = oracle_partition_count(c, mid);
  int pidx = oracle_partition_count(c, key_mid) - pc;
  int count = 0;
  for (int start = L - pc * K; start < L; start += K, pidx++) {
    const int lo = start > 0 ? start : 0;
    const int hi = (start + K < L) ? start + K : L;
    out[count].start = lo;
    out[count].size = hi - lo;
    out[count].partition_index = pidx;
    count++;
  }
  return count;
}

/* Partition constants: CKKSPrecomputed::make_partition_parameters,
 * precomputed.cpp:326-382.  The big-integer product of the partition's primes is
 * carried as its residue modulo each prime that needs it. */
typedef struct {
  int size;
  int64_t inv_r[16];        /* q_product_inverse_mult_r[ci-1], ci = 1..size-1 */
  int64_t prod_r[16][16];   /* q_product_mult_r[ci-1][mi-ci-1] */
  int64_t *prod_r2;         /* [(size-1)][prime_count(mid)] q_product_mult_r_squared */
} partition_params_t;

static void make_partition_params(const oracle_ctx *c, int mid, const partition_t *pt,
                                  partition_params_t *pp) {
  const int P = c->prime_count - mid; /* prime_count at mid incl. specials */
  const uint64_t *q = c->q + mid;
  const int64_t *r2 = c->r_squared + mid;
  pp->size = pt->size;
  pp->prod_r2 = malloc(sizeof(int64_t) * (size_t)(pt->size > 1 ? pt->size - 1 : 1) * P);
  for (int ci = 1; ci < pt->size; ci++) {
    const int64_t chain_q = (int64_t)q[pt->start + ci];
    /* residue of the product of primes start..start+ci-1 modulo m */
#define PROD_MOD(m)                                                                     \
  ({                                                                                    \
    int64_t acc_ = 1;                                                                   \
    for (int z_ = 0; z_ < ci; z_++) acc_ = mod_mul(acc_, (int64_t)q[pt->start + z_] % (m), (m)); \
    acc_;                                                                               \
  })
    const int64_t qpm = PROD_MOD(chain_q);
    const int64_t inv = mod_invert(qpm, chain_q);
    pp->inv_r[ci - 1] = (chain_q & 1) == 0 ? inv : mod_mul(inv, R_VALUE, chain_q);
    if (ci < pt->size - 1) {
      for (int mi = ci + 1; mi < pt->size; mi++) {
        const int64_t mq = (int64_t)q[pt->start + mi];
        const int64_t v = PROD_MOD(mq);
        pp->prod_r[ci - 1][mi - ci - 1] = (mq & 1) == 0 ? v : mod_mul(v, R_VALUE, mq);
      }
    }
    for (int mi = 0; mi < P; mi++) {
      const int64_t mq = (int64_t)q[mi];
      const int64_t v = PROD_MOD(mq);
      pp->prod_r2[(size_t)(ci - 1) * P + mi] = (mq & 1) == 0 ? v : mod_mul(v, r2[mi], mq);
    }
#undef PROD_MOD
  }
}

/* rns_to_mrs: core_key_switch.cpp:21-56.  x: coefficient-form limbs at mid;
 * y: `size` digit limbs. */
static void rns_to_mrs(const oracle_ctx *c, int mid, const int64_t *x, const partition_t *pt,
                       const partition_params_t *pp, int64_t *y) {
  const int n = c->n;
  for (int ci = 0; ci < pt->size; ci++) memcpy(LIMB(y, ci), LIMB(x, pt->start), sizeof(int64_t) * n);
  for (int ci = 0; ci < pt->size - 1; ci++) {
    const int yo = ci + 1;
    const int xo = pt->start + yo;
    const int pq = mid + xo;
    const uint64_t q = c->q[pq], k = c->k[pq];
    const int64_t q2 = (int64_t)(q << 1), qs = (int64_t)q;
    const int64_t constant = pp->inv_r[ci];
    const int64_t *xs = LIMB(x, xo);
    int64_t *ys = LIMB(y, yo);
    for (int t = 0; t < n; t++) { /* mont_sub_enter_reduce_2q_to_q: compound.cpp:36-43 */
      const int64_t diff = guard(xs[t] + q2 - ys[t], q2);
      ys[t] = guard(MM(diff, constant, q, k), qs);
    }
    if (ci + 2 < pt->size) {
      const int count = pt->size - (ci + 2);
      for (int t2 = 0; t2 < count; t2++) {
        const int pq2 = mid + pt->start + yo + 1 + t2;
        const uint64_t qq = c->q[pq2], kk = c->k[pq2];
        const int64_t qq2 = (int64_t)(qq << 1), qqs = (int64_t)qq;
        const int64_t cst = pp->prod_r[ci][t2];
        int64_t *dst = LIMB(y, yo + 1 + t2);
        for (int t = 0; t < n; t++) /* mont_enter_add_reduce_2q_to_q: compound.cpp:17-24 */
          dst[t] = guard(guard(MM(ys[t], cst, qq, kk) + dst[t], qq2), qqs);
      }
    }
  }
}

/* mod_up (K > 1): core_key_switch.cpp:92-108.  y: prime_count(mid) limbs, NTT form. */
static void mod_up(const oracle_ctx *c, int mid, const int64_t *mrs, const partition_t *pt,
                   const partition_params_t *pp, int64_t *y) {
  const int n = c->n;
  const int P = c->prime_count - mid;
  for (int j = 0; j < P; j++) {
    const int pq = mid + j;
    const uint64_t q = c->q[pq], k = c->k[pq];
    const int64_t q2 = (int64_t)(q << 1);
    int64_t *ys = LIMB(y, j);
    for (int t = 0; t < n; t++) ys[t] = MM(mrs[t], c->r_squared[pq], q, k);
    for (int ci = 0; ci < pt->size - 1; ci++) {
      const int64_t cst = pp->prod_r2[(size_t)ci * P + j];
      const int64_t *d = LIMB(mrs, ci + 1);
      for (int t = 0; t < n; t++) ys[t] = guard(MM(d[t], cst, q, k) + ys[t], q2);
    }
    oracle_ntt_limb(ys, ys, c->root + (size_t)pq * (n - 1), q, k, n, c->log_n);
  }
}

/* mod_up_single (K == 1): core_key_switch.cpp:81-90 */
static void mod_up_single(const oracle_ctx *c, int mid, const int64_t *x, int start, int64_t *y) {
  const int n = c->n;
  const int P = c->prime_count - mid;
  for (int j = 0; j < P; j++) {
    const int pq = mid + j;
    const uint64_t q = c->q[pq], k = c->k[pq];
    int64_t *ys = LIMB(y, j);
    const int64_t *xs = LIMB(x, start);
    for (int t = 0; t < n; t++) ys[t] = MM(xs[t], c->r_squared[pq], q, k);
    oracle_ntt_limb(ys, ys, c->root + (size_t)pq * (n - 1), q, k, n, c->log_n);
  }
}

/* mod_down: core_key_switch.cpp:110-160.  x: prime_count(mid) limbs NTT form
 * (modified); y: chain_count(mid) limbs, canonical coefficient form. */
static void mod_down(const oracle_ctx *c, int mid, int64_t *x, int64_t *y) {
  const int n = c->n;
  int reduced = c->prime_count - mid;
  to_intt_poly(c, mid, reduced, x, x);
  for (int j = 0; j < reduced; j++) {
    const int64_t qs = (int64_t)c->q[mid + j];
    int64_t *xs = LIMB(x, j);
    for (int t = 0; t < n; t++) xs[t] = guard(xs[t], qs);
  }
  for (int s = 0; s < c->special_count; s++) {
    reduced--;
    const int64_t *last = LIMB(x, reduced);
    for (int j = 0; j < reduced; j++) { /* mont_sub_enter: compound.cpp:45-52 */
      const int pq = mid + j;
      const uint64_t q = c->q[pq], k = c->k[pq];
      const int64_t q2 = (int64_t)(q << 1);
      const int64_t cst = c->p_inverse_mult_r[s][pq];
      int64_t *xs = LIMB(x, j);
      for (int t = 0; t < n; t++) xs[t] = MM(guard(xs[t] + q2 - last[t], q2), cst, q, k);
    }
  }
  for (int j = 0; j < reduced; j++) { /* make_unsigned_reduce_2q_to_q: compound.cpp:85-91 */
    const int64_t qs = (int64_t)c->q[mid + j];
    const int64_t *xs = LIMB(x, j);
    int64_t *ys = LIMB(y, j);
    for (int t = 0; t < n; t++) ys[t] = xs[t] < 0 ? xs[t] + qs : guard(xs[t], qs);
  }
}

void oracle_mixed_radix(const oracle_ctx *c, int mid, int key_mid, const int64_t *x, int64_t *out) {
  partition_t parts[64];
  const int pcount = make_partitions(c, mid, key_mid, parts);
  for (int pi = 0; pi < pcount; pi++) {
    partition_params_t pp;
    make_partition_params(c, mid, &parts[pi], &pp);
    rns_to_mrs(c, mid, x, &parts[pi], &pp, out + (size_t)parts[pi].start * c->n);
    free(pp.prod_r2);
  }
}

void oracle_mod_down(const oracle_ctx *c, int mid, const int64_t *x, int64_t *out) {
  const size_t words = (size_t)(c->prime_count - mid) * c->n;
  int64_t *w = malloc(sizeof(int64_t) * words);
  memcpy(w, x, sizeof(int64_t) * words);
  mod_down(c, mid, w, out);
  free(w);
}

/* create_key_switcher (K > 1, core_key_switch.cpp:293-358) and
 * create_key_switcher_single (K == 1, core_key_switch.cpp:225-291). */
void oracle_key_switch(const oracle_ctx *c, int mid, const int64_t *x, int key_mid,
                       const int64_t *key, int64_t *out) {
  const int n = c->n;
  const int P = c->prime_count - mid;
  const int L = oracle_chain_count(c, mid);
  const int key_P = c->prime_count - key_mid;
  const int key_offset = mid - key_mid; /* get_chain_offset(key, mid) */
  partition_t parts[64];
  const int pcount = make_partitions(c, mid, key_mid, parts);
  int64_t *x0 = malloc(sizeof(int64_t) * (size_t)P * n);
  int64_t *x1 = malloc(sizeof(int64_t) * (size_t)P * n);
  int64_t *ext = malloc(sizeof(int64_t) * (size_t)P * n);
  int64_t *mrs = malloc(sizeof(int64_t) * (size_t)c->special_count * n);
  for (int pi = 0; pi < pcount; pi++) {
    const partition_t *pt = &parts[pi];
    if (c->special_count == 1) {
      mod_up_single(c, mid, x, pt->start, ext);
    } else {
      partition_params_t pp;
      make_partition_params(c, mid, pt, &pp);
      rns_to_mrs(c, mid, x, pt, &pp, mrs);
      mod_up(c, mid, mrs, pt, &pp, ext);
      free(pp.prod_r2);
    }
    const int64_t *k0 = key + ((size_t)(pt->partition_index * 2) * key_P + key_offset) * n;
    const int64_t *k1 = key + ((size_t)(pt->partition_index * 2 + 1) * key_P + key_offset) * n;
    for (int j = 0; j < P; j++) {
      const int pq = mid + j;
      const uint64_t q = c->q[pq], k = c->k[pq];
      const int64_t q2 = (int64_t)(q << 1), qs = (int64_t)q;
      for (int t = 0; t < n; t++) {
        const size_t i = (size_t)j * n + t;
        const int64_t a0 = MM(ext[i], k0[i], q, k);
        const int64_t a1 = MM(ext[i], k1[i], q, k);
        if (pi == 0) {
          x0[i] = a0;
          x1[i] = a1;
        } else { /* mont_mult_add then reduce_2q_to_q */
          x0[i] = guard(guard(a0 + x0[i], q2), qs);
          x1[i] = guard(guard(a1 + x1[i], q2), qs);
        }
      }
    }
  }
  mod_down(c, mid, x0, out);
  mod_down(c, mid, x1, out + (size_t)L * n);
  free(x0);
  free(x1);
  free(ext);
  free(mrs);
}

/* CKKSCore::relinearize: core.cpp:713-741 */
void oracle_relinearize(const oracle_ctx *c, int mid, const int64_t *ct, int key_mid,
                        const int64_t *key, int64_t *out) {
  const int n = c->n, L = oracle_chain_count(c, mid);
  const size_t PS = (size_t)L * n;
  int64_t *x2 = malloc(sizeof(int64_t) * PS);
  int64_t *ks = malloc(sizeof(int64_t) * 2 * PS);
  to_intt_poly(c, mid, L, ct, out);
  to_intt_poly(c, mid, L, ct + PS, out + PS);
  to_intt_poly(c, mid, L, ct + 2 * PS, x2);
  oracle_key_switch(c, mid, x2, key_mid, key, ks);
  for (int j = 0; j < L; j++) {
    const int64_t q = (int64_t)c->q[mid + j], q2 = q << 1;
    for (int t = 0; t < n; t++) {
      const size_t i = (size_t)j * n + t;
      out[i] = guard(guard(out[i] + ks[i], q2), q);
      out[PS + i] = guard(guard(out[PS + i] + ks[PS + i], q2), q);
    }
  }
  free(x2);
  free(ks);
}

/* rescale_once_: core_rescale.cpp:5-25 */
void oracle_rescale(const oracle_ctx *c, int mid, int polys, const int64_t *x, int64_t *y) {
  const int n = c->n, L = oracle_chain_count(c, mid);
  const int next = mid + 1, NL = L - 1;
  const uint64_t q_half = c->q[mid] >> 1;
  for (int p = 0; p < polys; p++) {
    const int64_t *xp = x + (size_t)p * L * n;
    int64_t *yp = y + (size_t)p * NL * n;
    const int64_t *x0 = xp;
    for (int j = 0; j < NL; j++) {
      const int pq = next + j;
      const uint64_t q = c->q[pq], k = c->k[pq];
      const int64_t qs = (int64_t)q, q2 = qs << 1;
      const int64_t cst = c->rescale_scale[mid][j];
      const int64_t *xs = LIMB(xp, 1 + j);
      int64_t *ys = LIMB(yp, j);
      for (int t = 0; t < n; t++) {
        /* get_rounder (unit.cpp:67-70): the int64 word meets a uint64 q/2, so the
         * comparison is unsigned and a negative word rounds up. */
        const int64_t rounder = (uint64_t)x0[t] > q_half ? 1 : 0;
        int64_t v = xs[t] - x0[t];                       /* mont_subtract: unit.cpp:58 */
        v = v >= 0 ? v : v + q2;
        v = guard(v, qs);
        v = MM(v, cst, q, k);
        v = guard(v + rounder, q2); /* add_tiled = mont_add */
        ys[t] = guard(v, qs);
      }
    }
  }
}

/* engine.multiply(ct_a, ct_b, rk) then engine.rescale for two fresh ciphertexts
 * at the same level: prepare_for_multiply (engine_multiply.cpp:13-28) rescales
 * and NTTs each input, core multiply tensors, core relinearize, then rescale. */
void oracle_mult_relin_rescale(const oracle_ctx *c, int mid, const int64_t *a,
                               const int64_t *b, int key_mid, const int64_t *key,
                               int64_t *out) {
  const int n = c->n, L = oracle_chain_count(c, mid);
  const int L1 = L - 1;
  const size_t P1 = (size_t)L1 * n;
  int64_t *ra = malloc(sizeof(int64_t) * 2 * P1);
  int64_t *rb = malloc(sizeof(int64_t) * 2 * P1);
  int64_t *t3 = malloc(sizeof(int64_t) * 3 * P1);
  int64_t *rl = malloc(sizeof(int64_t) * 2 * P1);
  oracle_rescale(c, mid, 2, a, ra);
  oracle_rescale(c, mid, 2, b, rb);
  oracle_to_ntt(c, mid + 1, L1, 2, ra, ra);
  oracle_to_ntt(c, mid + 1, L1, 2, rb, rb);
  oracle_tensor(c, mid + 1, ra, rb, t3);
  oracle_relinearize(c, mid + 1, t3, key_mid, key, rl);
  oracle_rescale(c, mid + 1, 2, rl, out);
  free(ra);
  free(rb);
  free(t3);
  free(rl);
}

/* ------------------------------------------------- key switch variants -- */

/* CKKSCore::switch_key: core.cpp:1058-1083.  ct: [2][L][N] coefficient form. */
void oracle_switch_key(const oracle_ctx *c, int mid, const int64_t *ct, int key_mid,
                       const int64_t *key, int64_t *out) {
  const int n = c->n, L = oracle_chain_count(c, mid);
  const size_t PS = (size_t)L * n;
  int64_t *ks = malloc(sizeof(int64_t) * 2 * PS);
  oracle_key_switch(c, mid, ct + PS, key_mid, key, ks);
  for (int j = 0; j < L; j++) {
    const int64_t q = (int64_t)c->q[mid + j], q2 = q << 1;
    for (int t = 0; t < n; t++) {
      const size_t i = (size_t)j * n + t;
      out[i] = guard(guard(ks[i] + ct[i], q2), q);
      out[PS + i] = ks[PS + i];
    }
  }
  free(ks);
}

/* rotate_ with a (permutation, sign) pair: core.cpp:846-868, encode.cpp:567-575 */
static void rotate_coefficients(const oracle_ctx *c, int mid, int polys, const int32_t *perm,
                                const int32_t *sign, const int64_t *x, int64_t *y) {
  const int n = c->n, L = oracle_chain_count(c, mid);
  for (int p = 0; p < polys; p++)
    for (int j = 0; j < L; j++) {
      const int64_t q = (int64_t)c->q[mid + j];
      const int64_t *xs = x + ((size_t)p * L + j) * n;
      int64_t *ys = y + ((size_t)p * L + j) * n;
      for (int t = 0; t < n; t++) ys[perm[t]] = sign[t] * xs[t];
      for (int t = 0; t < n; t++) ys[t] = ys[t] < 0 ? ys[t] + q : guard(ys[t], q);
    }
}

/* CKKSCore::conjugate: core.cpp:1035-1056 (delta -1 permutation of both polys,
 * then a key switch of the permuted c1). */
void oracle_conjugate(const oracle_ctx *c, int mid, const int64_t *ct, int key_mid,
                      const int64_t *key, int64_t *out) {
  const int n = c->n, L = oracle_chain_count(c, mid);
  int32_t *perm = malloc(sizeof(int32_t) * n), *sign = malloc(sizeof(int32_t) * n);
  oracle_permutation_and_sign(perm, sign, n, -1);
  int64_t *conj = malloc(sizeof(int64_t) * 2 * (size_t)L * n);
  rotate_coefficients(c, mid, 2, perm, sign, ct, conj);
  oracle_switch_key(c, mid, conj, key_mid, key, out);
  free(conj);
  free(perm);
  free(sign);
}

/* CKKSCore::rotate(ct, fixed_rotation_key): core.cpp:939-963 with decompose
 * (core_key_switch.cpp:434-466), create_key_switcher_for_rotate (:550-576) and
 * key_switch_mod_down (core.cpp:916-937).  `delta` is the key's normalised step. */
void oracle_rotate(const oracle_ctx *c, int mid, const int64_t *ct, int key_mid,
                   const int64_t *key, int delta, int64_t *out) {
  const int n = c->n;
  const int L = oracle_chain_count(c, mid);
  const int P = c->prime_count - mid;
  const int key_P = c->prime_count - key_mid;
  const int key_offset = mid - key_mid;
  const size_t PS = (size_t)L * n;
  partition_t parts[64];
  /* decompose uses the partitions of (mid, mid); the key product re-indexes them
   * against the key's moduli id (create_key_switcher(decomposed, key), :510-548). */
  const int pcount = make_partitions(c, mid, mid, parts);
  partition_t kparts[64];
  make_partitions(c, mid, key_mid, kparts);
  int64_t *x0 = malloc(sizeof(int64_t) * (size_t)P * n);
  int64_t *x1 = malloc(sizeof(int64_t) * (size_t)P * n);
  int64_t *ext = malloc(sizeof(int64_t) * (size_t)P * n);
  int64_t *mrs = malloc(sizeof(int64_t) * (size_t)c->special_count * n);
  for (int pi = 0; pi < pcount; pi++) {
    const partition_t *pt = &parts[pi];
    if (c->special_count == 1) {
      mod_up_single(c, mid, ct + PS, pt->start, ext);
    } else {
      partition_params_t pp;
      make_partition_params(c, mid, pt, &pp);
      rns_to_mrs(c, mid, ct + PS, pt, &pp, mrs);
      mod_up(c, mid, mrs, pt, &pp, ext);
      free(pp.prod_r2);
    }
    const int kidx = kparts[pi].partition_index;
    const int64_t *k0 = key + ((size_t)(kidx * 2) * key_P + key_offset) * n;
    const int64_t *k1 = key + ((size_t)(kidx * 2 + 1) * key_P + key_offset) * n;
    for (int j = 0; j < P; j++) {
      const int pq = mid + j;
      const uint64_t q = c->q[pq], k = c->k[pq];
      const int64_t q2 = (int64_t)(q << 1), qs = (int64_t)q;
      for (int t = 0; t < n; t++) {
        const size_t i = (size_t)j * n + t;
        const int64_t a0 = MM(ext[i], k0[i], q, k);
        const int64_t a1 = MM(ext[i], k1[i], q, k);
        if (pi == 0) {
          x0[i] = a0;
          x1[i] = a1;
        } else {
          x0[i] = guard(guard(a0 + x0[i], q2), qs);
          x1[i] = guard(guard(a1 + x1[i], q2), qs);
        }
      }
    }
  }
  /* b * P (p_product_mult_r), Montgomery enter, NTT, added to x0 on the L limbs. */
  int64_t *bp = malloc(sizeof(int64_t) * PS);
  for (int j = 0; j < L; j++) {
    const int pq = mid + j;
    const uint64_t q = c->q[pq], k = c->k[pq];
    for (int t = 0; t < n; t++) {
      const size_t i = (size_t)j * n + t;
      bp[i] = MM(MM(ct[i], c->p_product_mult_r[pq], q, k), c->r_squared[pq], q, k);
    }
    oracle_ntt_limb(bp + (size_t)j * n, bp + (size_t)j * n, c->root + (size_t)pq * (n - 1), q, k,
                    n, c->log_n);
    const int64_t q2 = (int64_t)(q << 1), qs = (int64_t)q;
    for (int t = 0; t < n; t++) {
      const size_t i = (size_t)j * n + t;
      x0[i] = guard(guard(x0[i] + bp[i], q2), qs);
    }
  }
  int64_t *md = malloc(sizeof(int64_t) * 2 * PS);
  mod_down(c, mid, x0, md);
  mod_down(c, mid, x1, md + PS);
  int32_t *perm = malloc(sizeof(int32_t) * n), *sign = malloc(sizeof(int32_t) * n);
  oracle_permutation_and_sign(perm, sign, n, delta);
  rotate_coefficients(c, mid, 2, perm, sign, md, out);
  free(perm);
  free(sign);
  free(md);
  free(bp);
  free(x0);
  free(x1);
  free(ext);
  free(mrs);
}

/* ------------------------------------------------------------ rotation -- */

/* get_jump: ckks/encode.cpp:44-56 */
static int32_t get_jump(unsigned shift, int double_size) {
  if (shift == (unsigned)(double_size - 1)) return (int32_t)shift;
  int64_t jump = 1;
  for (int power = 0; power < double_size - (int)shift; power++) {
    jump *= 5;
    jump &= double_size - 1;
  }
  return (int32_t)jump;
}

/* get_permutation_and_sign: ckks/encode.cpp:513-526 */
void oracle_permutation_and_sign(int32_t *permutation, int32_t *sign, int n, int delta) {
  const unsigned long double_size = (unsigned long)n * 2;
  const unsigned long shift = ((unsigned long)(long)delta + double_size) % double_size;
  const int32_t jump = get_jump((unsigned)shift, (int)double_size);
  for (int i = 0; i < n; i++) {
    const unsigned long pi = ((unsigned long)(long)jump * (unsigned long)i) % double_size;
    permutation[i] = (int32_t)(pi % (unsigned long)n);
    sign[i] = ((pi / (unsigned long)n) & 1) ? -1 : 1;
  }
}

/* get_ntt_permutation: ckks/encode.cpp:528-557 */
void oracle_ntt_permutation(int32_t *permutation, int n, int delta) {
  const int mask = n - 1;
  uint32_t p5 = 1, base = 5, e = (uint32_t)delta;
  const uint32_t m2 = (uint32_t)n * 2;
  /* modulus_power<uint32_t>(5, delta, 2N): arithmetic.cpp:40-52 */
  for (; e > 0; e >>= 1) {
    if (e & 1) p5 = (uint32_t)mod_mul(p5, base, m2);
    base = (uint32_t)mod_mul(base, base, m2);
  }
  const uint32_t power_of_five = p5 & (uint32_t)mask;
  const int diff = delta == -1 ? -1 : (int)(((p5 - 1) >> 1) & (uint32_t)mask);
  const int64_t pinv = delta == -1 ? n - 1 : mod_invert(power_of_five, n);
  int32_t *tmp = malloc(sizeof(int32_t) * n);
  int log_n = 0;
  while ((1 << log_n) < n) log_n++;
  for (int i = 0; i < n; i++) {
    const int64_t pi = ((int64_t)n + (i - diff) % n) % n;
    tmp[i] = (int32_t)mod_mul(pi, pinv, n);
  }
  for (int i = 0; i < n; i++) permutation[i] = reverse_bits(tmp[reverse_bits(i, log_n)], log_n);
  free(tmp);
}

/* ----------------------------------------------------------- level down -- */

/* CKKSParameters deviations (ckks/parameters.cpp:60-104), one moduli id per
 * level; out[level] for level 0 .. chain_count-2, as the doubles the precomputed
 * tables keep (precomputed.h:54). */
void oracle_deviations(const oracle_ctx *c, double scale, int one_more_level, double *out) {
  const int full = c->chain_count - 2;
  long double dev[256];
  int count = 0, chain_index = 0;
  for (int level = full; level >= 0; level--) {
    if (level == full || (one_more_level && level == full - 1)) {
      dev[count++] = 1.0L;
    } else {
      const long double qprod = (long double)c->q[chain_index - 1];
      const long double alpha = powl((long double)scale / qprod, 2);
      dev[count] = powl(dev[count - 1], 2) * alpha;
      count++;
    }
    chain_index += 1;
  }
  for (int level = 0; level <= full; level++) out[level] = (double)dev[full - level];
}

/* (round(v) * 2^62) mod q: BigInt::from_double(round(v)) * r_ % q. */
static int64_t round_times_r(double v, uint64_t q) {
  const double r = round(v);
  const unsigned __int128 x = (unsigned __int128)(uint64_t)r << 62;
  return (int64_t)(x % q);
}

/* make_level_down_multiplier (precomputed.cpp:438-462) when !rescaled, else
 * make_level_down_multiplier_after_rescale (:418-436); entries from the source
 * (resp. destination) moduli id to the last scaling prime. Returns the count. */
int oracle_level_down_multiplier(const oracle_ctx *c, double scale, int one_more_level,
                                 int source_level, int destination_level, int rescaled,
                                 int64_t *out) {
  double dev[256];
  oracle_deviations(c, scale, one_more_level, dev);
  const int full = c->chain_count - 2;
  int first;
  double delta;
  if (rescaled) {
    const double diff = dev[destination_level] / sqrt(dev[source_level - 1]);
    delta = scale * diff;
    first = full - destination_level;
  } else {
    const int src_mid = full - source_level;
    const double diff = dev[destination_level] / dev[source_level];
    delta = (one_more_level && src_mid == 0) ? scale * diff : (double)c->q[src_mid] * diff;
    first = src_mid;
  }
  int count = 0;
  for (int i = first; i < c->chain_count; i++) out[count++] = round_times_r(delta, c->q[i]);
  return count;
}

/* CKKSCore::level_down (core.cpp:786-838) for coefficient-form, not rescaled
 * text at src_mid (level src_mid's not-rescaled level), and level_down_after_rescale
 * (core.cpp:743-778) for rescaled text (either form).  x: [polys][chains(src)][N];
 * y: [polys][chains(dst)][N]. */
void oracle_level_down(const oracle_ctx *c, int src_mid, int polys, int rescaled,
                       int dst_mid, const int64_t *multiplier, const int64_t *x, int64_t *y) {
  const int n = c->n;
  const int L = oracle_chain_count(c, src_mid);
  const int DL = oracle_chain_count(c, dst_mid);
  if (rescaled) {
    const int off = dst_mid - src_mid;
    for (int p = 0; p < polys; p++)
      for (int j = 0; j < DL; j++) {
        const int pq = dst_mid + j;
        const uint64_t q = c->q[pq], k = c->k[pq];
        const int64_t *xs = x + ((size_t)p * L + j + off) * n;
        int64_t *ys = y + ((size_t)p * DL + j) * n;
        for (int t = 0; t < n; t++) ys[t] = guard(MM(xs[t], multiplier[j], q, k), (int64_t)q);
      }
    return;
  }
  int64_t *entered = malloc(sizeof(int64_t) * (size_t)polys * L * n);
  int64_t *resc = malloc(sizeof(int64_t) * (size_t)polys * (L - 1) * n);
  for (int p = 0; p < polys; p++)
    for (int j = 0; j < L; j++) {
      const int pq = src_mid + j;
      const uint64_t q = c->q[pq], k = c->k[pq];
      const int64_t *xs = x + ((size_t)p * L + j) * n;
      int64_t *es = entered + ((size_t)p * L + j) * n;
      for (int t = 0; t < n; t++) es[t] = guard(MM(xs[t], multiplier[j], q, k), (int64_t)q);
    }
  oracle_rescale(c, src_mid, polys, entered, resc);
  const int off = dst_mid - (src_mid + 1);
  for (int p = 0; p < polys; p++)
    memcpy(y + (size_t)p * DL * n, resc + ((size_t)p * (L - 1) + off) * n,
           sizeof(int64_t) * (size_t)DL * n);
  free(entered);
  free(resc);
}

/* rotate_intt_form_ (core.cpp:871-880): signed permutation + make_unsigned. */
void oracle_rotate_plain(const oracle_ctx *c, int mid, int polys, int delta, const int64_t *x,
                         int64_t *y) {
  const int n = c->n;
  int32_t *perm = malloc(sizeof(int32_t) * n), *sign = malloc(sizeof(int32_t) * n);
  oracle_permutation_and_sign(perm, sign, n, delta);
  rotate_coefficients(c, mid, polys, perm, sign, x, y);
  free(perm);
  free(sign);
}

/* rotate_ntt_form_ (core.cpp:886-910): y[c] = x[ntt_permutation[c]] per limb. */
void oracle_rotate_plain_ntt(const oracle_ctx *c, int mid, int polys, int delta,
                             const int64_t *x, int64_t *y) {
  const int n = c->n, L = oracle_chain_count(c, mid);
  int32_t *perm = malloc(sizeof(int32_t) * n);
  oracle_ntt_permutation(perm, n, delta);
  for (int p = 0; p < polys; p++)
    for (int j = 0; j < L; j++) {
      const int64_t *xs = x + ((size_t)p * L + j) * n;
      int64_t *ys = y + ((size_t)p * L + j) * n;
      for (int t = 0; t < n; t++) ys[t] = xs[perm[t]];
    }
  free(perm);
}

/* ------------------------------------------------------- encode / decode -- */

typedef struct {
  double re, im;
} cplx;

/* std::complex<double> product as the reference's compiler expands it. */
static cplx cmul_(cplx a, cplx b) {
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}

/* ckks/encode.cpp:25-154: the codec permutations for codec = 2 * slot_count. */
static int32_t jump_of(unsigned shift, int double_size) {
  if (shift == (unsigned)(double_size - 1)) return (int32_t)shift;
  int64_t jump = 1;
  for (int power = 0; power < double_size - (int)shift; power++) {
    jump *= 5;
    jump &= double_size - 1;
  }
  return (int32_t)jump;
}

static void cycles_of(const uint64_t *p, int size, uint64_t *out) {
  char *visited = calloc(size, 1);
  int start = 0, o = 0;
  while (start < size) {
    uint64_t cur = p[start], next = p[cur];
    for (;;) {
      out[o++] = cur;
      visited[cur] = 1;
      cur = next;
      if (visited[next]) break;
      next = p[cur];
    }
    start++;
    while (start < size && visited[start]) start++;
  }
  free(visited);
}

static void codec_permutations(int codec, uint64_t *pre, uint64_t *post) {
  uint64_t *cs = calloc(codec, sizeof(uint64_t)), *fc = calloc(codec, sizeof(uint64_t));
  uint64_t *c1 = calloc(codec, sizeof(uint64_t)), *c2 = calloc(codec, sizeof(uint64_t));
  const int half = codec / 2;
  cs[0] = half - 1;
  for (int i = 1; i < half; i++) cs[i] = i - 1;
  for (int i = half; i < codec - 1; i++) cs[i] = i + 1;
  cs[codec - 1] = half;
  const int double_size = codec * 2;
  const int32_t jump = jump_of(1, double_size);
  int32_t jm = jump;
  for (int i = 0; i < codec; i++) {
    fc[i] = (uint64_t)((jm - 1) >> 1);
    jm = (jm + jump * 2) % double_size;
  }
  cycles_of(fc, codec, c1);
  cycles_of(cs, codec, c2);
  for (int i = 0; i < codec; i++) post[c1[i]] = c2[i];
  for (int i = 0; i < codec; i++) pre[post[i]] = i;
  free(cs);
  free(fc);
  free(c1);
  free(c2);
}

static void bit_reverse_(cplx *y, int size) { /* fft.cpp:56-75 */
  for (int i = 1, j = 0; i < size; i++) {
    int bit = size >> 1;
    while (j & bit) {
      j ^= bit;
      bit >>= 1;
    }
    j ^= bit;
    if (i < j) {
      cplx t = y[i];
      y[i] = y[j];
      y[j] = t;
    }
  }
}

static void fft_(cplx *y, const cplx *tw, int size) { /* fft.cpp:77-102 */
  for (int step = 2, ts = size / 2; step <= size; step <<= 1, ts >>= 1) {
    const int half = step >> 1;
    for (int off = 0; off < size; off += step) {
      int ti = 0;
      for (int d = off; d < off + half; d++) {
        const cplx l = y[d], r = cmul_(tw[ti], y[d + half]);
        y[d].re = l.re + r.re;
        y[d].im = l.im + r.im;
        y[d + half].re = l.re - r.re;
        y[d + half].im = l.im - r.im;
        ti += ts;
      }
    }
  }
}

static const double PI_ = 3.141592653589793;

/* precomputed.cpp:139-215 for one level: scale before the tile, the
 * one-more-level flag and r_mult_scale_after_tile from moduli id *first_mid. */
void oracle_encode_level(const oracle_ctx *c, double scale, int scale_bits, int one_more_level,
                         int level, long double *ckks_scale_out, double *scale_before_tile,
                         int *max_level_flag, int *first_mid, int64_t *r_mult) {
  double dev[256];
  oracle_deviations(c, scale, one_more_level, dev);
  const int full = c->chain_count - 2;
  int mid = full - level;
  int chains = c->prime_count - mid;
  long double ckks = (long double)dev[level] * scale * scale;
  if (one_more_level && mid == 0) ckks = scale * (long double)c->q[0];
  *ckks_scale_out = ckks;
  const uint64_t p0 = c->q[mid];
  const int max_flag = one_more_level && mid == 0 && (ckks >= p0 * scale);
  int64_t log_after = 0;
  if (max_flag) {
    *scale_before_tile = (double)(ckks / p0);
    chains -= 1;
    mid = full - (level - 1);
  } else {
    int e = 0;
    const double m = (double)frexpl(ckks, &e);
    if (e >= scale_bits) {
      *scale_before_tile = m * scale;
      log_after = e - scale_bits;
    } else {
      *scale_before_tile = (double)ckks;
    }
  }
  const int64_t r = (int64_t)1 << 62;
  for (int j = 0; j < chains; j++) {
    const int64_t qj = (int64_t)c->q[mid + j];
    if (max_flag) {
      r_mult[j] = mod_mul(r, (int64_t)p0, qj);
    } else {
      int64_t v = r % qj;
      for (int64_t ls = log_after; ls > 0; ls -= 60)
        v = mod_mul(v, (int64_t)1 << (ls < 60 ? ls : 60), qj);
      r_mult[j] = v;
    }
  }
  *max_level_flag = max_flag;
  *first_mid = mid;
}

static int64_t pmod_(int64_t x, int64_t m) { return (m + x % m) % m; }

/* CKKSCore::encode_polynomial (core_encode.cpp:33-150) for odd moduli.  Writes
 * `limbs` limbs (the plaintext's chain at its level, with or without specials)
 * [limbs][N]; im may be NULL (real input). */
void oracle_encode(const oracle_ctx *c, const double *re, const double *im, int log_slot,
                   double scale_before_tile, int max_level_flag, int first_mid,
                   const int64_t *r_mult, int limbs, int64_t *out) {
  const int n = c->n, slot = 1 << log_slot, codec = 2 * slot, jump = n / codec;
  uint64_t *pre = calloc(codec, sizeof(uint64_t)), *post = calloc(codec, sizeof(uint64_t));
  codec_permutations(codec, pre, post);
  cplx *y = calloc(codec, sizeof(cplx));
  for (int i = 0; i < slot; i++) { /* pre_permute, encode.cpp:156-185 */
    const uint64_t p = pre[i];
    const double r = re[i], m = im ? im[i] : 0.0;
    y[p].re = r;
    y[p].im = m;
    y[codec - p - 1].re = r;
    y[codec - p - 1].im = im ? -m : 0.0;
  }
  bit_reverse_(y, codec);
  cplx *tw = calloc(codec, sizeof(cplx));
  const double unit = -2 * PI_ / codec;
  for (int i = 0; i < codec; i++) {
    const double a = i * unit;
    tw[i].re = cos(a);
    tw[i].im = sin(a);
  }
  fft_(y, tw, codec);
  double *v = calloc(codec, sizeof(double));
  const double step = -PI_ / (codec * 2);
  double max_abs = 0.0;
  for (int i = 0; i < codec; i++) { /* normalize + apply_twister */
    const double a = y[i].re / codec, b = y[i].im / codec;
    const int ri = 2 * i;
    v[i] = (a * cos(ri * step) - b * sin(ri * step)) * scale_before_tile;
    if (fabs(v[i]) > max_abs) max_abs = fabs(v[i]);
  }
  const int offset = max_level_flag ? 1 : 0;
  const int filled = limbs - offset;
  memset(out, 0, sizeof(int64_t) * (size_t)limbs * n);
  for (int j = 0; j < filled; j++) {
    const int pq = first_mid + j;
    const uint64_t q = c->q[pq], k = c->k[pq];
    const int64_t qs = (int64_t)q;
    int64_t *o = out + (size_t)(j + offset) * n;
    for (int i = 0; i < codec; i++) {
      int64_t t;
      if (max_abs > (double)(1UL << 59)) { /* double_to_rns, arithmetic.cpp:242-270 */
        if (fabs(v[i]) < (double)(1L << 62)) {
          t = pmod_((int64_t)(v[i] + 0.5), qs);
        } else {
          int e;
          const double m = frexp(v[i] + 0.5, &e);
          t = pmod_((int64_t)(m * (double)(1L << 52)), qs);
          for (int le = 52; le < e; le++) {
            t <<= 1;
            t %= qs;
          }
        }
      } else { /* llround, then make_unsigned_reduce_2q_to_q */
        const int64_t r = llround(v[i]);
        t = r < 0 ? r + qs : guard(r, qs);
      }
      o[(size_t)i * jump] = MM(t, r_mult[j], q, k);
    }
  }
  free(pre);
  free(post);
  free(y);
  free(tw);
  free(v);
}

/* convert_plaintext_to_double after the rescale loop + decode_ (core_decode.cpp:
 * 77-124): x [limbs][N] coefficient form at mid; output_scale = the plaintext's
 * ckks_scale then; writes slot values (im may be NULL). */
void oracle_decode(const oracle_ctx *c, const int64_t *x, int mid, int limbs, int log_slot,
                   long double output_scale, double *re, double *im) {
  const int n = c->n, slot = 1 << log_slot, codec = 2 * slot, jump = n / codec;
  double *plain = calloc(codec, sizeof(double));
  const int words = (limbs * 61 + 63) / 64 + 2;
  uint64_t *Q = calloc(words, 8), *cof = calloc((size_t)limbs * words, 8);
  uint64_t *acc = calloc(words + 1, 8);
  int64_t *inv = calloc(limbs, sizeof(int64_t));
#define MULW(a, m)                                                  \
  do {                                                              \
    unsigned __int128 cr = 0;                                       \
    for (int w_ = 0; w_ < words; w_++) {                            \
      unsigned __int128 p_ = (unsigned __int128)(a)[w_] * (m) + cr; \
      (a)[w_] = (uint64_t)p_;                                       \
      cr = p_ >> 64;                                                \
    }                                                               \
  } while (0)
  Q[0] = 1;
  for (int j = 0; j < limbs; j++) MULW(Q, c->q[mid + j]);
  for (int j = 0; j < limbs; j++) { /* Q/q_j and (Q/q_j)^-1 mod q_j */
    uint64_t *cj = cof + (size_t)j * words;
    cj[0] = 1;
    const int64_t qj = (int64_t)c->q[mid + j];
    int64_t iv = 1;
    for (int i = 0; i < limbs; i++) {
      if (i == j) continue;
      MULW(cj, c->q[mid + i]);
      iv = mod_mul(iv, mod_invert((int64_t)(c->q[mid + i] % (uint64_t)qj), qj), qj);
    }
    inv[j] = iv;
  }
#undef MULW
  for (int i = 0; i < codec; i++) {
    const size_t pos = (size_t)i * jump;
    if (limbs == 1) { /* make_signed, unsigned q/2 comparison (unit.cpp:36-42) */
      const int64_t v = x[pos];
      const uint64_t q = c->q[mid];
      plain[i] = (double)((uint64_t)v <= (q >> 1) ? v : v - (int64_t)q);
      continue;
    }
    memset(acc, 0, 8 * (words + 1));
    for (int j = 0; j < limbs; j++) {
      const int64_t qj = (int64_t)c->q[mid + j];
      int64_t v = x[(size_t)j * n + pos];
      v = v < 0 ? v + qj : guard(v, qj);
      const int64_t d = mod_mul(v, inv[j], qj);
      unsigned __int128 cr = 0;
      const uint64_t *cj = cof + (size_t)j * words;
      for (int w = 0; w < words; w++) {
        unsigned __int128 s = (unsigned __int128)cj[w] * (uint64_t)d + acc[w] + cr;
        acc[w] = (uint64_t)s;
        cr = s >> 64;
      }
      acc[words] += (uint64_t)cr;
    }
    for (;;) { /* reduce modulo Q */
      int ge = acc[words] != 0;
      if (!ge) {
        ge = 1;
        for (int w = words - 1; w >= 0; w--)
          if (acc[w] != Q[w]) {
            ge = acc[w] > Q[w];
            break;
          }
      }
      if (!ge) break;
      unsigned __int128 br = 0;
      for (int w = 0; w < words; w++) {
        unsigned __int128 d = (unsigned __int128)acc[w] - Q[w] - br;
        acc[w] = (uint64_t)d;
        br = (d >> 64) ? 1 : 0;
      }
      acc[words] -= (uint64_t)br;
    }
    /* centre: X >= floor(Q/2) -> -(Q - X); then BigInt::get_double */
    int neg = 1;
    for (int w = words - 1; w >= 0; w--) {
      const uint64_t h = (Q[w] >> 1) | (w + 1 < words ? Q[w + 1] << 63 : 0);
      if (acc[w] != h) {
        neg = acc[w] > h;
        break;
      }
    }
    if (neg) {
      unsigned __int128 br = 0;
      for (int w = 0; w < words; w++) {
        unsigned __int128 d = (unsigned __int128)Q[w] - acc[w] - br;
        acc[w] = (uint64_t)d;
        br = (d >> 64) ? 1 : 0;
      }
    }
    int top = words - 1;
    while (top > 0 && acc[top] == 0) top--;
    double yv = 0;
    for (int w = 0; w <= top; w++) yv += (double)acc[w] * pow(2.0, 64 * w);
    plain[i] = neg ? -yv : yv;
  }
  /* apply_skewer, bit_reversal_permute, fft with the inverse twiddles,
   * permute_after_ifft */
  cplx *z = calloc(codec, sizeof(cplx)), *tw = calloc(codec, sizeof(cplx));
  const double step = PI_ / (codec * 2);
  for (int i = 0; i < codec; i++) {
    z[i].re = plain[i] * cos(2 * i * step);
    z[i].im = plain[i] * sin(2 * i * step);
  }
  bit_reverse_(z, codec);
  const double unit = -2 * PI_ / codec;
  for (int i = 0; i < codec; i++) {
    const double a = i * unit;
    tw[i].re = cos(a);
    tw[i].im = sin(-a);
  }
  fft_(z, tw, codec);
  uint64_t *pre = calloc(codec, sizeof(uint64_t)), *post = calloc(codec, sizeof(uint64_t));
  codec_permutations(codec, pre, post);
  const double sinv = (double)(1.0 / output_scale);
  for (int i = 0; i < codec; i++) {
    const uint64_t p = post[i];
    if (p < (uint64_t)slot) {
      re[p] = z[i].re * sinv;
      if (im) im[p] = z[i].im * sinv;
    }
  }
  free(plain);
  free(Q);
  free(cof);
  free(acc);
  free(inv);
  free(z);
  free(tw);
  free(pre);
  free(post);
}

/* Engine decode of a coefficient-form plaintext x [limbs][N] at moduli_id (no
 * specials) whose ckks_scale is *scale: the rescale loop of
 * convert_plaintext_to_double (core_decode.cpp:36-54, with get_rescaled_scale =
 * scale / q[moduli_id]), then decode. */
void oracle_decode_plaintext(const oracle_ctx *c, const int64_t *x, int mid, int log_slot,
                             const long double *scale, double engine_scale, double *re,
                             double *im) {
  const int n = c->n;
  int limbs = oracle_chain_count(c, mid);
  int64_t *cur = malloc(sizeof(int64_t) * (size_t)limbs * n);
  memcpy(cur, x, sizeof(int64_t) * (size_t)limbs * n);
  long double s = *scale;
  while (mid <= c->chain_count - 2) {
    const long double next = s / c->q[mid];
    if (next <= engine_scale) break;
    int64_t *y = malloc(sizeof(int64_t) * (size_t)(limbs - 1) * n);
    oracle_rescale(c, mid, 1, cur, y);
    free(cur);
    cur = y;
    s = next;
    mid++;
    limbs--;
  }
  oracle_decode(c, cur, mid, limbs, log_slot, s, re, im);
  free(cur);
}

/* ---------------------------------------------------------------- random -- */

#define ROTL32(x, s) (((x) << (s)) | ((x) >> (32 - (s))))
#define QR_(a, b, c, d)              \
  x[a] += x[b];                      \
  x[d] = ROTL32(x[d] ^ x[a], 16);    \
  x[c] += x[d];                      \
  x[b] = ROTL32(x[b] ^ x[c], 12);    \
  x[a] += x[b];                      \
  x[d] = ROTL32(x[d] ^ x[a], 8);     \
  x[c] += x[d];                      \
  x[b] = ROTL32(x[b] ^ x[c], 7)

/* chacha20 (random.cpp:76-92) for the state (constants, seed[8], counter, nonce[2]). */
void oracle_chacha_block(const uint32_t *seed, const uint32_t *nonce, uint64_t counter,
                         uint32_t *out) {
  uint32_t in[16] = {1634760805u, 857760878u, 2036477234u, 1797285236u};
  for (int i = 0; i < 8; i++) in[4 + i] = seed[i];
  in[12] = (uint32_t)counter;
  in[13] = (uint32_t)(counter >> 32);
  in[14] = nonce[0];
  in[15] = nonce[1];
  uint32_t x[16];
  memcpy(x, in, sizeof x);
  for (int r = 0; r < 10; r++) {
    QR_(0, 4, 8, 12);
    QR_(1, 5, 9, 13);
    QR_(2, 6, 10, 14);
    QR_(3, 7, 11, 15);
    QR_(0, 5, 10, 15);
    QR_(1, 6, 11, 12);
    QR_(2, 7, 8, 13);
    QR_(3, 4, 9, 14);
  }
  for (int i = 0; i < 16; i++) out[i] = x[i] + in[i];
}
#undef QR_
#undef ROTL32

/* rand_int (random.cpp:94-131): count samples from blocks counter0, counter0+1, ... */
void oracle_rand_int(const uint32_t *seed, const uint32_t *nonce, uint64_t counter0, int count,
                     uint64_t max_value, int64_t shift, int64_t *out) {
  uint32_t w[16];
  for (int i = 0; i < count; i++) {
    if (i % 4 == 0) oracle_chacha_block(seed, nonce, counter0 + (uint64_t)(i / 4), w);
    const uint32_t *l = w + 4 * (i % 4);
    const uint64_t x_low = ((uint64_t)l[0] << 32) | l[1];
    const uint64_t x_high = ((uint64_t)l[2] << 32) | l[3];
    const unsigned __int128 t =
        (unsigned __int128)max_value * x_high + (uint64_t)(((unsigned __int128)max_value * x_low) >> 64);
    out[i] = (int64_t)(uint64_t)(t >> 64) + shift;
  }
}

/* discrete_gaussian (random.cpp:133-170) with the CDT tree (low words [size],
 * then high words [size]) of depth `depth`. */
void oracle_discrete_gaussian(const uint32_t *seed, const uint32_t *nonce, uint64_t counter0,
                              int count, const uint64_t *tree, int size, int depth, int64_t *out) {
  uint32_t w[16];
  for (int i = 0; i < count; i++) {
    if (i % 4 == 0) oracle_chacha_block(seed, nonce, counter0 + (uint64_t)(i / 4), w);
    const uint32_t *l = w + 4 * (i % 4);
    const uint64_t x_low = ((uint64_t)l[0] << 32) | l[1];
    uint64_t x_high = ((uint64_t)l[2] << 32) | l[3];
    const int64_t sign = (int64_t)(x_high & 1);
    x_high >>= 1;
    int jump = 1, current = 0, counter = 0;
    for (int d = 0; d < depth; d++) {
      const uint64_t th = tree[counter + current + size], tl = tree[counter + current];
      const int ge = (x_high > th) || (x_high == th && x_low >= tl);
      current = 2 * current + ge;
      counter += jump;
      jump *= 2;
    }
    out[i] = (sign * 2 - 1) * (int64_t)current;
  }
}
