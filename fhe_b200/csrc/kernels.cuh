// Launchers of the engine's device kernels (element-wise families, hybrid key
// switching, rescale).  All pointers are device pointers; objects are laid out
// [poly][limb][N] int64 and limb j of an object at moduli id m is modulo prime m + j.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "modarith.cuh"

namespace fhe_b200 {

// The limbs of a mixed transform (ntt.cuh, kNttMixed) whose words must be the
// reference's: limbs in `mask` of polynomial `poly`.  A multiply followed by
// relinearization reduces every word it returns to [0, q) and reads most of its
// intermediate words only modulo q; what it reads word for word is the first limb of
// each key-switching partition of the tensor's third polynomial (Garner's first
// digit, rns_to_mrs, core_key_switch.cpp:21-56), and so the same limbs of the
// second polynomial of both transformed inputs.
struct ExactLimbs {
  int poly = -1;      // -1: none; kAllExact: every limb of every polynomial
  uint64_t mask = 0;  // limbs below 64
  static constexpr int kAllExact = -2;
  __host__ __device__ bool exact(int p, int limb) const {
    return poly == kAllExact || (p == poly && limb < 64 && ((mask >> limb) & 1) != 0);
  }
};

// Constants of the partitions of one (ciphertext moduli id, key moduli id) pair,
// resident on the device.  Host side: Parameters::partition_constants.
struct DevicePartitions {
  int count = 0;          // dnum
  int max_size = 0;       // max alpha
  unsigned size_mask = 0; // bit a set when some partition has alpha == a
  int extended = 0;       // prime_count(moduli_id): limbs of an extended polynomial
  int max_key_index = 0;  // largest partition_index (host copy)
  int *start = nullptr;   // [count]
  int *size = nullptr;    // [count]
  int *key_index = nullptr;           // [count] partition_index
  int key_index_first[8] = {};        // host copy of key_index[0 .. 7]
  int64_t *inverse_r = nullptr;       // [count][16]
  int64_t *product_r = nullptr;       // [count][16][16]
  int64_t *product_r_squared = nullptr;  // [count][16][extended]
};

// Process-wide count of kernel launches made by this library.
void note_launch(unsigned count = 1);
unsigned long long kernel_launch_count();
// Takes back launches counted while a stream was being captured (nothing ran).
void unnote_launches(unsigned long long count);

struct KeySwitchTables {
  const int64_t *p_inverse_mult_r;  // [K][P] (entry for prime i at [s*P + i])
  const int64_t *rescale_scale;     // [P][P] (entry for from,to at [from*P + to])
  // [P][P][2]: (C, C') per entry of rescale_scale for shoup_mult, C = the plain
  // q_from^-1 mod q_to (rescale_scale R^-1) and C' = floor(C 2^64 / q_to).
  const int64_t *rescale_shoup;
  // [P][P][2]: the rescale and to_ntt's enter as one product, for words that only
  // matter modulo q_to: (C, C') with C = rescale_scale mod q_to (q_from^-1 R, the
  // product of the two multipliers) and C' = floor(C 2^64 / q_to).
  const int64_t *rescale_enter_shoup;
  const int64_t *r_mod;             // [P] R mod q: the rounder's 1 after the enter
  const int64_t *p_product_mult_r;  // [P] P mod q * R (zero for the special primes)
  const int64_t *p_shoup;           // [P][2] (P mod q, floor((P mod q) 2^64 / q))
  int prime_count;
  int special_count;
};

// What the ModDown epilogue does with the divided limbs of each polynomial.
struct EpilogueOps {
  const int64_t *base = nullptr;  // [2][L][N] coefficient-form addend (mont_add_reduce_2q_to_q)
  int base_polys = 0;             // polynomials 0 .. base_polys-1 receive the addend
  bool rescale = false;           // rescale by the first prime of the chain (output L-1 limbs)
  // Signed coefficient permutation applied last (rotate_, core.cpp:846-868):
  // word c goes to index perm[c] when perm[c] >= 0, negated to ~perm[c] otherwise,
  // then make_unsigned_reduce_2q_to_q.
  const int32_t *signed_perm = nullptr;
  int polys = 2;  // polynomials of the accumulator ([polys][L+K][N]) divided
};

// z = tensor of two NTT-form ciphertexts (core.cpp:284-314): z0 = a0 b0,
// z1 = a0 b1 + a1 b0 (reduced to [0,q)), z2 = a1 b1.
cudaError_t launch_tensor(const PrimeTables &t, int n, int limbs, int prime_base,
                          const int64_t *a, const int64_t *b, int64_t *z, cudaStream_t s);

// y = guard(guard(x1 + x2, 2q), q) over polys x limbs (mont_add_reduce_2q_to_q).
cudaError_t launch_add_reduce(const PrimeTables &t, int n, int polys, int limbs, int prime_base,
                              const int64_t *x1, const int64_t *x2, int64_t *y, cudaStream_t s);

// rescale_once_ (core_rescale.cpp:5-25): x [polys][L][N] at moduli id m -> y
// [polys][L-1][N] at m+1.
cudaError_t launch_rescale(const PrimeTables &t, const KeySwitchTables &ks, int n, int polys,
                           int limbs, int moduli_id, const int64_t *x, long long x_poly_stride,
                           int64_t *y, long long y_poly_stride, cudaStream_t s);

// Full relinearize / key switch pipeline pieces ------------------------------

// rns_to_mrs for every partition (core_key_switch.cpp:21-56): x is the
// coefficient-form polynomial at moduli_id (L limbs); digits [L][N] hold partition
// p's alpha digits at limbs [start_p, start_p + alpha_p).
cudaError_t launch_mixed_radix(const PrimeTables &t, const DevicePartitions &dp, int n,
                               int moduli_id, const int64_t *x, int64_t *digits, cudaStream_t s);

// ModUp + NTT of every partition (core_key_switch.cpp:92-108): ext [count][E][N].
// With skip_own, each partition's own limbs [start_p, start_p + alpha_p) of ext
// already hold NTT-form words of the same values (the caller had the input in NTT
// form) and are neither contracted nor transformed.
cudaError_t launch_mod_up_ntt(const PrimeTables &t, const DevicePartitions &dp, int log_n,
                              int moduli_id, const int64_t *digits, int64_t *ext,
                              cudaStream_t s, bool skip_own = false);

// Word offsets of the first 8 key partitions' polynomial-0 rows at the text's
// first limb, ((2 partition_index) key_primes + view_offset) N.
struct KeyRowOffsets {
  long long off[8] = {};
};

// The first two polynomials of a tensor, folded into a relinearization's key inner
// product instead of being added after ModDown: ModDown is linear and P = prod p_s is
// zero modulo every special prime, so ModDown(acc + P d) = ModDown(acc) + d, and a
// relinearization reads its addends (and returns its words) only modulo q.  With
// the NTT-form factors a, b of the product, d0 = a0 b0 and d1 = a0 b1 + a1 b0
// (Montgomery products); acc0 gains a0 (b0 P) and acc1 a0 (b1 P) + a1 (b0 P) inside
// the exact sum before its one REDC, which makes them P d0 and P d1.  Without b, a is
// a three-polynomial text being relinearized and acc gains a0 (P R), a1 (P R), which
// the REDC makes P a0, P a1.
struct TensorAddend {
  const int64_t *a = nullptr;  // [2][limbs][N] NTT form, poly stride a_stride
  const int64_t *b = nullptr;  // [2][limbs][N] NTT form, poly stride b_stride; or null
  long long a_stride = 0;
  long long b_stride = 0;
  const int64_t *p_shoup = nullptr;  // [P][2]: (P mod q, floor((P mod q) 2^64 / q)) by prime
  const int64_t *p_mont = nullptr;   // [P]: P R mod q by prime (KeySwitchTables::p_product_mult_r)
  int limbs = 0;                     // the normal limbs; 0: no addend
};

// Key inner product (core_key_switch.cpp:320-349): acc[2][E][N] = sum over
// partitions of ext_p * (key_{2i}, key_{2i+1}), reference reduction pattern.
// key is [2*dnum_key][key_primes][N]; view_offset = moduli_id - key_moduli_id.
// An addend (up to 8 partitions) adds the tensor's P d0, P d1 on the normal limbs.
cudaError_t launch_key_inner_product(const PrimeTables &t, const DevicePartitions &dp, int n,
                                     int moduli_id, const int64_t *ext, const int64_t *key,
                                     int key_primes, int view_offset, int64_t *acc,
                                     cudaStream_t s, const TensorAddend &addend = TensorAddend{});

// Inverse NTT of both accumulators, then to_intt_ scaling and reduce_2q_to_q
// (mod_down, core_key_switch.cpp:110-121), in place.
cudaError_t launch_mod_down_intt(const PrimeTables &t, int log_n, int moduli_id, int extended,
                                 int64_t *acc, cudaStream_t s, int polys = 2);

// Epilogue of a key switch on (acc0, acc1) = INTT'd extended accumulators:
// the sequential division by the special primes (core_key_switch.cpp:123-160),
// then
//   mode 0: out[p] = ks[p]                                  (key switcher)
//   mode 1: out[p] = add_reduce(base[p], ks[p])             (relinearize)
//   mode 2: as mode 1, then rescale (drops limb 0)          (relinearize+rescale)
// base is [2][L][N] (coefficient form); out is [2][L or L-1][N].
cudaError_t launch_mod_down_epilogue(const PrimeTables &t, const KeySwitchTables &ks, int n,
                                     int moduli_id, int limbs, const int64_t *acc,
                                     const int64_t *base, int mode, int64_t *out,
                                     cudaStream_t s);
// The same epilogue with an explicit list of operations (switch_key adds the base
// to polynomial 0 only, rotate permutes).
cudaError_t launch_mod_down_epilogue_ops(const PrimeTables &t, const KeySwitchTables &ks, int n,
                                         int moduli_id, int limbs, const int64_t *acc,
                                         const EpilogueOps &ops, int64_t *out, cudaStream_t s);

// Constants of the tensor-core ModDown at one moduli id (built by the engine):
// the exact division by the special primes is the linear map
//   v_j = x_j * prod_s pinv_s - sum_s d_s * prod_{t>=s} pinv_t   (mod q_j)
// of the divisor sequence d_s, whose sum runs on the INT8 tensor pipe with 8-bit
// limbs of d_s and of the constants (S32 accumulation, exact).
struct ModDownTcTables {
  const uint8_t *b = nullptr;   // [rounds][128 columns][kb bytes], UMMA K-major core matrices
  const int64_t *c_r = nullptr; // [L] prod_s pinv_s * R mod q_j (x_j's Montgomery factor)
  const int64_t *c_shoup = nullptr;  // [L][2] (C, C'): C = prod_s pinv_s mod q_j, C' = floor(C 2^64 / q_j)
  int rounds = 0;               // ceil(L / 16) MMA rounds of 16 target limbs
  int kb = 0;                   // A row bytes: 9 K rounded up to 32
};

// Where the tensor-core kernels report a bounded wait that ran out, and how long
// their first wait on each MMA round may poll (the wait that drains the MMAs before
// tensor memory is freed always polls for the full limit).
constexpr uint32_t kTcDefaultWaitLimit = 1u << 22;
struct TcStatus {
  int *error = nullptr;                     // set to 1 when a wait ran out (outputs unspecified)
  uint32_t wait_limit = kTcDefaultWaitLimit;  // polls of the mbarrier per MMA round
};

// The epilogue of launch_mod_down_epilogue_ops with the division as an INT8
// tensor-core contraction (tcgen05.mma kind::i8, accumulator in tensor memory).
// Same words as the CUDA-core form.  n must be a multiple of 128; error receives 1
// if a tensor-core wait ran out (the outputs are then unspecified).
cudaError_t launch_mod_down_epilogue_tc(const PrimeTables &t, const KeySwitchTables &ks,
                                        const ModDownTcTables &tc, int n, int moduli_id,
                                        int limbs, const int64_t *acc, const EpilogueOps &ops,
                                        int64_t *out, const TcStatus &status, cudaStream_t s);
// Whether the tensor-core epilogue serves this shape (special primes, limbs, n).
bool mod_down_tc_supported(int special_count, int limbs, int n);
// Host copies of the tables of ModDownTcTables at one moduli id, from the prime
// chain and the p^-1 R constants per division step ([K][prime]).
struct ModDownTcHost {
  std::vector<uint8_t> b;
  std::vector<int64_t> c_r;
  std::vector<int64_t> c_shoup;
  int rounds = 0;
  int kb = 0;
};
ModDownTcHost make_mod_down_tc_tables(const std::vector<uint64_t> &q,
                                      const std::vector<std::vector<int64_t>> &p_inverse_mult_r,
                                      int moduli_id, int limbs, int special_count);

// Constants of the tensor-core ModUp contraction at one moduli id (modup_tc.cu): per
// partition, the bytes of C_ij 2^(8a) mod q_j (i < alpha, byte a < 8, j < extended
// limbs) as the UMMA B operand, 16 targets per MMA round.
struct ModUpTcTables {
  const uint8_t *b = nullptr;           // per partition: [rounds][128 columns][kb bytes]
  const long long *b_offset = nullptr;  // [partitions] byte offset of each partition's B
  int rounds = 0;                       // ceil(extended / 16)
};
struct ModUpTcHost {
  std::vector<uint8_t> b;
  std::vector<long long> b_offset;
  int rounds = 0;
};
struct Partition;
struct PartitionConstants;
bool mod_up_tc_supported(int max_size, int n);
ModUpTcHost make_mod_up_tc_tables(const std::vector<uint64_t> &q,
                                  const std::vector<int64_t> &r_squared, int moduli_id,
                                  int extended, const std::vector<Partition> &parts,
                                  const std::vector<PartitionConstants> &constants);
// ModUp's contraction (core_key_switch.cpp:92-108) of every partition into ext
// [count][extended][N] (coefficient form, before the NTT) with the digit products on
// the INT8 tensor pipe; same words as the CUDA-core contraction.
cudaError_t launch_mod_up_contract_tc(const PrimeTables &t, const DevicePartitions &dp,
                                      const ModUpTcTables &tc, int n, int moduli_id,
                                      const int64_t *digits, int64_t *ext, const TcStatus &status,
                                      cudaStream_t s, bool skip_own = false);
// Tensor-core NTT of the value-only transforms (ntt_tc.cu, N = 2^16): per prime, the
// four byte-split 16 x 16 transform matrices as UMMA B operands and the powers
// psi^e R mod q for e < N in natural order.
struct TcNttTables {
  const uint8_t *bmat = nullptr;     // [P][4][128 columns][128 bytes], core-matrix order
  const int64_t *psi_pow = nullptr;  // [P][N]
};
struct TcNttHost {
  std::vector<uint8_t> bmat;
  std::vector<int64_t> psi_pow;
};
struct Parameters;
bool tc_ntt_supported(int log_n);
TcNttHost make_tc_ntt_tables(const Parameters &p);
// In-place forward (ModUp's) or inverse (ModDown's, with its enter-exit scaling and
// a reduction to [0, q)) transform of polys x limbs limbs ([poly][limb][N], poly
// stride poly_stride) on the INT8 tensor pipe; the values modulo q equal the
// reference's transforms' (forward outputs in [0, 2q)).
cudaError_t launch_tc_ntt(const TcNttTables &tt, const PrimeTables &t, bool inverse, int polys,
                          int limbs, int prime_base, int64_t *data, long long poly_stride,
                          const TcStatus &status, cudaStream_t s);

// The forward NTT that completes ModUp, over every partition's extended limbs (with
// skip_own, not over each partition's own limbs).
cudaError_t launch_extended_ntt(const PrimeTables &t, const DevicePartitions &dp, int log_n,
                                int moduli_id, int64_t *ext, cudaStream_t s,
                                bool skip_own = false);

// Rotation's b * P term (create_key_switcher_for_rotate, core_key_switch.cpp:550-576):
// acc0[j] = reduce(acc0[j] + NTT(mont(mont(c0[j], P mod q * R), R^2))) for the L
// limbs of the ciphertext; `work` holds L limbs of intermediate data.
cudaError_t launch_rotate_base(const PrimeTables &t, const KeySwitchTables &ks, int log_n,
                               int moduli_id, int limbs, const int64_t *c0, int64_t *work,
                               int64_t *acc0, cudaStream_t s);

// rotate_ (core.cpp:846-868): y[perm[c]] = sign[c] * x[c], make_unsigned, over polys x
// limbs, with the signed permutation encoding of EpilogueOps.
cudaError_t launch_permute_signed(const PrimeTables &t, int n, int polys, int limbs,
                                  int prime_base, const int64_t *x, long long x_stride,
                                  const int32_t *signed_perm, int64_t *y, long long y_stride,
                                  cudaStream_t s);
// permute_chain (encode.cpp:575-580): y[c] = x[perm[c]] (NTT-form rotation).
cudaError_t launch_permute_gather(int n, int polys, int limbs, const int64_t *x,
                                  long long x_stride, const int32_t *perm, int64_t *y,
                                  long long y_stride, cudaStream_t s);

// ntt_rotate's tail (core.cpp:965-1000) on extended NTT-form texts of `limbs` limbs:
// y[0][c] = guard(x0[perm[c]] + acc[0][perm[c]], 2q), y[1][c] = acc[1][perm[c]];
// acc and y are [2][limbs][N].
cudaError_t launch_ntt_rotate_finish(const PrimeTables &t, int log_n, int limbs, int prime_base,
                                     const int64_t *x0, const int64_t *acc, const int32_t *perm,
                                     int64_t *y, cudaStream_t s);

// The baby-step sums of the hoisted linear transform (apply_butterfly,
// engine_bootstrap.cpp:248-262) in one pass: for both polynomials of extended
// NTT-form texts, y = the reference's chain over t_i = mont_mult(x_i, d_i) (the
// first term as is, each further one added as add_inplace does,
// reduce(reduce(acc + t_i, 2q), q)); with `accumulate` the chain continues from y.
constexpr int kMaxMacTerms = 32;
struct MacTerms {
  const int64_t *x[kMaxMacTerms];  // 2-polynomial texts, polynomial stride x_stride
  const int64_t *d[kMaxMacTerms];  // 1-polynomial plaintexts
  int count = 0;
};
cudaError_t launch_diagonal_mac(const PrimeTables &t, int log_n, int limbs, int prime_base,
                                const MacTerms &terms, long long x_stride, bool accumulate,
                                int64_t *y, long long y_stride, cudaStream_t s);

// The whole inner loop of the hoisted linear transform (apply_butterfly with a
// bootstrap key, engine_bootstrap.cpp:218-262) in one pass over the extended chain:
// inner text 0 is x itself, inner text i >= 1 is x rotated by inner delta i through
// the decomposition (ntt_rotate: the key inner product with rotation key i, x's
// polynomial 0 added, gathered by perm i), and every outer index g sums its
// diagonal products over the inner texts, i ascending.  Consecutive outer indices
// that share a giant-step delta share an output (their sums added): bit g of
// `lead` marks the first of a run, and out[g] is the run's output.
constexpr int kBsgsMaxInner = 16;
constexpr int kBsgsMaxGroups = 8;
constexpr int kBsgsMaxPartitions = 8;
struct BsgsInner {
  int inner = 0;
  int groups = 0;
  const int32_t *perm[kBsgsMaxInner] = {};  // [N] source position per output position
  const int64_t *key[kBsgsMaxInner] = {};   // rotation key i
  // Words from the key to partition p's polynomial-0 row at the text's first limb,
  // ((2 key partition) key_primes + moduli_id - key_moduli_id) N, and from a
  // polynomial-0 row to its polynomial-1 row, key_primes N.
  int32_t key_off[kBsgsMaxInner][kBsgsMaxPartitions] = {};
  int32_t key_poly[kBsgsMaxInner] = {};
  const int64_t *diag[kBsgsMaxInner][kBsgsMaxGroups] = {};  // [extended][N], or none
  uint32_t mask[kBsgsMaxInner] = {};  // bit g: diag[i][g] present
  uint32_t lead = 0;                  // bit g: outer index g starts an output
  int64_t *out[kBsgsMaxGroups] = {};  // [2][extended][N]
};
// x: [2][extended][N] at poly stride x_stride; decomposed: [partitions][extended][N].
cudaError_t launch_bsgs_inner(const PrimeTables &t, int log_n, int moduli_id, int extended,
                              int partitions, const int64_t *x, long long x_stride,
                              const int64_t *decomposed, const BsgsInner &b, cudaStream_t s);

// Shapes of the two-pass NTT of 2^log_n words (12 <= log_n <= 17): the inner pass
// covers s_second stages, the outer (strided) pass the others; first_columns_log
// sub-transforms share a CTA in the outer pass, 2^second_tile_log words make a CTA
// tile in the inner pass.  The defaults are hand-chosen; fhe_b200/autotune.py
// measures the candidates on the device and the package installs the fastest.
struct NttTuning {
  int s_second = 0;
  int first_columns_log = 0;
  int second_tile_log = 0;
};
constexpr int kNttMaxSmem = 128 * 1024;
NttTuning ntt_tuning(int log_n);
NttTuning ntt_default_tuning(int log_n);
// Installs a tuning for log_n; false (and nothing changes) when it is not valid.
bool set_ntt_tuning(int log_n, const NttTuning &tuning);

// Per-limb Montgomery constants passed by value.
constexpr int kMaxScalarLimbs = 128;
struct LimbScalars {
  int64_t v[kMaxScalarLimbs];
};
// y[p][j] = reduce_2q_to_q(mont(x[p][j + x_limb_offset], s[j])) for j < limbs: the
// mont_enter_scalar_ + reduce_2q_to_q pair of level_down (core.cpp:743-838).
cudaError_t launch_scalar_enter(const PrimeTables &t, int n, int polys, int limbs,
                                int prime_base, const int64_t *x, long long x_stride,
                                int x_limb_offset, const LimbScalars &s, int64_t *y,
                                long long y_stride, cudaStream_t st);

// CKKSCore::multiply(ct, double) (core.cpp:196-229): y [polys][limbs - 1][N] at
// moduli_id + 1 = rescale_once_ of reduce(mont_enter(x, c[limb])) of coefficient-form x.
cudaError_t launch_scalar_rescale(const PrimeTables &t, const KeySwitchTables &ks, int n,
                                  int polys, int limbs, int moduli_id, const LimbScalars &c,
                                  const int64_t *x, long long x_stride, int64_t *y,
                                  long long y_stride, cudaStream_t s);

// Forward NTT with Montgomery enter (to_ntt_) of polys x limbs, in place or not.
cudaError_t launch_to_ntt(const PrimeTables &t, int log_n, int polys, int limbs, int prime_base,
                          const int64_t *x, long long x_stride, int64_t *y, long long y_stride,
                          cudaStream_t s);
// to_ntt_ of the rescale of a coefficient-form text in one pass: x is [polys][limbs +
// 1][N] at src_moduli_id, y is [polys][limbs][N] at src_moduli_id + 1 (NTT form).
// Limbs outside `exact` (all of them exact by default) are transformed value-only: a
// word of the same value modulo q, in [0, 2q).
cudaError_t launch_rescale_to_ntt(const PrimeTables &t, const KeySwitchTables &ks, int log_n,
                                  int polys, int limbs, int src_moduli_id, const int64_t *x,
                                  long long x_stride, int64_t *y, long long y_stride,
                                  cudaStream_t s,
                                  const ExactLimbs &exact = ExactLimbs{ExactLimbs::kAllExact, 0});
// attach_special_prime_chains_ of a coefficient-form text: y [polys][limbs + K][N]
// = to_ntt_ of (x * P on the limbs, zero special limbs); the zero limbs are written
// as zeros (their transform), the others go through one fused NTT.
cudaError_t launch_attach_special_ntt(const PrimeTables &t, const KeySwitchTables &ks, int log_n,
                                      int polys, int limbs, int moduli_id, const int64_t *x,
                                      long long x_stride, int64_t *y, long long y_stride,
                                      cudaStream_t s);
// Inverse NTT with N^-1 enter-exit (to_intt_).
cudaError_t launch_to_intt(const PrimeTables &t, int log_n, int polys, int limbs, int prime_base,
                           const int64_t *x, long long x_stride, int64_t *y, long long y_stride,
                           cudaStream_t s);
// Plain transforms (operation/ntt.cpp ntt/intt on each limb), in place.
cudaError_t launch_ntt_plain(const PrimeTables &t, int log_n, int polys, int limbs,
                             int prime_base, int64_t *x, long long stride, bool inverse,
                             cudaStream_t s);
// Inverse NTT (to_intt_) of the tensor of two NTT-form 2-poly ciphertexts a, b
// without materialising the tensor: y [3][L][N] coefficient form.  With own_ext, the
// NTT-form words of the third polynomial are also written to each partition's own
// limbs of the extended buffer own_ext [count][E][N] (ModUp with skip_own).  Limbs
// outside `exact` are transformed value-only, as in launch_rescale_to_ntt.
// With third_only, y is [1][L][N] and receives the third polynomial alone (its first
// two then go to the key inner product as a TensorAddend), formed by a streaming pass
// before the transform; `exact` names its polynomial as 0.
cudaError_t launch_tensor_to_intt(const PrimeTables &t, int log_n, int limbs, int prime_base,
                                  const int64_t *a, const int64_t *b, int64_t *y,
                                  cudaStream_t s, int64_t *own_ext = nullptr,
                                  const DevicePartitions *dp = nullptr,
                                  const ExactLimbs &exact = ExactLimbs{ExactLimbs::kAllExact, 0},
                                  bool third_only = false);

}  // namespace fhe_b200
