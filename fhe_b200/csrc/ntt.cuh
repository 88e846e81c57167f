// Batched negacyclic NTT / inverse NTT for the B200 CKKS engine.
//
// The transform of one limb (N = 2^log_n words) is split into passes.  A pass
// performs S consecutive radix-2 stages on independent sub-transforms of 2^S words
// each: "strided" passes take one word out of every T = 2^(log_n - S) (the early
// forward stages / late inverse stages), "contiguous" passes take 2^S adjacent
// words.  A CTA stages a tile of sub-transforms in shared memory; inside a tile the
// stages are done three at a time in registers (radix-8 rounds), so shared memory
// is touched once per three stages.  The first round of a pass reads global memory
// through a Loader and the last round writes through a Storer, which is where the
// element-wise work before and after a transform (Montgomery enter, N^-1 scaling,
// ModUp digit contraction, key products ...) is fused.
//
// Each butterfly is exactly the reference's (operation/ntt.cpp:46-134 forward,
// Cooley-Tukey with the bit-reversed psi table; 177-272 inverse, Gentleman-Sande
// with the "backward paint" table), so the output words are bit-identical whatever
// the pass split.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "kernels.cuh"
#include "modarith.cuh"

namespace fhe_b200 {

void note_launch(unsigned count);

// Which words a transform must reproduce (template parameter VALUE_ONLY):
//   kNttExact      every butterfly is the reference's, every word identical;
//   kNttValueOnly  only each result's value modulo q matters (Harvey's butterflies
//                  on Shoup twiddles where the words are in range);
//   kNttMixed      value-only except the limbs that NttPass::exact names, which take
//                  the exact butterflies (a CTA transforms one limb, so the choice is
//                  uniform per CTA).
constexpr int kNttExact = 0;
constexpr int kNttValueOnly = 1;
constexpr int kNttMixed = 2;

struct NttPass {
  int log_n;
  int stride_log;  // log2(T); 0 for contiguous passes
  int first;       // forward: first global stage; inverse: first distance exponent
  int columns_log; // log2(sub-transforms per CTA tile)
  int polys;       // batch: polys x limbs, grid.y = limbs * polys (poly fastest)
  int limbs;
  int prime_base;  // prime index of limb 0
  // Optional: polynomial p's limbs [skip_start[p], skip_start[p] + skip_size[p]) are
  // left untouched (ModUp's partitions' own limbs, already in NTT form).
  const int *skip_start = nullptr;
  const int *skip_size = nullptr;
  // A kNttMixed transform keeps the exact butterflies on these limbs only.
  ExactLimbs exact;
};

// Reads word gi of (poly, limb) from a [poly][limb][N] buffer.
struct PlainLoad {
  const int64_t *src;
  long long poly_stride;
  __device__ __forceinline__ int64_t operator()(int poly, int limb, int, int gi, int n) const {
    return src[poly * poly_stride + (long long)limb * n + gi];
  }
};

struct PlainStore {
  int64_t *dst;
  long long poly_stride;
  __device__ __forceinline__ void operator()(int poly, int limb, int, int gi, int n, int64_t v) const {
    dst[poly * poly_stride + (long long)limb * n + gi] = v;
  }
};

// mont_enter by a per-prime constant on the way in: to_ntt_ (core_ntt.cpp:91-100).
struct EnterLoad {
  const int64_t *src;
  long long poly_stride;
  const int64_t *constant;  // indexed by prime
  const uint64_t *q;
  const uint64_t *k;
  __device__ __forceinline__ int64_t operator()(int poly, int limb, int prime, int gi, int n) const {
    const int64_t x = src[poly * poly_stride + (long long)limb * n + gi];
    return mont_mult_lazy(x, constant[prime], q[prime], k[prime]);
  }
};

// rescale_once_ (core_rescale.cpp:5-25) and to_ntt_'s enter on the way in: limb
// `limb` of the rescaled text is made from limbs limb + 1 and 0 of the source, whose
// first prime is prime - limb - 1 (the rounder compares unsigned, as get_rounder).
//
// MIXED: the limbs outside `exact` only matter modulo q.  Their word is
// ((x_j - x_0) q_0^-1 + rounder) R mod q, the value of the two steps, formed as one
// Shoup product of the difference by q_0^-1 R plus the rounder's R, in [0, 2q); a
// difference still negative after adding 2q (words far out of range) takes the
// exact steps, whose value is the same.
template <bool MIXED = false>
struct RescaleEnterLoad {
  const int64_t *src;             // [poly][limbs + 1][N]
  long long poly_stride;
  const int64_t *rescale_scale;   // the dropped prime's row, indexed by prime
  const int64_t *rescale_shoup;   // the same row's (C, C') pairs
  const int64_t *r_squared;
  const uint64_t *q;
  const uint64_t *k;
  const int64_t *enter_shoup = nullptr;  // MIXED: the row's rescale_enter_shoup pairs
  const int64_t *r_mod = nullptr;        // MIXED: R mod q, indexed by prime
  ExactLimbs exact;
  __device__ __forceinline__ int64_t operator()(int poly, int limb, int prime, int gi, int n) const {
    const int64_t *s = src + poly * poly_stride;
    const int64_t x0 = s[gi];
    const int64_t xj = s[static_cast<long long>(limb + 1) * n + gi];
    const int64_t rounder = static_cast<uint64_t>(x0) > (q[prime - limb - 1] >> 1) ? 1 : 0;
    const uint64_t qq = q[prime], kk = k[prime];
    if (MIXED && !exact.exact(poly, limb)) {
      const int64_t q2 = static_cast<int64_t>(qq << 1);
      int64_t d = xj - x0;
      d = d >= 0 ? d : d + q2;
      if (d >= 0) {
        const uint64_t y = shoup_mult(static_cast<uint64_t>(enter_shoup[2 * prime]),
                                      static_cast<uint64_t>(enter_shoup[2 * prime + 1]),
                                      static_cast<uint64_t>(d), qq) +
                           (rounder ? static_cast<uint64_t>(r_mod[prime]) : 0);  // [0, 3q)
        return static_cast<int64_t>(y) >= q2 ? static_cast<int64_t>(y) - q2 : static_cast<int64_t>(y);
      }
    }
    const int64_t v = rescale_word_shoup(xj, x0, rounder, qq, kk, rescale_scale[prime],
                                         rescale_shoup + 2 * prime);
    return mont_mult_lazy(v, r_squared[prime], qq, kk);
  }
};

// attach_special_prime_chains_ (core.cpp:1127-1155) on the way in: x * P R^-1
// (mont_enter_scalar_ by P * R mod q) then to_ntt_'s enter.
struct ProductEnterLoad {
  const int64_t *src;
  long long poly_stride;
  const int64_t *p_product;  // P * R mod q, indexed by prime
  const int64_t *r_squared;
  const uint64_t *q;
  const uint64_t *k;
  __device__ __forceinline__ int64_t operator()(int poly, int limb, int prime, int gi, int n) const {
    const uint64_t qq = q[prime], kk = k[prime];
    const int64_t x = src[poly * poly_stride + (long long)limb * n + gi];
    return mont_mult_lazy(mont_mult_lazy(x, p_product[prime], qq, kk), r_squared[prime], qq, kk);
  }
};

// mont_enter_exit by N^-1*R on the way out: to_intt_ (core_ntt.cpp:131-148),
// optionally followed by reduce_2q_to_q (mod_down, core_key_switch.cpp:121).  With
// the reduction the word is the canonical residue of v N^-1 R^-1, so for v in
// [0, 2^62) one Shoup product by that constant and one subtraction give it.
template <bool REDUCE>
struct EnterExitStore {
  int64_t *dst;
  long long poly_stride;
  const int64_t *n_inverse;
  const uint64_t *q;
  const uint64_t *k;
  const int64_t *exit_shoup = nullptr;  // PrimeTables::exit_shoup, used when REDUCE
  __device__ __forceinline__ void operator()(int poly, int limb, int prime, int gi, int n, int64_t v) const {
    const uint64_t qq = q[prime], kk = k[prime];
    if (REDUCE && (static_cast<uint64_t>(v) >> kMontBits) == 0) {
      const uint64_t r = shoup_mult(static_cast<uint64_t>(exit_shoup[2 * prime]),
                                    static_cast<uint64_t>(exit_shoup[2 * prime + 1]),
                                    static_cast<uint64_t>(v), qq);
      dst[poly * poly_stride + (long long)limb * n + gi] = static_cast<int64_t>(r >= qq ? r - qq : r);
      return;
    }
    int64_t y = mont_exit(mont_mult_lazy(v, n_inverse[prime], qq, kk), qq, kk);
    if (REDUCE) y = guard(y, static_cast<int64_t>(qq));
    dst[poly * poly_stride + (long long)limb * n + gi] = y;
  }
};

// to_intt_'s exit (EnterExitStore<false>) after a mixed inverse transform: the exact
// limbs keep mont_exit(mont_mult(v, N^-1 R)); the others, whose words only matter
// modulo q, take one Shoup product by N^-1 R^-1, a word in [0, 2q) of the same value.
struct MixedExitStore {
  int64_t *dst;
  long long poly_stride;
  const int64_t *n_inverse;
  const uint64_t *q;
  const uint64_t *k;
  const int64_t *exit_shoup;  // PrimeTables::exit_shoup
  ExactLimbs exact;
  __device__ __forceinline__ void operator()(int poly, int limb, int prime, int gi, int n, int64_t v) const {
    const uint64_t qq = q[prime], kk = k[prime];
    int64_t *d = dst + poly * poly_stride + (long long)limb * n + gi;
    if (!exact.exact(poly, limb) && (static_cast<uint64_t>(v) >> kMontBits) == 0) {
      *d = static_cast<int64_t>(shoup_mult(static_cast<uint64_t>(exit_shoup[2 * prime]),
                                           static_cast<uint64_t>(exit_shoup[2 * prime + 1]),
                                           static_cast<uint64_t>(v), qq));
      return;
    }
    *d = mont_exit(mont_mult_lazy(v, n_inverse[prime], qq, kk), qq, kk);
  }
};

// Shared-memory word of element i of sub-transform c.  A 128-byte bank row holds 16
// words and a half-warp's 8-byte accesses are served together, so the swizzle must
// give the 16 threads of a half-warp 16 different rows positions.  XOR-ing
// (i >> 4) ^ ((i >> 5) << 2) and the column into the low four bits does that for
// every round of the 256-word passes (N = 2^16) in both directions, checked by
// simulating each round's access pattern; other shapes stay within 2 wavefronts.
// (For sub-transforms shorter than a row the XOR stays inside the sub-transform.)
template <int M>
__device__ __forceinline__ int tile_index(int c, int i) {
  constexpr int kMask = M >= 16 ? 15 : M - 1;
  return c * M + (i ^ (((i >> 4) ^ ((i >> 5) << 2) ^ c) & kMask));
}

// The swizzle is linear over XOR: tile_index(c, i ^ v) = tile_index(c, i) ^
// tile_xor(v) for i, v < M.  The elements of a radix-8 group are base ^ (e << dlog),
// so each costs one XOR with a constant.
template <int M>
__device__ __forceinline__ constexpr int tile_xor(int v) {
  return v ^ (((v >> 4) ^ ((v >> 5) << 2)) & (M >= 16 ? 15 : M - 1));
}

// A pass of S stages runs in R = ceil(S / 3) rounds of as equal a size as possible
// (S = 8: 3 + 3 + 2; S = 10: 3 + 3 + 2 + 2), each round a radix-2^r group of up to 8
// words per thread held in registers.  (Radix-16 rounds measured slower: at 80
// registers they spill and fewer CTAs fit an SM.)
constexpr int kNttMaxRoundLog = 3;
__host__ __device__ constexpr int ntt_rounds(int S) {
  return (S + kNttMaxRoundLog - 1) / kNttMaxRoundLog;
}
__host__ __device__ constexpr int ntt_round_log(int S, int round) {
  return S / ntt_rounds(S) + (round < S % ntt_rounds(S) ? 1 : 0);
}
__host__ __device__ constexpr int ntt_round_first(int S, int round) {
  return round * (S / ntt_rounds(S)) + (round < S % ntt_rounds(S) ? round : S % ntt_rounds(S));
}

constexpr int kNttThreads = 256;  // threads of every pass kernel

// A pass shape known at compile time: the default two-pass plan of N = 2^16
// (8 + 8 stages, 16 sub-transforms per CTA in both passes), whose index arithmetic
// then folds to constants.  kShapeStrided is the pass over sub-transforms of stride
// 256, kShapeContiguous the one over 256 adjacent words.
enum NttShape { kShapeRuntime = 0, kShapeStrided = 1, kShapeContiguous = 2 };
constexpr int kFixedLogN = 16;
constexpr int kFixedStages = 8;
constexpr int kFixedColumnsLog = 4;

template <int S, bool INVERSE, class Loader, class Storer, int VALUE_ONLY = kNttExact,
          int SHAPE = kShapeRuntime>
__global__ void __launch_bounds__(kNttThreads, 4)
    ntt_pass_kernel(NttPass a, PrimeTables t, Loader load, Storer store) {
  constexpr int M = 1 << S;
  constexpr int R = ntt_rounds(S);
  constexpr int kMaxE = 1 << kNttMaxRoundLog;
  extern __shared__ int64_t tile_smem[];
  static_assert(SHAPE == kShapeRuntime || S == kFixedStages, "fixed shapes are 8-stage passes");
  if (SHAPE != kShapeRuntime) {
    // The runtime fields hold the same values; the constants let them fold.
    a.log_n = kFixedLogN;
    a.stride_log = SHAPE == kShapeStrided ? kFixedLogN - kFixedStages : 0;
    a.first = (SHAPE == kShapeStrided) == INVERSE ? kFixedLogN - kFixedStages : 0;
    a.columns_log = kFixedColumnsLog;
  }

  const int pl = blockIdx.y;
  const int poly = pl % a.polys;
  const int limb = pl / a.polys;
  if (a.skip_start != nullptr && limb >= a.skip_start[poly] &&
      limb < a.skip_start[poly] + a.skip_size[poly])
    return;  // uniform per CTA, before any barrier
  const int prime = a.prime_base + limb;
  const uint64_t q = t.q[prime];
  const uint64_t k = t.k[prime];
  const int64_t q2 = static_cast<int64_t>(q << 1);
  const int n = 1 << a.log_n;
  // This CTA's limb only matters modulo q (uniform per CTA).
  const bool value_limb =
      VALUE_ONLY == kNttValueOnly || (VALUE_ONLY == kNttMixed && !a.exact.exact(poly, limb));
  // Twiddles of the general product: a mixed pass has exact limbs, which need the
  // reference's words; the same values serve its value-only limbs out of range.
  const int64_t *tw = (VALUE_ONLY == kNttValueOnly ? (INVERSE ? t.root_inverse_reduced : t.root_reduced)
                                                   : (INVERSE ? t.root_inverse : t.root)) +
                     static_cast<size_t>(prime) * (n - 1);
  // Value-only limbs' in-range words multiply by Shoup's (W, W') pairs instead.
  const longlong2 *tws =
      VALUE_ONLY ? reinterpret_cast<const longlong2 *>(INVERSE ? t.root_inverse_shoup : t.root_shoup) +
                       static_cast<size_t>(prime) * (n - 1)
                 : nullptr;
  // A forward value-only pass after the first reads words in [0, 4q).
  const uint64_t in_bound = (value_limb && !INVERSE && a.first > 0) ? (q << 2) : (q << 1);
  const bool last_pass = !INVERSE && a.first + S == a.log_n;
  const int T = 1 << a.stride_log;
  const bool strided = T > 1;
  const int C = 1 << a.columns_log;
  const int u0 = blockIdx.x * C;
  // Round 0 checks the words it loads; if every group of the CTA was in range, the
  // tile stays in range through the later rounds, which then skip the check.
  bool slow = false;
  bool tile_lazy = false;

#pragma unroll
  for (int round = 0; round < R; round++) {
    const int r = ntt_round_log(S, round);
    const int E = 1 << r;
    const int first_local = ntt_round_first(S, round);
    const int dlog = INVERSE ? first_local : (S - first_local - r);
    const int D = 1 << dlog;
    const int groups_per_col = M >> r;
    const int total = C * groups_per_col;
#pragma unroll 1
    for (int gid = threadIdx.x; gid < total; gid += kNttThreads) {
      int c, g;
      if (strided) {
        c = gid & (C - 1);
        g = gid >> a.columns_log;
      } else {
        c = gid / groups_per_col;
        g = gid - c * groups_per_col;
      }
      const int base = ((g >> dlog) << (dlog + r)) | (g & (D - 1));
      const int u = u0 + c;
      const int gbase = (u >> a.stride_log) * (M << a.stride_log) + (u & (T - 1));
      const int tb = tile_index<M>(c, base);
      int64_t x[kMaxE];
#pragma unroll
      for (int e = 0; e < kMaxE; e++) {
        if (e < E) {
          if (round == 0) {
            x[e] = load(poly, limb, prime, gbase + (base + e * D) * T, n);
          } else {
            x[e] = tile_smem[tb ^ tile_xor<M>(e << dlog)];
          }
        }
      }
      // Global index of element 0 of this radix-8 group.  Inside the group the
      // butterflies of one stage that share a twiddle form blocks of consecutive
      // elements, and the blocks' twiddles are consecutive table entries, so each
      // stage needs a single index computation.
      const int gi0 = gbase + base * T;
      // For q < 2^60, words in [0, 2q) stay there through every butterfly (the
      // reference's lazy range; twiddles are below 2q), and for them the
      // butterfly's signed compares and sign-extended product reduce to the short
      // forms below (same words); any other word takes the reference's forms.
      bool in_range = tile_lazy;
      if (round == 0) {
        in_range = q < (uint64_t(1) << 60);
#pragma unroll
        for (int e = 0; e < kMaxE; e++)
          if (e < E) in_range = in_range && static_cast<uint64_t>(x[e]) < in_bound;
        slow = slow || !in_range;
      }
      auto stages = [&](auto lazy, auto shoup) {
        constexpr bool kLazy = decltype(lazy)::value;
        // guard(a + b, q2) and guard(a + q2 - b, q2) (unit.h:13)
        auto add_guard = [&](int64_t a1, int64_t b1) -> int64_t {
          if (kLazy) {
            const int64_t y = a1 + b1 - q2;
            return y < 0 ? y + q2 : y;
          }
          return guard(a1 + b1, q2);
        };
        auto sub_guard = [&](int64_t a1, int64_t b1) -> int64_t {
          if (kLazy) {
            const int64_t y = a1 - b1;
            return y < 0 ? y + q2 : y;
          }
          return guard(a1 + q2 - b1, q2);
        };
        auto product = [&](int64_t w, int64_t v) -> int64_t {
          if (kLazy) return mont_mult_small(static_cast<uint64_t>(w), static_cast<uint64_t>(v), q, k);
          return mont_mult_const(w, v, q, k);
        };
        // The twiddle of table entry i: the Montgomery word, or for Harvey's form
        // on in-range words the Shoup pair (its product is the same value mod q).
        constexpr bool kShoup = kLazy && decltype(shoup)::value;
        struct Twiddle {
          int64_t w, wp;
        };
        auto twiddle = [&](size_t i) -> Twiddle {
          if (kShoup) {
            const longlong2 v = __ldg(tws + i);
            return {v.x, v.y};
          }
          return {__ldg(tw + i), 0};
        };
        auto value_product = [&](const Twiddle &w, int64_t v) -> int64_t {
          return static_cast<int64_t>(shoup_mult(static_cast<uint64_t>(w.w), static_cast<uint64_t>(w.wp),
                                                 static_cast<uint64_t>(v), q));
        };
#pragma unroll
        for (int j = 0; j < kNttMaxRoundLog; j++) {
          if (j < r) {
            if (!INVERSE) {
              // stage s: twiddle root[2^s - 1 + (gi >> (log_n - s))]; the block of
              // element e is e >> (r - j) (ntt.cpp:46-134)
              const int s = a.first + first_local + j;
              const int half = E >> (j + 1);
              const size_t wi = (1 << s) - 1 + (gi0 >> (a.log_n - s));
#pragma unroll
              for (int h = 0; h < (1 << j); h++) {
                const Twiddle w = twiddle(wi + h);
#pragma unroll
                for (int e2 = 0; e2 < kMaxE / 2; e2++) {
                  if (e2 < half) {
                    const int e = h * 2 * half + e2;
                    if (kShoup) {
                      // Harvey's form: words in [0, 4q), one guard per butterfly;
                      // Shoup's product is below 2q.
                      int64_t uu = x[e] - q2;
                      uu = uu < 0 ? uu + q2 : uu;
                      const int64_t p = value_product(w, x[e + half]);
                      x[e] = uu + p;
                      x[e + half] = uu - p + q2;
                      continue;
                    }
                    const int64_t uu = x[e];
                    const int64_t p = product(w.w, x[e + half]);
                    x[e] = add_guard(uu, p);
                    x[e + half] = sub_guard(uu, p);
                  }
                }
              }
            } else {
              // distance 2^dg: twiddle root_inverse[N - N/2^dg + (gi >> (dg + 1))]
              // (ntt.cpp:177-272); the block of element e is e >> (j + 1)
              const int dg = a.first + first_local + j;
              const int half = 1 << j;
              const size_t wi = n - (n >> dg) + (gi0 >> (dg + 1));
#pragma unroll
              for (int h = 0; h < kMaxE / 2; h++) {
                if (h < (E >> (j + 1))) {
                  const Twiddle w = twiddle(wi + h);
#pragma unroll
                  for (int e2 = 0; e2 < kMaxE / 2; e2++) {
                    if (e2 < half) {
                      const int e = h * 2 * half + e2;
                      const int64_t uu = x[e];
                      const int64_t vv = x[e + half];
                      x[e] = add_guard(uu, vv);
                      // Harvey's form: the product's operand in (0, 4q) needs no guard.
                      x[e + half] = kShoup ? value_product(w, uu - vv + q2)
                                           : product(w.w, sub_guard(uu, vv));
                    }
                  }
                }
              }
            }
          }
        }
      };
      if (in_range) {
        if constexpr (VALUE_ONLY == kNttValueOnly) {
          stages(std::true_type{}, std::true_type{});
        } else if constexpr (VALUE_ONLY == kNttMixed) {
          if (value_limb) {
            stages(std::true_type{}, std::true_type{});
          } else {
            stages(std::true_type{}, std::false_type{});
          }
        } else {
          stages(std::true_type{}, std::false_type{});
        }
      } else {
        stages(std::false_type{}, std::false_type{});
      }
#pragma unroll
      for (int e = 0; e < kMaxE; e++) {
        if (e < E) {
          if (round == R - 1) {
            if (VALUE_ONLY && value_limb && !INVERSE && last_pass && in_range) {
              const int64_t y = x[e] - q2;  // [0, 4q) -> [0, 2q)
              x[e] = y < 0 ? x[e] : y;
            }
            store(poly, limb, prime, gbase + (base + e * D) * T, n, x[e]);
          } else {
            tile_smem[tb ^ tile_xor<M>(e << dlog)] = x[e];
          }
        }
      }
    }
    if (round == 0 && R > 1) {
      tile_lazy = __syncthreads_or(slow) == 0;
    } else if (round < R - 1) {
      __syncthreads();
    }
  }
}

// Pass plan of a transform of 2^log_n words: for two passes, the tuned or default
// split and tile shapes (ntt_tuning, kernels.cuh).  Every plan performs the same
// butterflies, so every plan gives the same words.
struct NttPlan {
  int passes;             // 1 or 2
  int s_first;            // S of the strided (outer) pass, or log_n for a single pass
  int s_second;           // S of the contiguous (inner) pass
  int first_columns_log;  // sub-transforms per CTA of the strided pass
  int second_columns_log; // sub-transforms per CTA of the contiguous pass
};

inline NttPlan ntt_plan(int log_n) {
  if (log_n <= 11) return {1, log_n, 0, 0, 0};
  const NttTuning tu = ntt_tuning(log_n);
  return {2, log_n - tu.s_second, tu.s_second, tu.first_columns_log,
          tu.second_tile_log - tu.s_second};
}


template <int S, bool INVERSE, class Loader, class Storer, int VALUE_ONLY = kNttExact,
          int SHAPE = kShapeRuntime>
cudaError_t launch_ntt_pass(const NttPass &a, const PrimeTables &t, const Loader &ld,
                            const Storer &st, cudaStream_t stream) {
  const int subs = (1 << a.log_n) >> S;
  const dim3 grid(subs >> a.columns_log, a.polys * a.limbs);
  const size_t smem = sizeof(int64_t) << (a.columns_log + S);
  auto kernel = ntt_pass_kernel<S, INVERSE, Loader, Storer, VALUE_ONLY, SHAPE>;
  // Raised once per instantiation to the most any valid plan uses, so no attribute
  // call lands inside a graph capture.
  static bool raised = false;
  if (!raised) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kNttMaxSmem);
    if (e != cudaSuccess) return e;
    raised = true;
  }
  if (smem > static_cast<size_t>(kNttMaxSmem)) return cudaErrorInvalidValue;
  note_launch(1);
  kernel<<<grid, kNttThreads, smem, stream>>>(a, t, ld, st);
  return cudaGetLastError();
}

template <bool INVERSE, class Loader, class Storer, int VALUE_ONLY = kNttExact>
cudaError_t dispatch_ntt_pass(int S, const NttPass &a, const PrimeTables &t, const Loader &ld,
                              const Storer &st, cudaStream_t stream) {
  if (S == kFixedStages && a.log_n == kFixedLogN && a.columns_log == kFixedColumnsLog) {
    const int strided_first = INVERSE ? kFixedLogN - kFixedStages : 0;
    if (a.stride_log == kFixedLogN - kFixedStages && a.first == strided_first)
      return launch_ntt_pass<kFixedStages, INVERSE, Loader, Storer, VALUE_ONLY, kShapeStrided>(
          a, t, ld, st, stream);
    if (a.stride_log == 0 && a.first == kFixedLogN - kFixedStages - strided_first)
      return launch_ntt_pass<kFixedStages, INVERSE, Loader, Storer, VALUE_ONLY, kShapeContiguous>(
          a, t, ld, st, stream);
  }
  switch (S) {
    case 1: return launch_ntt_pass<1, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 2: return launch_ntt_pass<2, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 3: return launch_ntt_pass<3, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 4: return launch_ntt_pass<4, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 5: return launch_ntt_pass<5, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 6: return launch_ntt_pass<6, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 7: return launch_ntt_pass<7, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 8: return launch_ntt_pass<8, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 9: return launch_ntt_pass<9, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 10: return launch_ntt_pass<10, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    case 11: return launch_ntt_pass<11, INVERSE, Loader, Storer, VALUE_ONLY>(a, t, ld, st, stream);
    default: return cudaErrorInvalidValue;
  }
}

// Batched forward NTT of `polys` x `limbs` limbs.  The first pass reads through
// `ld`, the last pass writes through `st`; intermediate data lives in `work`
// ([poly][limb][N], stride work_stride), which may alias the final destination.
template <class Loader, class Storer, int VALUE_ONLY = kNttExact>
cudaError_t forward_ntt(int log_n, int polys, int limbs, int prime_base, const PrimeTables &t,
                        const Loader &ld, const Storer &st, int64_t *work, long long work_stride,
                        cudaStream_t stream, const int *skip_start = nullptr,
                        const int *skip_size = nullptr, const ExactLimbs &exact = ExactLimbs{}) {
  const NttPlan plan = ntt_plan(log_n);
  NttPass a{log_n, 0, 0, 1, polys, limbs, prime_base, skip_start, skip_size, exact};
  if (plan.passes == 1) {
    a.stride_log = 0;
    a.first = 0;
    a.columns_log = 0;
    return dispatch_ntt_pass<false, Loader, Storer, VALUE_ONLY>(plan.s_first, a, t, ld, st, stream);
  }
  PlainStore mid_store{work, work_stride};
  PlainLoad mid_load{work, work_stride};
  a.stride_log = plan.s_second;
  a.first = 0;
  a.columns_log = plan.first_columns_log;
  cudaError_t e = dispatch_ntt_pass<false, Loader, PlainStore, VALUE_ONLY>(plan.s_first, a, t, ld,
                                                                          mid_store, stream);
  if (e != cudaSuccess) return e;
  a.stride_log = 0;
  a.first = plan.s_first;
  a.columns_log = plan.second_columns_log;
  return dispatch_ntt_pass<false, PlainLoad, Storer, VALUE_ONLY>(plan.s_second, a, t, mid_load, st,
                                                                 stream);
}

template <class Loader, class Storer, int VALUE_ONLY = kNttExact>
cudaError_t inverse_ntt(int log_n, int polys, int limbs, int prime_base, const PrimeTables &t,
                        const Loader &ld, const Storer &st, int64_t *work, long long work_stride,
                        cudaStream_t stream, const ExactLimbs &exact = ExactLimbs{}) {
  const NttPlan plan = ntt_plan(log_n);
  NttPass a{log_n, 0, 0, 1, polys, limbs, prime_base};
  a.exact = exact;
  if (plan.passes == 1) {
    a.stride_log = 0;
    a.first = 0;
    a.columns_log = 0;
    return dispatch_ntt_pass<true, Loader, Storer, VALUE_ONLY>(plan.s_first, a, t, ld, st, stream);
  }
  PlainStore mid_store{work, work_stride};
  PlainLoad mid_load{work, work_stride};
  a.stride_log = 0;
  a.first = 0;
  a.columns_log = plan.second_columns_log;
  cudaError_t e = dispatch_ntt_pass<true, Loader, PlainStore, VALUE_ONLY>(plan.s_second, a, t, ld,
                                                                         mid_store, stream);
  if (e != cudaSuccess) return e;
  a.stride_log = plan.s_second;
  a.first = plan.s_second;
  a.columns_log = plan.first_columns_log;
  return dispatch_ntt_pass<true, PlainLoad, Storer, VALUE_ONLY>(plan.s_first, a, t, mid_load, st,
                                                                stream);
}

}  // namespace fhe_b200
