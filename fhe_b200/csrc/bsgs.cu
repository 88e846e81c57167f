// The inner loop of the hoisted baby-step giant-step linear transform in one kernel
// (CKKSEngine::apply_butterfly with a bootstrap key, engine_bootstrap.cpp:218-262;
// ntt_rotate, core.cpp:965-1000; the key switcher, core_key_switch.cpp:510-548).
//
// The reference rotates the special-prime-extended NTT-form text x by every inner
// delta through one decomposition -- for inner text i, word c of polynomial p is
//   r_i[p][c] = [p == 0] x[0][s] + sum_part dec[part][s] key_i[2 part + p][s],
//   s = perm_i[c] (each product a Montgomery product) --
// and then sums, per outer group g, the products r_i * d_gi with the group's
// pre-encoded diagonals d_gi.  Every group sum reaches the output only through
// ModDown (its inverse transform reduces every word; the giant-step rotation adds
// the sum's polynomial 0 to a key product and ModDowns that), so only its value
// modulo q matters.  Here one thread owns one output word of one polynomial and
// keeps the sums of all groups in registers: per inner text it gathers the
// decomposition and the rotation key at s, forms r_i from one exact 128-bit sum and
// one REDC, and adds r_i d_gi to every group's exact 128-bit sum; each group sum gets
// one REDC at the end, a word in [0, q).  The rotated texts, the key products and
// the per-term reductions never reach memory.
//
// With every operand in [0, 2^61) the sums are exact: a key product term is below
// 2^122 (at most 8 partitions), r_i is below q + 2^61, a diagonal product below 2^123
// and a group holds at most 16 terms.  The operands' high words are OR-ed as they
// are read; a thread that met a word outside that range recomputes its outputs with
// the unfused kernels' chains, word for word.
#include "kernels.cuh"
#include "modarith.cuh"

namespace fhe_b200 {

namespace {

constexpr int kBsgsThreads = 256;
constexpr int kBsgsCoeffs = kBsgsThreads / 2;  // a CTA: 128 words x both polynomials

struct BsgsWord {
  int poly;
  long long r, row, per_poly;  // r = row + c: word r of the polynomial, row = limb * N
  int c;
  uint64_t q, k;
  double inv_q;
};

__device__ __forceinline__ uint32_t high_word(int64_t v) {
  return static_cast<uint32_t>(static_cast<uint64_t>(v) >> 32);
}

// Inner text i at the thread's word as the unfused path computes it: the key inner
// product at the gathered position (key_inner_product_kernel, wide form), then
// ntt_rotate_finish_kernel's addition of x's polynomial 0.
__device__ int64_t rotated_word_chain(const BsgsWord &w, const BsgsInner &b, int parts, int i,
                                      const int64_t *x, long long x_stride,
                                      const int64_t *dec) {
  if (i == 0) return x[w.poly * x_stride + w.r];
  const long long src = w.row + b.perm[i][w.c];
  const int64_t *key = b.key[i] + src;
  const int64_t qs = static_cast<int64_t>(w.q), q2 = qs << 1;
  bool fast = true;
  WideSum s0, s1;
  for (int p = 0; p < parts && fast; p++) {
    const int64_t e = dec[p * w.per_poly + src];
    const int64_t k0 = key[b.key_off[i][p]];
    const int64_t k1 = key[b.key_off[i][p] + static_cast<long long>(b.key_poly[i])];
    fast = redc_operand_ok(e) && redc_operand_ok(k0) && redc_operand_ok(k1);
    s0.add(static_cast<uint64_t>(e), static_cast<uint64_t>(k0));
    s1.add(static_cast<uint64_t>(e), static_cast<uint64_t>(k1));
  }
  int64_t v;
  if (fast) {
    v = (w.poly == 0 ? s0 : s1).reduce(w.q, w.k, w.q, w.inv_q);
  } else {
    v = 0;
    const long long poly_off = w.poly == 0 ? 0 : b.key_poly[i];
    for (int p = 0; p < parts; p++) {
      const int64_t e = dec[p * w.per_poly + src];
      const int64_t a = mont_mult(e, key[b.key_off[i][p] + poly_off], w.q, w.k);
      v = p == 0 ? a : guard(guard(a + v, q2), qs);
    }
  }
  if (w.poly == 0) v = guard(x[src] + v, q2);
  return v;
}

// Eight groups keep their sums and loads in flight at two CTAs per SM; four groups
// run fastest at three (measured).
template <int G, int P>
__global__ void __launch_bounds__(kBsgsThreads, G <= 4 ? 3 : 2)
bsgs_inner_kernel(PrimeTables t, int log_n, int moduli_id, int extended, const int64_t *x,
                  long long x_stride, const int64_t *dec, const __grid_constant__ BsgsInner b) {
  BsgsWord w;
  const int n = 1 << log_n;
  w.per_poly = static_cast<long long>(extended) << log_n;
  w.poly = threadIdx.x / kBsgsCoeffs;
  w.r = static_cast<long long>(blockIdx.x) * kBsgsCoeffs + threadIdx.x % kBsgsCoeffs;
  if (w.r >= w.per_poly) return;
  const int j = static_cast<int>(w.r >> log_n);
  w.c = static_cast<int>(w.r & (n - 1));
  w.row = w.r - w.c;
  const int prime = moduli_id + j;
  w.q = t.q[prime];
  w.k = t.k[prime];
  w.inv_q = t.inv_q[prime];

  WideSum acc[G];
  uint32_t high = 0;  // OR of every operand's high word
  {
    const int64_t x0 = x[w.poly * x_stride + w.r];
    const uint32_t mask = b.mask[0];
    high = high_word(x0);
#pragma unroll
    for (int g = 0; g < G; g++) {
      if (mask >> g & 1) {
        const int64_t dv = b.diag[0][g][w.r];
        high |= high_word(dv);
        acc[g].add(static_cast<uint64_t>(x0), static_cast<uint64_t>(dv));
      }
    }
  }
  const int64_t *x_row = x + w.row;
  const int64_t *dec_row = dec + w.row;
  int perm_next = b.inner > 1 ? b.perm[1][w.c] : 0;
  for (int i = 1; i < b.inner; i++) {
    const uint32_t mask = b.mask[i];
    int64_t dv[G];
#pragma unroll
    for (int g = 0; g < G; g++) dv[g] = (mask >> g & 1) ? b.diag[i][g][w.r] : 0;
    const int s = perm_next;
    if (i + 1 < b.inner) perm_next = b.perm[i + 1][w.c];
    const int64_t *key = b.key[i] + w.row + s + (w.poly == 0 ? 0 : b.key_poly[i]);
    int64_t e[P], kw[P];
#pragma unroll
    for (int p = 0; p < P; p++) {
      e[p] = dec_row[p * w.per_poly + s];
      kw[p] = key[b.key_off[i][p]];
    }
    const int64_t x0 = w.poly == 0 ? x_row[s] : 0;
    WideSum ks;
#pragma unroll
    for (int p = 0; p < P; p++) {
      high |= high_word(e[p]) | high_word(kw[p]);
      ks.add(static_cast<uint64_t>(e[p]), static_cast<uint64_t>(kw[p]));
    }
    high |= high_word(x0);
    const uint64_t v =
        static_cast<uint64_t>(ks.reduce(w.q, w.k, w.q, w.inv_q)) + static_cast<uint64_t>(x0);
#pragma unroll
    for (int g = 0; g < G; g++) {
      if (mask >> g & 1) {
        high |= high_word(dv[g]);
        acc[g].add(v, static_cast<uint64_t>(dv[g]));
      }
    }
  }

  const int64_t qs = static_cast<int64_t>(w.q), q2 = qs << 1;
  if ((high >> 29) == 0) {  // every operand below 2^61
    int64_t run = 0;
#pragma unroll
    for (int g = 0; g < G; g++) {
      if (g < b.groups) {
        const int64_t v = acc[g].reduce(w.q, w.k, w.q, w.inv_q);
        run = (b.lead >> g & 1) ? v : guard(run + v, qs);
        if (g + 1 == b.groups || (b.lead >> (g + 1) & 1)) b.out[g][w.poly * w.per_poly + w.r] = run;
      }
    }
    return;
  }
  // diagonal_mac_kernel's chain over each output's terms: its outer indices in
  // order, i ascending within each.
  int64_t a = 0;
  bool first = true;
  for (int g = 0; g < b.groups; g++) {
    if (b.lead >> g & 1) first = true;
    for (int i = 0; i < b.inner; i++) {
      if (!(b.mask[i] >> g & 1)) continue;
      const int64_t xv = rotated_word_chain(w, b, P, i, x, x_stride, dec);
      const int64_t m = mont_mult_lazy(xv, b.diag[i][g][w.r], w.q, w.k);
      a = first ? m : guard(guard(a + m, q2), qs);
      first = false;
    }
    if (g + 1 == b.groups || (b.lead >> (g + 1) & 1)) b.out[g][w.poly * w.per_poly + w.r] = a;
  }
}

template <int G>
cudaError_t launch_groups(unsigned grid, cudaStream_t s, int partitions, const PrimeTables &t,
                          int log_n, int moduli_id, int extended, const int64_t *x,
                          long long x_stride, const int64_t *dec, const BsgsInner &b) {
  switch (partitions) {
#define FHE_BSGS_CASE(P)                                                                     \
  case P:                                                                                    \
    bsgs_inner_kernel<G, P><<<grid, kBsgsThreads, 0, s>>>(t, log_n, moduli_id, extended, x, \
                                                          x_stride, dec, b);                 \
    break;
    FHE_BSGS_CASE(1) FHE_BSGS_CASE(2) FHE_BSGS_CASE(3) FHE_BSGS_CASE(4)
    FHE_BSGS_CASE(5) FHE_BSGS_CASE(6) FHE_BSGS_CASE(7) FHE_BSGS_CASE(8)
#undef FHE_BSGS_CASE
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_bsgs_inner(const PrimeTables &t, int log_n, int moduli_id, int extended,
                              int partitions, const int64_t *x, long long x_stride,
                              const int64_t *decomposed, const BsgsInner &b, cudaStream_t s) {
  if (b.inner < 1 || b.inner > kBsgsMaxInner || b.groups < 1 || b.groups > kBsgsMaxGroups ||
      partitions < 1 || partitions > kBsgsMaxPartitions || extended < 1)
    return cudaErrorInvalidValue;
  if (!(b.lead & 1) || (b.lead >> b.groups)) return cudaErrorInvalidValue;
  for (int g = 0; g < b.groups; g++) {
    int terms = 0;
    for (int i = 0; i < b.inner; i++) terms += b.mask[i] >> g & 1;
    if (terms < 1 || b.out[g] == nullptr) return cudaErrorInvalidValue;
  }
  for (int i = 0; i < b.inner; i++) {
    if (b.mask[i] >> b.groups) return cudaErrorInvalidValue;
    for (int g = 0; g < b.groups; g++)
      if ((b.mask[i] >> g & 1) != (b.diag[i][g] != nullptr ? 1u : 0u)) return cudaErrorInvalidValue;
    if (i > 0 && (b.perm[i] == nullptr || b.key[i] == nullptr)) return cudaErrorInvalidValue;
  }
  const long long words = static_cast<long long>(extended) << log_n;
  const unsigned grid = static_cast<unsigned>((words + kBsgsCoeffs - 1) / kBsgsCoeffs);
  note_launch();
  if (b.groups <= 4)
    return launch_groups<4>(grid, s, partitions, t, log_n, moduli_id, extended, x, x_stride,
                            decomposed, b);
  return launch_groups<8>(grid, s, partitions, t, log_n, moduli_id, extended, x, x_stride,
                          decomposed, b);
}

}  // namespace fhe_b200
