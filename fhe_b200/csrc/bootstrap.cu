// CKKS bootstrapping with a rotation key (DESILO FHE ckks/engine_bootstrap.cpp,
// engine_mod_raise.cpp, operation/bootstrap.cpp): mod raise through a sparse secret,
// coefficients-to-slots butterflies, EvalRound (sine by Chebyshev
// Paterson-Stockmeyer and three double-angle steps), slots-to-coefficients, and the
// final correction.  Every step is an engine operation already on the device; this
// file composes them in the reference's order so each intermediate word matches,
// and builds the butterfly twiddles on the host with the reference's expressions.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <complex>
#include <map>

#include "engine.hpp"

namespace fhe_b200 {

namespace {

using cvec = std::vector<std::complex<double>>;
using Stages = std::vector<std::vector<cvec>>;

constexpr double kPi = 3.141592653589793;  // std::numbers::pi
constexpr int64_t kRoundBound = 28;         // operation/bootstrap.h:9
constexpr int kBabyDegree = 7;
constexpr int kGiantDegree = 3;

int pmod(int x, int m) { return (m + x % m) % m; }

cvec phi(int count, double sign) {
  // get_phi / get_inverse_phi (operation/bootstrap.cpp:9-33).
  cvec out(count);
  const double pi_over = kPi / count;
  for (int i = 0; i < count; i++) out[i] = std::exp(std::complex<double>(0, sign * 2 * pi_over * i));
  return out;
}

struct Factors {
  std::vector<cvec> center, left, right;
};

Factors twiddle_factors(int slot_count, int log_slot_count, bool inverse) {
  // get_twiddle_factor / get_inverse_twiddle_factor (operation/bootstrap.cpp:35-123).
  Factors f;
  const cvec table = phi(slot_count << 2, inverse ? 1.0 : -1.0);
  int jump_size = inverse ? 1 : slot_count;
  for (int step = 0; step < log_slot_count; step++) {
    const int log_slot_index = inverse ? log_slot_count - 1 - step : step;
    const int jump_count = 1 << log_slot_index;
    if (!inverse) jump_size >>= 1;
    std::vector<int> index_table;
    int power_of_five = 1;
    for (int s = 0; s < jump_size; s++) {
      index_table.push_back(power_of_five * jump_count);
      power_of_five *= 5;
      power_of_five &= (jump_size << 3) - 1;
    }
    cvec center(slot_count, 0), left(slot_count, 0), right(slot_count, 0);
    for (int j = 0; j < jump_count; j++) {
      int index = 2 * j * jump_size;
      for (int s = 0; s < jump_size; s++) {
        const auto value = table[index_table[s]];
        center[index] = 1;
        center[jump_size + index] = -value;
        if (inverse) {
          left[index] = value;
          right[jump_size + index] = 1;
        } else {
          left[index] = 1;
          right[jump_size + index] = value;
        }
        index++;
      }
    }
    f.center.push_back(center);
    f.left.push_back(left);
    f.right.push_back(right);
    if (inverse) jump_size <<= 1;
  }
  return f;
}

int cts_log_radix(int stage, int stages, int log_slot) {
  return stage >= stages - log_slot % stages ? log_slot / stages + 1 : log_slot / stages;
}

int stc_log_radix(int stage, int stages, int log_slot) {
  return stage < log_slot % stages ? log_slot / stages + 1 : log_slot / stages;
}

Stages butterfly_twiddles(int slot_count, int log_slot_count, int stage_count, bool to_slot) {
  // get_coeff_to_slot_twiddles / get_slot_to_coeff_twiddles (operation/bootstrap.cpp:125-263).
  const Factors f = twiddle_factors(slot_count, log_slot_count, !to_slot);
  Stages out;
  int radix_jump_size = to_slot ? slot_count : 1;
  int offset = 0;
  for (int stage = 0; stage < stage_count; stage++) {
    const int log_radix = to_slot ? cts_log_radix(stage, stage_count, log_slot_count)
                                  : stc_log_radix(stage, stage_count, log_slot_count);
    const int radix_count = 1 << log_radix;
    const int total = 2 * radix_count - 1;
    std::vector<cvec> stage_tw(total, cvec(slot_count, 1));
    for (int lr = 0; lr < log_radix; lr++) {
      if (to_slot) radix_jump_size >>= 1;
      const int radix_index = 1 << lr;
      const int jump_size = to_slot ? radix_count / (2 * radix_index) : radix_index;
      const int ti = offset + lr;
      std::vector<cvec> radix_tw(total, cvec(slot_count, 0));
      stage_tw.swap(radix_tw);
      const cvec &center = f.center[ti], &left = f.left[ti], &right = f.right[ti];
      for (int index = -radix_index + 1; index < radix_index; index++) {
        const int unit = to_slot ? index * radix_count / radix_index : index;
        const int ci = pmod(unit, total);
        const int li = pmod(unit - jump_size, total);
        const int ri = pmod(unit + jump_size, total);
        for (int s = 0; s < slot_count; s++) {
          stage_tw[ci][s] += center[s] * radix_tw[ci][s];
          stage_tw[li][s] += left[s] * radix_tw[ci][pmod(s + radix_jump_size, slot_count)];
          stage_tw[ri][s] += right[s] * radix_tw[ci][pmod(s - radix_jump_size, slot_count)];
        }
      }
      if (!to_slot) radix_jump_size <<= 1;
    }
    if (to_slot && stage == stage_count - 1) {
      const int normalizing = 2 * slot_count * static_cast<int>(kRoundBound);
      for (auto &v : stage_tw)
        for (auto &x : v) x /= normalizing;
    }
    out.push_back(std::move(stage_tw));
    offset += log_radix;
  }
  return out;
}

std::pair<int, int> stage_loop_counts(int twiddle_count, int inner_loop_shift = 0) {
  // get_stage_loop_counts (operation/bootstrap.cpp:265-278).
  int bits = 0;
  for (int t = twiddle_count; t > 0; t >>= 1) bits++;
  const int inner = 1 << ((bits + 1) / 2 + inner_loop_shift);
  return {inner, (twiddle_count + 1) / inner};
}

cvec rotate_vector(const cvec &input, int delta) {
  // CKKSEngine::rotate_vector (engine_bootstrap.cpp:856-870).
  const int count = static_cast<int>(input.size());
  if (count == 0) return input;
  const int nd = (delta + 2 * count) % count;
  cvec out(count);
  for (int i = 0; i < count; i++) out[(i + nd) % count] = input[i];
  return out;
}

// Coefficients of sine's Chebyshev evaluation (engine_bootstrap.cpp:500-524).
const std::vector<double> kAuxiliary = {-0.4674215360340989,   -0.24807246365084598,
                                        -0.03360736343811264,  0.10485552200765141,
                                        0.012171628025753911,  -0.031034212401993305,
                                        -0.003985828764410408, 0.0};
const std::vector<std::vector<double>> kQuotient = {
    {-0.7500012154934053, 4.148627473785995e-06, 2.707983311367457e-07, -4.324538856989888e-07,
     -2.648274421485692e-08, 3.9515438249932484e-08, 2.4720260690299275e-09, 0.0},
    {-6.511205244110998e-09, -7.076428529570776e-10, 1.0183620860162692e-09, 0.0, 0.0, 0.0, 0.0,
     4.0},
    {0.007868944223231958, 0.0014193060148561195, -0.003081157124604844, -0.00025275745577540515,
     0.0005030348400875631, 3.734766164626263e-05, -7.780382338014487e-05, 1.0}};
const std::vector<std::vector<double>> kRemainder = {
    {-1.1324455480972702, -0.8116709016985189, -0.20294197180913795, 0.5290215620326779,
     -0.32084902738708476, 0.43458317383580536, -0.06303880005650665, 0.0},
    {0.23316927298939902, 0.12938749185636858, -0.3042902283756468, -0.008967445477730096,
     -0.6955791340472846, -0.07562064123442451, 1.2510854562849574, 2.0},
    {0.1429148264191405, 0.4544397978460022, -0.8401926425765848, -0.4292803758141986,
     -1.495563076527614, 0.3580084476476745, 1.7971594278092713, 1.0}};

using Owned = std::unique_ptr<Data>;

}  // namespace

// --------------------------------------------------------------- helpers --

void Engine::add_inplace(Data &a, const Data &b) {
  // CKKSCore::add_inplace (core.cpp:498-512): polynomial-wise reduce(a + b).
  const long long ps = a.poly_stride();
  for (int p = 0; p < a.polys; p++)
    pointwise(kOpAddReduce, a.chains, a.moduli_id, a.d + p * ps, b.d + p * b.poly_stride(), nullptr,
              a.d + p * ps);
}

std::unique_ptr<Data> Engine::multiply_imaginary(const Data &ct, int64_t value) {
  // CKKSEngine::multiply_imaginary (engine_multiply.cpp:468-491): the NTT-form text
  // times the plaintext X^(N/2) * value (encode_imaginary, encode.cpp:387-394), back
  // to coefficient form when the input was.
  std::unique_ptr<Data> hold;
  const Data *x = &ct;
  if (!x->is_ntt()) {
    hold = to_ntt(*x);
    x = hold.get();
  }
  const int mid = x->moduli_id, L = params.chains(mid);
  auto pt = make_data(kUnitPlaintext, kFlagComplex, mid, 1, 1.0L);
  const std::vector<int64_t> monomial(L, value);
  pointwise(kOpMonomial, L, mid, nullptr, nullptr, monomial.data(), pt->d);
  ntt_in_place(pt->d, L, mid, pt->poly_stride(), 1);
  auto out = make_data(kUnitCiphertext, (x->flag | kFlagComplex) & ~kFlagRescaled, mid, x->polys,
                       x->scale);
  const long long ps = x->poly_stride();
  for (int p = 0; p < x->polys; p++)
    pointwise(kOpMult, x->chains, mid, x->d + p * ps, pt->d, nullptr, out->d + p * ps);
  if (!ct.is_ntt()) return to_intt(*out);
  return out;
}

std::unique_ptr<Data> Engine::weighted_sum(const std::vector<const Data *> &basis,
                                           const std::vector<double> &weights) {
  // CKKSEngine::weighted_sum_ (engine_advanced.cpp:228-269).
  Owned result;
  for (int index = static_cast<int>(weights.size()) - 1; index > 0; index--) {
    const double w = weights[index];
    if (w == 0) continue;
    auto product = multiply_scalar(*basis[index - 1], w);
    if (!result) {
      result = std::move(product);
      continue;
    }
    result = add(*result, *product);
  }
  if (weights[0] != 0) result = add_scalar(*result, weights[0]);
  return result;
}

std::vector<std::unique_ptr<Data>> Engine::rotate_batch(const Data &ct,
                                                        const std::vector<const Data *> &keys,
                                                        const std::vector<int> &deltas) {
  // CKKSEngine::rotate_batch (engine_rotate.cpp:304-408): each delta is the chain of
  // the fixed keys of its set bits, lowest first, from the prepared input; results
  // repeat for repeated deltas.
  if (deltas.empty())
    throw std::runtime_error(
        "Batch Rotate Unit Ciphertext With Rotation Key: the input delta vector is empty.");
  Owned prepared;
  const Data *x = &ct;
  if (params.preset.one_more_level && ct.moduli_id == 0) {
    prepared = level_down_any(ct, ct.level() - 1);
    x = prepared.get();
  }
  if (x->is_ntt()) {
    prepared = to_intt(*x);
    x = prepared.get();
  }
  std::map<int, Owned> done;
  std::vector<Owned> out;
  for (int delta : deltas) {
    const int nd = normalized_delta(delta);
    if (nd == 0) {
      out.push_back(clone(*x));
      continue;
    }
    Owned cur;
    for (const Data *k : keys) {
      if ((nd & k->delta) == 0) continue;
      const int current = (nd & (k->delta - 1)) + k->delta;
      auto it = done.find(current);
      if (it == done.end()) {
        auto r = core_rotate(cur ? *cur : *x, *k);
        it = done.emplace(current, std::move(r)).first;
      }
      cur = clone(*it->second);
      if (current == nd) break;
    }
    out.push_back(std::move(cur));
  }
  return out;
}

// ------------------------------------------------------------- the stages --

const std::vector<std::vector<std::vector<std::complex<double>>>> &Engine::bootstrap_twiddles(
    bool to_slot, int stage_count) {
  const auto key = std::make_pair(to_slot, stage_count);
  auto it = twiddle_cache_.find(key);
  if (it == twiddle_cache_.end())
    it = twiddle_cache_
             .emplace(key, butterfly_twiddles(params.slot_count, params.log_slot_count, stage_count,
                                              to_slot))
             .first;
  return it->second;
}

std::unique_ptr<Data> Engine::apply_butterfly(const Data &ct, bool to_slot, int stage_count,
                                              int stage, const std::vector<const Data *> &keys,
                                              int rotate_count) {
  // CKKSEngine::apply_butterfly with a rotation key (engine_bootstrap.cpp:155-216).  The
  // reference encodes each diagonal at every call and multiplies through
  // prepare_for_multiply; the prepared (rescaled, NTT-form) diagonal depends only on
  // the stage, its position and the level, so it is made once and kept on the device.
  const auto &twiddle = bootstrap_twiddles(to_slot, stage_count)[stage];
  const int count = static_cast<int>(twiddle.size());
  const auto [inner, outer] = stage_loop_counts(count);
  std::vector<int> inner_deltas;
  for (int i = 0; i < inner; i++) inner_deltas.push_back(rotate_count * i);
  auto rotated = rotate_batch(ct, keys, inner_deltas);
  Owned outer_sum;
  for (int o = 0; o < outer; o++) {
    const int norm_o = o - outer / 2;
    const int factor_delta = inner * norm_o * rotate_count;
    Owned inner_sum;
    for (int i = (o == 0 ? 1 : 0); i < inner; i++) {
      const int index = inner * norm_o + i;
      const int level = rotated[i]->level();
      const auto key = std::make_tuple(to_slot, stage_count, stage, o, i, level);
      auto cached = diagonal_cache_.find(key);
      if (cached == diagonal_cache_.end()) {
        const cvec factor = rotate_vector(twiddle[pmod(index, count)], -factor_delta);
        std::vector<double> re(factor.size()), im(factor.size());
        for (size_t s = 0; s < factor.size(); s++) {
          re[s] = factor[s].real();
          im[s] = factor[s].imag();
        }
        auto pt = encode(re.data(), im.data(), static_cast<int>(factor.size()), level);
        cached = diagonal_cache_.emplace(key, prepare_for_multiply(*pt, level)).first;
      }
      // multiply(ct, encoded diagonal): CKKSCore::multiply(ct, pt) (core.cpp:257-282).
      const Data &p = *cached->second;
      auto c = prepare_for_multiply(*rotated[i], level);
      auto product = make_data(kUnitCiphertext, (c->flag | p.flag) & ~kFlagRescaled, c->moduli_id,
                               c->polys, c->scale * p.scale);
      const long long ps = c->poly_stride();
      for (int q = 0; q < c->polys; q++)
        pointwise(kOpMult, c->chains, c->moduli_id, c->d + q * ps, p.d, nullptr,
                  product->d + q * ps);
      if (!inner_sum)
        inner_sum = std::move(product);
      else
        add_inplace(*inner_sum, *product);
    }
    auto turned = rotate(*inner_sum, keys, factor_delta);
    if (!outer_sum)
      outer_sum = std::move(turned);
    else
      add_inplace(*outer_sum, *turned);
  }
  return outer_sum;
}

std::pair<std::unique_ptr<Data>, std::unique_ptr<Data>> Engine::coeff_to_slot(
    const Data &ct, const Data &conjugation_key, const std::vector<const Data *> &keys,
    int stage_count) {
  // engine_bootstrap.cpp:331-371.
  const int slot = params.slot_count, log_slot = params.log_slot_count;
  int rotate_count = slot;
  Owned current;
  for (int stage = 0; stage < stage_count; stage++) {
    rotate_count >>= cts_log_radix(stage, stage_count, log_slot);
    current = apply_butterfly(current ? *current : ct, true, stage_count, stage, keys, rotate_count);
  }
  auto conjugated = conjugate(*current, conjugation_key);
  auto real_part = add(*current, *conjugated);
  auto difference = subtract(*current, *conjugated);
  auto imaginary_part = multiply_imaginary(*difference, -1);
  return {std::move(real_part), std::move(imaginary_part)};
}

std::unique_ptr<Data> Engine::slot_to_coeff(const Data &real_part, const Data &imaginary_part,
                                            const std::vector<const Data *> &keys,
                                            int stage_count) {
  // engine_bootstrap.cpp:405-434.
  const int log_slot = params.log_slot_count;
  auto multiplied = multiply_imaginary(imaginary_part, 1);
  auto current = add(real_part, *multiplied);
  int rotate_count = 1;
  for (int stage = 0; stage < stage_count; stage++) {
    current = apply_butterfly(*current, false, stage_count, stage, keys, rotate_count);
    rotate_count <<= stc_log_radix(stage, stage_count, log_slot);
  }
  return current;
}

std::unique_ptr<Data> Engine::chebyshev_ps(const std::vector<const Data *> &baby,
                                           const Data &giant, const Data *rk,
                                           const std::vector<std::vector<double>> &coefficients) {
  // chebyshev_paterson_stockmeyer (engine_bootstrap.cpp:459-498).
  auto baby0 = weighted_sum(baby, coefficients[0]);
  auto added = add(giant, *baby0);
  auto baby1 = weighted_sum(baby, coefficients[1]);
  auto multiplied = rk ? multiply_relinearize(*added, *baby1, *rk) : multiply(*added, *baby1);
  auto baby2 = weighted_sum(baby, coefficients[2]);
  return add(*multiplied, *baby2);
}

std::unique_ptr<Data> Engine::sine(const Data &ct, const Data &rk) {
  // CKKSEngine::sine (engine_bootstrap.cpp:526-638).
  std::vector<Owned> baby(kBabyDegree);
  baby[0] = clone(ct);
  for (int bi = 2; bi <= kBabyDegree; bi++) {
    const int basis = bi - 1, half = bi / 2 - 1;
    if ((bi & 1) == 0) {
      auto m = square(*baby[half], &rk);
      add_inplace(*m, *m);
      baby[basis] = add_scalar(*m, -1);
    } else {
      auto m = multiply_relinearize(*baby[half], *baby[half + 1], rk);
      add_inplace(*m, *m);
      baby[basis] = subtract(*m, *baby[0]);
    }
  }
  const int destination = baby.back()->level();
  for (int bi = 0; bi < kBabyDegree - 2; bi++)
    if (baby[bi]->level() > destination) baby[bi] = level_down(*baby[bi], destination);

  std::vector<Owned> giant(kGiantDegree);
  giant[0] = clone(*baby.back());
  for (int gi = 1; gi < kGiantDegree; gi++) {
    auto m = square(*giant[gi - 1], &rk);
    add_inplace(*m, *m);
    giant[gi] = add_scalar(*m, -1);
  }
  Owned ps = clone(*giant[0]);
  for (int gi = 1; gi < kGiantDegree - 1; gi++) {
    auto m = multiply_relinearize(*ps, *giant[gi], rk);
    add_inplace(*m, *m);
    ps = subtract(*m, *giant[0]);
  }
  {
    auto m = multiply(*ps, *giant[kGiantDegree - 1]);
    add_inplace(*m, *m);
    ps = subtract(*m, *giant[0]);
  }
  std::vector<const Data *> basis;
  for (auto &b : baby) basis.push_back(b.get());
  auto auxiliary = weighted_sum(basis, kAuxiliary);
  auto added = add(*auxiliary, *giant.back());
  auto quotient = chebyshev_ps(basis, *giant[kGiantDegree - 2], &rk, kQuotient);
  auto multiplied = multiply(*added, *quotient);
  auto remainder = chebyshev_ps(basis, *giant[kGiantDegree - 2], nullptr, kRemainder);
  auto sum = add(*multiplied, *remainder);
  auto difference = subtract(*sum, *ps);
  return relinearize(*difference, rk);
}

std::unique_ptr<Data> Engine::round_to_integer(const Data &ct, const Data &rk) {
  // round = x * ROUND_BOUND - modulo(x), modulo = three double-angle steps on the
  // sine approximation (engine_bootstrap.cpp:640-692).
  auto current = sine(ct, rk);
  const double two_pi = 2 * kPi;
  const int iterations = 3;
  for (int it = 1; it <= iterations; it++) {
    auto m = square(*current, &rk);
    add_inplace(*m, *m);
    const double scalar = -std::pow(two_pi, -std::pow(2, it - iterations));
    current = add_scalar(*m, scalar);
  }
  auto multiplied = multiply_integer(ct, kRoundBound);
  return subtract(*multiplied, *current);
}

std::unique_ptr<Data> Engine::make_signed_tile(const Data &ct) {
  // CKKSCore::make_signed_tile (core.cpp:1085-1108): make_signed at the text's first
  // prime (unsigned comparison with q/2), tiled onto the key-switching level's chain.
  const int mid = params.moduli_id(params.max_key_switching_level());
  const int L = params.chains(mid);
  const long double scale = static_cast<long double>(params.scale * params.scale);
  auto out = make_data(kUnitCiphertext, ct.flag & ~kFlagRescaled, mid, 2, scale);
  const int64_t q = static_cast<int64_t>(params.q[ct.moduli_id]);
  signed_tile(ct.d, q, L, mid, out->d, params.n);
  signed_tile(ct.d + ct.poly_stride(), q, L, mid, out->d + out->poly_stride(), params.n);
  return out;
}

std::unique_ptr<Data> Engine::mod_raise(const Data &ct, const Data &to_sparse, const Data &to_dense) {
  // CKKSEngine::mod_raise_ (engine_mod_raise.cpp:5-31) with get_mod_raise_ratio
  // (core.cpp:1110-1117).
  auto rescaled = rescale_any(ct);
  auto sparse = switch_key(*rescaled, to_sparse);
  auto tiled = make_signed_tile(*sparse);
  auto dense = switch_key(*tiled, to_dense);
  const double scale = params.scale;
  const double partial_sum_ratio = 1 << (params.log_n - params.log_slot_count - 1);
  const double base_prime = static_cast<double>(params.base_prime());
  const int64_t ratio =
      static_cast<int64_t>(std::round(scale * scale / (partial_sum_ratio * base_prime)));
  return multiply_integer(*dense, ratio);
}

std::pair<std::unique_ptr<Data>, std::unique_ptr<Data>> Engine::create_small_bootstrap_key(
    const Data &sk) {
  // CKKSEngine::create_small_bootstrap_key (engine.cpp:141-160): key switching to a
  // sparse secret (Hamming weight 128) at level 0, and back at the key-switching level.
  if (!params.preset.bootstrap)
    throw std::runtime_error("Create Small Bootstrap Key: the engine is not for bootstrapping.");
  auto sparse = create_sparse_secret_key(128, params.max_level());
  auto to_sparse = create_key_switching_key(sk, *sparse, 0, kKeySwitchingKey);
  auto to_dense =
      create_key_switching_key(*sparse, sk, params.max_key_switching_level(), kKeySwitchingKey);
  return {std::move(to_sparse), std::move(to_dense)};
}

std::unique_ptr<Data> Engine::bootstrap(const Data &ct, const Data &rk, const Data &ck,
                                        const std::vector<const Data *> &keys,
                                        const Data &to_sparse, const Data &to_dense,
                                        int stage_count) {
  // CKKSEngine::bootstrap(UnitCiphertext*, RelinearizationKey*, ConjugationKey*,
  // RotationKey*, SmallBootstrapKey*, int) (engine_bootstrap.cpp:712-754).
  const std::string fn = "Bootstrap Unit Ciphertext With Rotation Key";
  if (!params.preset.bootstrap)
    throw std::runtime_error(fn + ": the engine is not for bootstrapping.");
  if (ct.polys != 2)
    throw std::runtime_error(fn + ": the input unit ciphertext should have 2 polynomials.");
  if (ct.is_ntt())
    throw std::runtime_error(fn + ": the input unit ciphertext should not be in NTT form.");
  require_bootstrap_stage_count(fn, stage_count, 0);
  auto leveled = level_down(ct, 0);
  auto raised = mod_raise(*leveled, to_sparse, to_dense);
  if (params.log_slot_count != params.log_n - 1) {
    // partial_sum_inplace (engine_bootstrap.cpp:315-329): deltas normalised by N/2.
    for (int delta = params.slot_count; delta < params.n / 2; delta <<= 1) {
      auto turned = rotate(*raised, keys, delta, false);
      add_inplace(*raised, *turned);
    }
  }
  auto [slot_real, slot_imag] = coeff_to_slot(*raised, ck, keys, stage_count);
  auto rounded_real = round_to_integer(*slot_real, rk);
  auto rounded_imag = round_to_integer(*slot_imag, rk);
  auto coeff = slot_to_coeff(*rounded_real, *rounded_imag, keys, stage_count);
  auto bootstrapped = subtract(*raised, *coeff);
  const int64_t ratio =
      static_cast<int64_t>(std::round(static_cast<double>(params.base_prime()) / params.scale));
  return multiply_integer(*bootstrapped, ratio);
}

// ------------------------------------------- bootstrap key (hoisted BSGS) --

size_t BootstrapKey::bytes() const {
  size_t total = 0;
  auto add = [&](const Data *d) {
    if (d) total += d->words() * sizeof(int64_t);
  };
  for (const auto &kv : rotation_keys) add(kv.second.get());
  for (const auto *stages : {&coeff_to_slot, &slot_to_coeff})
    for (const auto &stage : *stages)
      for (const auto &row : stage.diagonals)
        for (const auto &entry : row.second) add(entry.second.get());
  add(to_sparse.get());
  add(to_dense.get());
  return total;
}

void Engine::require_bootstrap_stage_count(const std::string &fn, int stage_count,
                                           int inner_loop_shift) const {
  // CKKSEngine::require_bootstrap_stage_count (engine_require.cpp:1018-1100): the
  // admissible stage counts per slot count and inner loop shift.
  int lo = 3, hi = 5;
  bool invalid = false;
  const int ls = params.log_slot_count;
  if (inner_loop_shift == 0) {
    if (ls >= 1 && ls <= 3) lo = 1, hi = 1;
    else if (ls <= 5 && ls >= 4) lo = 1, hi = 2;
    else if (ls == 6) lo = 2, hi = 2;
    else if (ls >= 7 && ls <= 9) lo = 2, hi = 3;
    else if (ls == 10) lo = 2, hi = 4;
    else if (ls == 11 || ls == 12) lo = 3, hi = 4;
    else if (ls == 13 || ls == 14) lo = 3, hi = 5;
  } else if (inner_loop_shift == 1) {
    if (ls == 1 || ls == 2) invalid = true;
    else if (ls >= 3 && ls <= 5) lo = 1, hi = 1;
    else if (ls >= 6 && ls <= 8) lo = 2, hi = 2;
    else if (ls == 9 || ls == 10) lo = 2, hi = 3;
    else if (ls == 11) lo = 3, hi = 3;
    else if (ls >= 12 && ls <= 14) lo = 3, hi = 4;
  }
  if (invalid || stage_count < lo || stage_count > hi)
    throw std::runtime_error(fn + ": invalid stage count.");
}

void Engine::make_bootstrap_stage(BootstrapStage &stage, const std::vector<cvec> &twiddles,
                                  int rotate_count, int level, int inner_loop_shift) {
  // make_bootstrap_stage (engine_bootstrap.cpp:8-67): loop deltas, the order in which
  // equal outer deltas are summed, and every diagonal encoded with the special
  // primes at the stage's level, rescaled and put in NTT form.
  const int count = static_cast<int>(twiddles.size());
  const auto [inner, outer] = stage_loop_counts(count, inner_loop_shift);
  stage.level = level;
  stage.inner = inner;
  stage.outer = outer;
  stage.inner_deltas.assign(1, 0);
  for (int i = 1; i < inner; i++) stage.inner_deltas.push_back(normalized_delta(i * rotate_count));
  for (int o = 0; o < outer; o++) {
    const int norm_o = o - outer / 2;
    const int delta = normalized_delta(inner * norm_o * rotate_count);
    stage.outer_deltas.push_back(delta);
    bool fresh = true;
    for (auto &entry : stage.process_order)
      if (entry.first == delta) {
        entry.second.push_back(o);
        fresh = false;
        break;
      }
    if (fresh) stage.process_order.push_back({delta, {o}});
    auto &row = stage.diagonals[o];
    for (int i = (o == 0 ? 1 : 0); i < inner; i++) {
      const cvec factor = rotate_vector(twiddles[pmod(inner * norm_o + i, count)], -delta);
      std::vector<double> re(factor.size()), im(factor.size());
      for (size_t k = 0; k < factor.size(); k++) {
        re[k] = factor[k].real();
        im[k] = factor[k].imag();
      }
      auto encoded = encode(re.data(), im.data(), static_cast<int>(factor.size()), level, true);
      auto rescaled = rescale_any(*encoded);
      row[i] = to_ntt(*rescaled);
    }
  }
}

std::unique_ptr<BootstrapKey> Engine::create_bootstrap_key(const Data &sk, int stage_count,
                                                           const std::string &size) {
  // CKKSEngine::create_bootstrap_key (engine.cpp:162-215).
  const std::string fn = "Create Bootstrap Key";
  if (!params.preset.bootstrap)
    throw std::runtime_error(fn + ": the engine is not for bootstrapping.");
  if (sk.type != kSecretKey) throw std::invalid_argument(fn + ": the key is not a secret key.");
  if (sk.level() < params.max_key_switching_level())
    throw std::runtime_error(fn + ": the target level cannot be reached with the provided keys.");
  std::string lower = size;
  std::transform(lower.begin(), lower.end(), lower.begin(),
                 [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
  int shift;
  if (lower == "medium")
    shift = 0;
  else if (lower == "large")
    shift = 1;
  else
    throw std::runtime_error(fn + ": invalid size.");
  require_bootstrap_stage_count(fn, stage_count, shift);

  auto bk = std::make_unique<BootstrapKey>();
  bk->serial = ++serial_;
  bk->stage_count = stage_count;
  bk->inner_loop_shift = shift;
  // get_bootstrap_stage_levels (engine_bootstrap.cpp:121-130): nine levels for EvalRound.
  const int max_level = params.max_key_switching_level();
  const int cts_level = max_level;
  const int stc_level = max_level - stage_count - 9;
  const int slot = params.slot_count, log_slot = params.log_slot_count;

  const auto &cts = bootstrap_twiddles(true, stage_count);
  bk->coeff_to_slot.resize(stage_count);
  int rotate_count = slot;
  for (int s = 0; s < stage_count; s++) {
    rotate_count >>= cts_log_radix(s, stage_count, log_slot);
    make_bootstrap_stage(bk->coeff_to_slot[s], cts[s], rotate_count, cts_level - s, shift);
  }
  const auto &stc = bootstrap_twiddles(false, stage_count);
  bk->slot_to_coeff.resize(stage_count);
  rotate_count = 1;
  for (int s = 0; s < stage_count; s++) {
    make_bootstrap_stage(bk->slot_to_coeff[s], stc[s], rotate_count, stc_level - s, shift);
    rotate_count <<= stc_log_radix(s, stage_count, log_slot);
  }

  // Rotation contexts in the reference's order (the random stream sees the same
  // sequence of key generations): partial sums, then each stage's inner and outer
  // deltas; a delta gets its key at the first level that needs it.
  auto add_keys = [&](const std::vector<int> &deltas, int level, bool by_slot_count) {
    for (int delta : deltas) {
      if (delta == 0 || bk->rotation_keys.count(delta)) continue;
      const int nd = normalized_delta(delta, by_slot_count);
      bk->rotation_keys[delta] = create_fixed_rotation_key(sk, nd, level);
    }
  };
  std::vector<int> partial;
  for (int d = slot; d < params.n / 2; d <<= 1) partial.push_back(d);
  add_keys(partial, max_level, false);
  for (const auto *stages : {&bk->coeff_to_slot, &bk->slot_to_coeff})
    for (const auto &stage : *stages) {
      add_keys(stage.inner_deltas, stage.level, true);
      add_keys(stage.outer_deltas, stage.level, true);
    }
  auto small = create_small_bootstrap_key(sk);
  bk->to_sparse = std::move(small.first);
  bk->to_dense = std::move(small.second);
  return bk;
}

void Engine::decompose_into(const int64_t *x, int moduli_id, int64_t *out) {
  const int n = params.n;
  const DevicePartitions &dp = partitions(moduli_id, moduli_id);
  int64_t *digits = alloc_words(static_cast<size_t>(params.chains(moduli_id)) * n);
  cudaError_t e = timed("mixed_radix", [&] {
    return launch_mixed_radix(tables_, dp, n, moduli_id, x, digits, stream_);
  });
  if (e == cudaSuccess) e = mod_up(dp, moduli_id, digits, out);
  free_words(digits);
  check(e, "decompose");
}

void Engine::mod_down_polys(int64_t *extended, int moduli_id, int polys, int64_t *out) {
  const int L = params.chains(moduli_id), E = params.chains(moduli_id, true);
  cudaError_t e = mod_down_transform(moduli_id, E, extended, polys);
  if (e == cudaSuccess) {
    EpilogueOps ops;
    ops.polys = polys;
    e = mod_down_epilogue(moduli_id, L, extended, ops, out);
  }
  check(e, "mod down");
}

std::unique_ptr<Data> Engine::decompose(const Data &ct) {
  // CKKSCore::decompose (core_key_switch.cpp:434-466): polynomial 1 of a
  // coefficient-form text, every partition raised to the extended chain, NTT form.
  if (ct.polys < 2 || (ct.flag & kFlagSpecial))
    throw std::invalid_argument("decompose: the input should be a ciphertext without special primes.");
  const int m = ct.moduli_id;
  const DevicePartitions &dp = partitions(m, m);
  auto out = make_data(kDecomposed, ct.flag | kFlagNtt | kFlagSpecial, m, dp.count, ct.scale);
  decompose_into(ct.d + ct.poly_stride(), m, out->d);
  return out;
}

std::unique_ptr<Data> Engine::mod_down_then_decompose(Data &ct) {
  // CKKSCore::mod_down_then_decompose (core_key_switch.cpp:468-508): polynomial 1 of
  // an extended NTT-form text brought down to its chain, then decomposed.  The
  // ModDown works in place: polynomial 1 of `ct` is clobbered (its caller keeps only
  // polynomial 0).
  const int m = ct.moduli_id, n = params.n;
  const DevicePartitions &dp = partitions(m, m);
  auto out = make_data(kDecomposed, ct.flag, m, dp.count, ct.scale);
  int64_t *reduced = alloc_words(static_cast<size_t>(params.chains(m)) * n);
  try {
    mod_down_polys(ct.d + ct.poly_stride(), m, 1, reduced);
    decompose_into(reduced, m, out->d);
  } catch (...) {
    free_words(reduced);
    throw;
  }
  free_words(reduced);
  return out;
}

std::unique_ptr<Data> Engine::attach_special_primes(const Data &text) {
  // attach_special_prime_chains_ (core.cpp:1127-1155): x * P on the chain, zero
  // special limbs, then to_ntt_ over the extended chain.
  if (text.flag & kFlagSpecial)
    throw std::invalid_argument("attach special primes: the text already has them.");
  if (text.is_ntt()) throw std::invalid_argument("attach special primes: the text is in NTT form.");
  const int m = text.moduli_id, L = text.chains;
  auto out = make_data(text.type, text.flag | kFlagNtt | kFlagSpecial, m, text.polys, text.scale);
  check(timed("attach_special_ntt", [&] {
          return launch_attach_special_ntt(tables_, ks_, params.log_n, text.polys, L, m, text.d,
                                           text.poly_stride(), out->d, out->poly_stride(),
                                           stream_);
        }),
        "attach special primes");
  return out;
}

std::unique_ptr<Data> Engine::remove_special_primes(const Data &text) {
  // remove_special_prime_chains_ (core.cpp:1165-1187): ModDown of every polynomial,
  // on a copy (the ModDown works in place).
  auto copy = clone(text);
  return remove_special_primes_in_place(*copy);
}

std::unique_ptr<Data> Engine::remove_special_primes_in_place(Data &text) {
  if (!(text.flag & kFlagSpecial) || !text.is_ntt() || text.polys > 2)
    throw std::invalid_argument("remove special primes: the text has no special primes.");
  const int m = text.moduli_id;
  auto out = make_data(text.type, text.flag & ~(kFlagNtt | kFlagSpecial), m, text.polys,
                       text.scale);
  mod_down_polys(text.d, m, text.polys, out->d);
  return out;
}

std::unique_ptr<Data> Engine::core_ntt_rotate(const Data &ct, const Data &decomposed,
                                              const Data &key, int delta) {
  // CKKSCore::ntt_rotate (core.cpp:965-1000): the key switcher of the decomposition
  // (create_key_switcher, core_key_switch.cpp:510-548), polynomial 0 added, both
  // permuted in NTT form.
  const int m = ct.moduli_id, n = params.n;
  if (key.moduli_id > m)
    throw std::runtime_error("the fixed rotation key was created at a lower level than the text.");
  const DevicePartitions &dp = partitions(m, key.moduli_id);
  if (dp.count != decomposed.polys || decomposed.moduli_id != m || ct.chains != decomposed.chains)
    throw std::invalid_argument("ntt rotate: the decomposition does not match the text.");
  if (key.polys < 2 * (dp.max_key_index + 1))
    throw std::invalid_argument("the key switching key has too few polynomials.");
  int64_t *acc = alloc_words(static_cast<size_t>(2) * ct.chains * n);
  auto out = make_data(kUnitCiphertext, decomposed.flag, m, 2, ct.scale);
  cudaError_t e = timed("key_inner_product", [&] {
    return launch_key_inner_product(tables_, dp, n, m, decomposed.d, key.d, key.chains,
                                    m - key.moduli_id, acc, stream_);
  });
  if (e == cudaSuccess) {
    const int32_t *perm = device_ntt_permutation(delta);
    e = timed("ntt_rotate", [&] {
      return launch_ntt_rotate_finish(tables_, params.log_n, ct.chains, m, ct.d, acc, perm, out->d,
                                      stream_);
    });
  }
  free_words(acc);
  check(e, "ntt rotate");
  return out;
}

namespace {
const Data &rotation_context(const std::string &fn, const BootstrapKey &bk, int delta) {
  // get_rotation_context (engine_rotate.cpp:172-184).
  auto it = bk.rotation_keys.find(delta);
  if (it == bk.rotation_keys.end())
    throw std::runtime_error(fn + ": the bootstrap key does not contain a rotation context for delta " +
                             std::to_string(delta) + ".");
  return *it->second;
}
}  // namespace

std::unique_ptr<Data> Engine::ntt_rotate(const Data &ct, const Data &decomposed,
                                         const BootstrapKey &bk, int delta) {
  // CKKSEngine::ntt_rotate / ntt_rotate_ (engine_rotate.cpp:223-259).
  const std::string fn = "Rotate Unit Ciphertext in NTT Form with Bootstrap Key";
  if (ct.polys != 2)
    throw std::runtime_error(fn + ": the input unit ciphertext should have 2 polynomials.");
  if (!ct.is_ntt())
    throw std::runtime_error(fn + ": the input unit ciphertext should be in NTT form.");
  if (ct.level() != decomposed.level())
    throw std::runtime_error(fn + ": the levels of the inputs do not match.");
  const int nd = normalized_delta(delta);
  if (nd == 0) return clone(ct);
  return core_ntt_rotate(ct, decomposed, rotation_context(fn, bk, nd), nd);
}

std::unique_ptr<Data> Engine::rotate(const Data &ct, const BootstrapKey &bk, int delta,
                                     bool normalize_by_slot_count) {
  const std::string fn = "Rotate Unit Ciphertext with Bootstrap Key";
  const int nd = normalized_delta(delta, normalize_by_slot_count);
  if (nd == 0) return clone(ct);
  return rotate(ct, rotation_context(fn, bk, nd));
}

std::vector<Owned> Engine::bsgs_inner_sums(const Data &x, const Data &decomposed,
                                           const BootstrapKey &bk, const BootstrapStage &stage) {
  // The limits of bsgs.cu (up to 16 inner texts, 8 outer indices, 8 partitions);
  // outside them, or with a rotation the unfused path would refuse, the caller runs
  // the unfused path, which also raises its errors.  One sum per process-order
  // entry; the outer indices of an entry are consecutive kernel groups.
  const int m = x.moduli_id, n = params.n;
  if (!fused_bsgs_ || stage.inner < 1 || stage.inner > kBsgsMaxInner ||
      stage.process_order.empty() || x.polys != 2 || decomposed.moduli_id != m ||
      decomposed.chains != x.chains || decomposed.polys > kBsgsMaxPartitions ||
      static_cast<int>(stage.inner_deltas.size()) != stage.inner)
    return {};
  BsgsInner b;
  b.inner = stage.inner;
  for (int i = 1; i < stage.inner; i++) {
    const int nd = normalized_delta(stage.inner_deltas[i]);
    auto it = bk.rotation_keys.find(nd);
    if (nd == 0 || it == bk.rotation_keys.end()) return {};
    const Data &key = *it->second;
    if (key.moduli_id > m) return {};
    const DevicePartitions &dp = partitions(m, key.moduli_id);
    if (dp.count != decomposed.polys || key.polys < 2 * (dp.max_key_index + 1)) return {};
    const auto parts = params.partitions(m, key.moduli_id);
    const long long kp = key.chains, vo = m - key.moduli_id;
    for (int p = 0; p < dp.count; p++) {
      const long long off = (2LL * parts[p].partition_index * kp + vo) * n;
      if (off + kp * n > INT32_MAX) return {};
      b.key_off[i][p] = static_cast<int32_t>(off);
    }
    b.key_poly[i] = static_cast<int32_t>(kp * n);
    b.perm[i] = device_ntt_permutation(nd);
    b.key[i] = key.d;
  }
  std::vector<Owned> sums;
  int g = 0;  // kernel group: one outer index
  for (size_t e = 0; e < stage.process_order.size(); e++) {
    b.lead |= 1u << g;
    for (int o : stage.process_order[e].second) {
      if (g == kBsgsMaxGroups) return {};
      const auto row = stage.diagonals.find(o);
      if (row == stage.diagonals.end()) return {};
      for (int i = (o == 0 ? 1 : 0); i < stage.inner; i++) {
        const auto cell = row->second.find(i);
        if (cell == row->second.end()) return {};
        const Data &diagonal = *cell->second;
        if (diagonal.moduli_id != m || diagonal.chains != x.chains) return {};
        b.diag[i][g] = diagonal.d;
        b.mask[i] |= 1u << g;
        if (sums.size() == e)  // the unfused path's inner_sum, made at the entry's first term
          sums.push_back(make_data(kUnitCiphertext, (x.flag | diagonal.flag) & ~kFlagRescaled, m,
                                   2, x.scale * diagonal.scale));
      }
      if (sums.size() != e + 1) return {};
      b.out[g] = sums.back()->d;
      g++;
    }
  }
  b.groups = g;
  check(timed("bsgs_inner", [&] {
          return launch_bsgs_inner(tables_, params.log_n, m, x.chains, decomposed.polys, x.d,
                                   x.poly_stride(), decomposed.d, b, stream_);
        }),
        "apply butterfly");
  return sums;
}

std::unique_ptr<Data> Engine::apply_butterfly(const Data &ct, const BootstrapKey &bk,
                                              const BootstrapStage &stage) {
  // CKKSEngine::apply_butterfly(ct, bootstrap key, stage) (engine_bootstrap.cpp:216-291):
  // one decomposition serves every inner rotation; the diagonal products of each
  // outer group are summed in the extended domain and rotated once.  The inner loop
  // runs as one fused kernel where bsgs_inner_sums covers the stage.
  if (ct.level() <= 0)
    throw std::runtime_error(
        "Rescale Unit Ciphertext: the input unit ciphertext should have a positive level.");
  Owned inner0;
  std::vector<Owned> rotated;
  std::vector<Owned> fused;
  {
    auto rescaled = rescale_any(ct);
    auto decomposed = decompose(*rescaled);
    inner0 = attach_special_primes(*rescaled);
    fused = bsgs_inner_sums(*inner0, *decomposed, bk, stage);
    if (fused.empty()) {
      for (int delta : stage.inner_deltas) {
        if (delta == 0) continue;
        rotated.push_back(ntt_rotate(*inner0, *decomposed, bk, delta));
      }
    }
  }
  auto inner_text = [&](int i) -> const Data & { return i == 0 ? *inner0 : *rotated[i - 1]; };
  Owned outer_sum;
  for (size_t gi = 0; gi < stage.process_order.size(); gi++) {
    const auto &[delta, outer_indices] = stage.process_order[gi];
    // multiply_for_butterfly (CKKSCore::multiply(ct, pt), core.cpp:257-282) of every
    // (text, diagonal) pair of the group, summed with add_inplace: one fused pass per
    // kMaxMacTerms pairs.
    Owned inner_sum;
    if (!fused.empty()) inner_sum = std::move(fused[gi]);
    MacTerms terms;
    bool continued = false;  // a previous pass already started the chain in inner_sum
    auto flush = [&]() {
      if (terms.count == 0) return;
      const Data &x = *inner_sum;
      check(timed("diagonal_mac", [&] {
              return launch_diagonal_mac(tables_, params.log_n, x.chains, x.moduli_id, terms,
                                         x.poly_stride(), continued, inner_sum->d,
                                         x.poly_stride(), stream_);
            }),
            "diagonal products");
      terms.count = 0;
      continued = true;
    };
    for (int o : fused.empty() ? outer_indices : std::vector<int>{}) {
      const auto &row = stage.diagonals.at(o);
      for (int i = (o == 0 ? 1 : 0); i < stage.inner; i++) {
        const Data &x = inner_text(i);
        const Data &diagonal = *row.at(i);
        if (diagonal.moduli_id != x.moduli_id || diagonal.chains != x.chains || x.polys != 2)
          throw std::runtime_error("apply butterfly: the diagonal does not match the text.");
        if (!inner_sum)
          inner_sum = make_data(kUnitCiphertext, (x.flag | diagonal.flag) & ~kFlagRescaled,
                                x.moduli_id, x.polys, x.scale * diagonal.scale);
        if (terms.count == kMaxMacTerms) flush();
        terms.x[terms.count] = x.d;
        terms.d[terms.count] = diagonal.d;
        terms.count++;
      }
    }
    flush();
    Owned turned = std::move(inner_sum);
    if (delta != 0) {
      auto decomposed = mod_down_then_decompose(*turned);
      turned = ntt_rotate(*turned, *decomposed, bk, delta);
    }
    if (!outer_sum)
      outer_sum = std::move(turned);
    else
      add_inplace(*outer_sum, *turned);
  }
  return remove_special_primes_in_place(*outer_sum);
}

std::unique_ptr<Data> Engine::bootstrap(const Data &ct, const Data &rk, const Data &ck,
                                        const BootstrapKey &bk) {
  auto out = run_captured({kGraphBootstrap, rk.serial, ck.serial, bk.serial}, {&ct},
                          [&](const std::vector<const Data *> &in) {
                            std::vector<Owned> r;
                            r.push_back(bootstrap_direct(*in[0], rk, ck, bk));
                            return r;
                          });
  return std::move(out[0]);
}

std::unique_ptr<Data> Engine::bootstrap_direct(const Data &ct, const Data &rk, const Data &ck,
                                               const BootstrapKey &bk) {
  // CKKSEngine::bootstrap(UnitCiphertext*, RelinearizationKey*, ConjugationKey*,
  // BootstrapKey*) (engine_bootstrap.cpp:804-838).
  const std::string fn = "Bootstrap Unit Ciphertext With Bootstrap Key";
  if (!params.preset.bootstrap)
    throw std::runtime_error(fn + ": the engine is not for bootstrapping.");
  if (ct.polys != 2)
    throw std::runtime_error(fn + ": the input unit ciphertext should have 2 polynomials.");
  if (ct.is_ntt())
    throw std::runtime_error(fn + ": the input unit ciphertext should not be in NTT form.");
  if (!bk.to_sparse || !bk.to_dense || static_cast<int>(bk.coeff_to_slot.size()) != bk.stage_count ||
      static_cast<int>(bk.slot_to_coeff.size()) != bk.stage_count)
    throw std::invalid_argument(fn + ": the bootstrap key is incomplete.");
  auto leveled = level_down(ct, 0);
  auto raised = mod_raise(*leveled, *bk.to_sparse, *bk.to_dense);
  if (params.log_slot_count != params.log_n - 1) {
    // partial_sum_inplace with the bootstrap key (engine_bootstrap.cpp:298-313).
    for (int delta = params.slot_count; delta < params.n / 2; delta <<= 1) {
      auto turned = rotate(*raised, bk, delta, false);
      add_inplace(*raised, *turned);
    }
  }
  // coeff_to_slot with the bootstrap key (engine_bootstrap.cpp:370-400).
  Owned current;
  for (const auto &stage : bk.coeff_to_slot)
    current = apply_butterfly(current ? *current : *raised, bk, stage);
  auto conjugated = conjugate(*current, ck);
  auto real_part = add(*current, *conjugated);
  auto subtracted = subtract(*current, *conjugated);
  auto imaginary_part = multiply_imaginary(*subtracted, -1);
  current.reset();
  conjugated.reset();
  subtracted.reset();
  auto rounded_real = round_to_integer(*real_part, rk);
  auto rounded_imag = round_to_integer(*imaginary_part, rk);
  // slot_to_coeff with the bootstrap key (engine_bootstrap.cpp:436-452).
  auto multiplied = multiply_imaginary(*rounded_imag, 1);
  current = add(*rounded_real, *multiplied);
  for (const auto &stage : bk.slot_to_coeff) current = apply_butterfly(*current, bk, stage);
  auto bootstrapped = subtract(*raised, *current);
  const int64_t ratio =
      static_cast<int64_t>(std::round(static_cast<double>(params.base_prime()) / params.scale));
  return multiply_integer(*bootstrapped, ratio);
}

}  // namespace fhe_b200
