// CKKS bootstrapping with a rotation key (DESILO FHE ckks/engine_bootstrap.cpp,
// engine_mod_raise.cpp, operation/bootstrap.cpp): mod raise through a sparse secret,
// coefficients-to-slots butterflies, EvalRound (sine by Chebyshev
// Paterson-Stockmeyer and three double-angle steps), slots-to-coefficients, and the
// final correction.  Every step is an engine operation already on the device; this
// file composes them in the reference's order so each intermediate word matches,
// and builds the butterfly twiddles on the host with the reference's expressions.
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

std::pair<int, int> stage_loop_counts(int twiddle_count) {
  // get_stage_loop_counts (operation/bootstrap.cpp:265-278), inner shift 0.
  int bits = 0;
  for (int t = twiddle_count; t > 0; t >>= 1) bits++;
  const int inner = 1 << ((bits + 1) / 2);
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
  if (stage_count < 1 || stage_count > params.log_slot_count)
    throw std::runtime_error(fn + ": the stage count is not supported.");
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

}  // namespace fhe_b200
