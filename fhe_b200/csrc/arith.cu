// Ciphertext arithmetic of the engine: addition, subtraction, negation, products
// with plaintexts and scalars, squaring (DESILO FHE ckks/engine_add.cpp,
// engine_subtract.cpp, engine_multiply.cpp, engine_negate.cpp and the CKKSCore
// operations of ckks/core.cpp:196-712).  Every limb operation runs in the element-wise
// kernel of keygen.cu; this file holds the level / form matching and the scalar
// constants, which follow the reference's double arithmetic.
#include <cmath>

#include "engine.hpp"

namespace fhe_b200 {

namespace {

// floor(|x|) * 2^extra mod q: BigInt::from_double(std::abs(x)) (big_int.cpp:30-44)
// truncates the fraction and keeps every integer bit of a large double.
int64_t floor_abs_mod(double x, uint64_t q, int extra) {
  const double a = std::fabs(x);
  unsigned __int128 v;
  int shift = extra;
  if (a < 18446744073709551616.0) {
    v = static_cast<unsigned __int128>(static_cast<uint64_t>(a)) % q;
  } else {
    int e = 0;
    const double m = std::frexp(a, &e);
    v = static_cast<unsigned __int128>(static_cast<uint64_t>(std::ldexp(m, 53))) % q;
    shift += e - 53;
  }
  for (; shift > 0; shift--) v = (v << 1) % q;
  return static_cast<int64_t>(v);
}

}  // namespace

struct Engine::Matched {
  std::unique_ptr<Data> own_a, own_b;
  const Data *a = nullptr;
  const Data *b = nullptr;
};

std::vector<int64_t> Engine::add_multiplier(double value, int level) const {
  // make_add_multiplier (precomputed.cpp:476-498) with scale_modulo
  // (arithmetic.cpp:60-76).
  const int mid = params.moduli_id(level);
  const int L = params.chains(mid);
  double deviation = static_cast<double>(params.deviations[level]);
  if (params.preset.one_more_level && mid == 0) deviation = params.q[mid] / params.scale;
  const double scale = params.scale;
  const double product = (value * scale * deviation + 0.5) * scale;
  std::vector<int64_t> out(L);
  for (int j = 0; j < L; j++) {
    const uint64_t q = params.q[mid + j];
    int64_t s = floor_abs_mod(product, q, 0);
    if (product < 0) s = static_cast<int64_t>(q) - s;
    out[j] = s;
  }
  return out;
}

std::vector<int64_t> Engine::mult_multiplier(double value, int level) const {
  // make_mult_multiplier(double, level) (precomputed.cpp:499-517) with
  // scale_enter_modulo (arithmetic.cpp:78-95).
  const int mid = params.moduli_id(level);
  const int L = params.chains(mid);
  const double deviation = static_cast<double>(params.deviations[level - 1]);
  const double product = value * params.scale * std::sqrt(deviation) + 0.5;
  std::vector<int64_t> out(L);
  for (int j = 0; j < L; j++) {
    const uint64_t q = params.q[mid + j];
    int64_t s = floor_abs_mod(product, q, 62);
    if (product < 0) s = static_cast<int64_t>(q) - s;
    out[j] = s;
  }
  return out;
}

std::unique_ptr<Data> Engine::rescale_any(const Data &text) {
  // CKKSEngine::rescale_ (engine_rescale.cpp:5-33).
  if (text.is_rescaled()) return clone(text);
  if (text.is_ntt()) {
    auto intt = to_intt(text);
    auto r = core_rescale(*intt);
    return to_ntt(*r);
  }
  return core_rescale(text);
}

Engine::Matched Engine::match_texts(const Data &t1, const Data &t2, bool plain) {
  // match_form (engine_add.cpp:36-79 for two ciphertexts, :180-211 for a ciphertext
  // and a plaintext, which stays in coefficient form).
  Matched m;
  m.a = &t1;
  m.b = &t2;
  const bool ntt = t1.is_ntt();
  auto set_a = [&](std::unique_ptr<Data> d) {
    m.own_a = std::move(d);
    m.a = m.own_a.get();
  };
  auto set_b = [&](std::unique_ptr<Data> d) {
    m.own_b = std::move(d);
    m.b = m.own_b.get();
  };
  if (plain) {
    if (m.b->is_ntt()) set_b(to_intt(*m.b));
    if (!ntt || t1.level() > t2.level()) {
      if (m.a->is_ntt()) set_a(to_intt(*m.a));
    }
  } else if (!ntt) {
    if (m.a->is_ntt()) set_a(to_intt(*m.a));
    if (m.b->is_ntt()) set_b(to_intt(*m.b));
  } else if (t1.level() > t2.level()) {
    set_a(to_intt(*m.a));
  } else if (t1.level() < t2.level()) {
    set_b(to_intt(*m.b));
  }
  const int min_level = std::min(t1.level(), t2.level());
  if (m.a->level() != min_level) set_a(level_down_any(*m.a, min_level));
  if (m.b->level() != min_level) set_b(level_down_any(*m.b, min_level));
  if (m.a->is_rescaled() != m.b->is_rescaled()) {
    if (!m.a->is_rescaled())
      set_a(rescale_any(*m.a));
    else
      set_b(rescale_any(*m.b));
  }
  if (ntt) {
    if (!m.a->is_ntt()) set_a(to_ntt(*m.a));
    if (!plain && !m.b->is_ntt()) set_b(to_ntt(*m.b));
  }
  return m;
}

static void require_add_operands(const std::string &fn, const Data &a, const Data &b) {
  for (const Data *t : {&a, &b}) {
    if (t->type == kUnitCiphertext && t->polys != 2 && t->polys != 3)
      throw std::runtime_error(fn + ": the input unit ciphertext should have either 2 or 3 "
                                    "polynomials.");
  }
  // MATCH_CKKS_SCALE (engine_require.cpp:462-474): a relative difference above 1e-4
  // between texts at the same level and rescale state.
  const long double diff = std::fabs(b.scale - a.scale) / b.scale;
  if (diff > 1e-4L && a.level() == b.level() && a.is_rescaled() == b.is_rescaled())
    throw std::runtime_error(fn + ": the ckks scale of the input " + std::string(b.type_name()) +
                             "s does not match.");
}

std::unique_ptr<Data> Engine::add(const Data &x, const Data &y) {
  require_add_operands("Add Unit Ciphertexts", x, y);
  Matched m = match_texts(x, y, false);
  const Data *a = m.a, *b = m.b;
  if (a->polys < b->polys) std::swap(a, b);  // add_trio_and_duo(trio, duo), engine_add.cpp:93-100
  auto out = make_data(kUnitCiphertext, a->flag | b->flag, a->moduli_id, a->polys, a->scale);
  const long long ps = a->poly_stride();
  for (int p = 0; p < a->polys; p++) {
    if (p < b->polys)
      pointwise(kOpAddReduce, a->chains, a->moduli_id, a->d + p * ps, b->d + p * b->poly_stride(),
                nullptr, out->d + p * ps);
    else
      check(cudaMemcpyAsync(out->d + p * ps, a->d + p * ps, ps * sizeof(int64_t),
                            cudaMemcpyDeviceToDevice, stream_),
            "copy");
  }
  return out;
}

std::unique_ptr<Data> Engine::subtract(const Data &x, const Data &y) {
  require_add_operands("Subtract Unit Ciphertexts", x, y);
  Matched m = match_texts(x, y, false);
  const Data *a = m.a, *b = m.b;
  const int polys = std::max(a->polys, b->polys);
  const Data *shape = a->polys >= b->polys ? a : b;
  auto out = make_data(kUnitCiphertext, a->flag | b->flag, shape->moduli_id, polys,
                       a->polys >= b->polys ? a->scale : b->scale);
  const long long ps = out->poly_stride();
  const int L = out->chains, mid = out->moduli_id;
  for (int p = 0; p < polys; p++) {
    int64_t *o = out->d + p * ps;
    if (p < a->polys && p < b->polys) {
      pointwise(kOpSubReduce, L, mid, a->d + p * a->poly_stride(), b->d + p * b->poly_stride(),
                nullptr, o);
    } else if (p < a->polys) {  // subtract_trio_by_duo: third polynomial copied
      check(cudaMemcpyAsync(o, a->d + p * a->poly_stride(), ps * sizeof(int64_t),
                            cudaMemcpyDeviceToDevice, stream_),
            "copy");
    } else {  // subtract_duo_by_trio: reduce then negate the third polynomial
      pointwise(kOpReduce, L, mid, b->d + p * b->poly_stride(), nullptr, nullptr, o);
      pointwise(kOpNegate, L, mid, o, nullptr, nullptr, o);
    }
  }
  return out;
}

std::unique_ptr<Data> Engine::add_plain(const Data &ct, const Data &pt) {
  // CKKSEngine::add(UnitCiphertext*, UnitPlaintext*) and CKKSCore::add
  // (core.cpp:374-413): the plaintext joins polynomial 0.
  require_add_operands("Add Unit Ciphertext And Unit Plaintext", ct, pt);
  Matched m = match_texts(ct, pt, true);
  const Data *c = m.a;
  std::unique_ptr<Data> pn;
  const Data *p = m.b;
  if (c->is_ntt()) {
    pn = to_ntt(*p);
    p = pn.get();
  }
  auto out = clone(*c);
  pointwise(kOpAddReduce, params.chains(c->moduli_id), c->moduli_id, c->d, p->d, nullptr, out->d);
  return out;
}

std::unique_ptr<Data> Engine::subtract_plain(const Data &ct, const Data &pt) {
  // CKKSCore::subtract(UnitCiphertext*, UnitPlaintext*) (core.cpp:558-596).
  require_add_operands("Subtract Unit Ciphertext By Unit Plaintext", ct, pt);
  Matched m = match_texts(ct, pt, true);
  const Data *c = m.a;
  std::unique_ptr<Data> pn;
  const Data *p = m.b;
  if (c->is_ntt()) {
    pn = to_ntt(*p);
    p = pn.get();
  }
  auto out = clone(*c);
  pointwise(kOpSubReduce, params.chains(c->moduli_id), c->moduli_id, c->d, p->d, nullptr, out->d);
  return out;
}

std::unique_ptr<Data> Engine::subtract_from_plain(const Data &pt, const Data &ct) {
  // CKKSCore::subtract(UnitPlaintext*, UnitCiphertext*) (core.cpp:514-556): p - c0,
  // then the other polynomials negated (reduced first in NTT form).
  require_add_operands("Subtract Unit Plaintext By Unit Ciphertext", ct, pt);
  Matched m = match_texts(ct, pt, true);
  const Data *c = m.a;
  std::unique_ptr<Data> pn;
  const Data *p = m.b;
  if (c->is_ntt()) {
    pn = to_ntt(*p);
    p = pn.get();
  }
  auto out = make_data(kUnitCiphertext, c->flag, c->moduli_id, c->polys, c->scale);
  const int L = params.chains(c->moduli_id), mid = c->moduli_id;
  const long long ps = c->poly_stride();
  pointwise(kOpSubReduce, L, mid, p->d, c->d, nullptr, out->d);
  for (int q = 1; q < c->polys; q++) {
    const int64_t *src = c->d + q * ps;
    if (c->is_ntt()) {
      pointwise(kOpReduce, L, mid, src, nullptr, nullptr, out->d + q * ps);
      src = out->d + q * ps;
    }
    pointwise(kOpNegate, L, mid, src, nullptr, nullptr, out->d + q * ps);
  }
  return out;
}

std::unique_ptr<Data> Engine::add_scalar(const Data &ct, double value) {
  // CKKSEngine::add(UnitCiphertext*, double) (engine_add.cpp:518-536): an encoded
  // constant vector for NTT-form or rescaled input, else CKKSCore::add(ct, double)
  // (core.cpp:340-372), the scaled constant added to coefficient 0 of polynomial 0.
  if (ct.is_ntt() || ct.is_rescaled()) {
    std::vector<double> message(params.slot_count, value);
    auto pt = encode(message.data(), nullptr, params.slot_count, ct.level(), false);
    return add_plain(ct, *pt);
  }
  const auto mult = add_multiplier(value, ct.level());
  auto out = clone(ct);
  pointwise(kOpAddScalarFirst, params.chains(ct.moduli_id), ct.moduli_id, ct.d, nullptr,
            mult.data(), out->d);
  return out;
}

std::unique_ptr<Data> Engine::subtract_scalar(const Data &ct, double value) {
  return add_scalar(ct, -value);  // engine_subtract.cpp:319-325
}

std::unique_ptr<Data> Engine::multiply_plain(const Data &ct, const Data &pt) {
  // CKKSEngine::multiply(UnitCiphertext*, UnitPlaintext*) (engine_multiply.cpp:210-227)
  // and CKKSCore::multiply(ct, pt) (core.cpp:257-282).
  const std::string fn = "Multiply Unit Ciphertext And Unit Plaintext";
  if (ct.polys != 2 && ct.polys != 3)
    throw std::runtime_error(fn + ": the input unit ciphertext should have either 2 or 3 "
                                  "polynomials.");
  if (ct.level() <= 0 || pt.level() <= 0)
    throw std::runtime_error(fn + ": the input texts should have a positive level.");
  const int level = std::min(ct.level(), pt.level());
  auto c = prepare_for_multiply(ct, level);
  auto p = prepare_for_multiply(pt, level);
  auto out = make_data(kUnitCiphertext, (c->flag | p->flag) & ~kFlagRescaled, c->moduli_id,
                       c->polys, c->scale * p->scale);
  const long long ps = c->poly_stride();
  for (int q = 0; q < c->polys; q++)
    pointwise(kOpMult, c->chains, c->moduli_id, c->d + q * ps, p->d, nullptr, out->d + q * ps);
  return out;
}

std::unique_ptr<Data> Engine::multiply_scalar(const Data &ct, double value) {
  // CKKSEngine::multiply(UnitCiphertext*, double) (engine_multiply.cpp:418-432) and
  // CKKSCore::multiply(ct, double) (core.cpp:196-229): enter the scaled constant,
  // reduce, then rescale by the first prime.
  const std::string fn = "Multiply Unit Ciphertext And Double Scalar";
  if (ct.polys != 2 && ct.polys != 3)
    throw std::runtime_error(fn + ": the input unit ciphertext should have either 2 or 3 "
                                  "polynomials.");
  if (ct.is_rescaled())
    throw std::runtime_error(fn + ": the input unit ciphertext should not be rescaled.");
  if (ct.level() <= 0)
    throw std::runtime_error(fn + ": the input unit ciphertext should have a positive level.");
  std::unique_ptr<Data> hold;
  const Data *x = &ct;
  if (x->is_ntt()) {
    hold = to_intt(*x);
    x = hold.get();
  }
  const int level = x->level();
  const int mid = x->moduli_id;
  const int L = x->chains;
  const auto mult = mult_multiplier(value, level);
  if (L > kMaxScalarLimbs) throw std::invalid_argument(fn + ": too many limbs.");
  LimbScalars c{};
  for (int j = 0; j < L; j++) c.v[j] = mult[j];
  const long double rs = params.rescaled_scale(x->scale, mid);
  auto out = make_data(kUnitCiphertext, x->flag, params.moduli_id(level - 1), x->polys, rs * rs);
  check(timed("scalar_rescale", [&] {
          return launch_scalar_rescale(tables_, ks_, params.n, x->polys, L, mid, c, x->d,
                                       x->poly_stride(), out->d, out->poly_stride(), stream_);
        }),
        "multiply scalar");
  return out;
}

std::unique_ptr<Data> Engine::multiply_integer(const Data &ct, int64_t value) {
  // CKKSEngine::multiply(UnitCiphertext*, int64_t) (engine_multiply.cpp:443-457),
  // make_mult_multiplier(int64_t, moduli_id) (precomputed.cpp:519-532).
  const std::string fn = "Multiply Unit Ciphertext And Integer Scalar";
  if (ct.polys != 2 && ct.polys != 3)
    throw std::runtime_error(fn + ": the input unit ciphertext should have either 2 or 3 "
                                  "polynomials.");
  if (ct.is_rescaled())
    throw std::runtime_error(fn + ": the input unit ciphertext should not be rescaled.");
  std::unique_ptr<Data> hold;
  const Data *x = &ct;
  if (x->is_ntt()) {
    hold = to_intt(*x);
    x = hold.get();
  }
  std::vector<int64_t> mult(x->chains);
  for (int j = 0; j < x->chains; j++)
    mult[j] = mod_mul(value, INT64_C(1) << 62, static_cast<int64_t>(params.q[x->moduli_id + j]));
  auto out = make_data(kUnitCiphertext, x->flag, x->moduli_id, x->polys, x->scale);
  const long long ps = x->poly_stride();
  for (int q = 0; q < x->polys; q++)
    pointwise(kOpEnterReduce, x->chains, x->moduli_id, x->d + q * ps, nullptr, mult.data(),
              out->d + q * ps);
  return out;
}

std::unique_ptr<Data> Engine::negate(const Data &ct) {
  // CKKSCore::negate (core.cpp:1002-1023): NTT-form words are reduced first.
  if (ct.polys != 2 && ct.polys != 3)
    throw std::runtime_error("Negate Unit Ciphertext: the input unit ciphertext should have "
                             "either 2 or 3 polynomials.");
  auto out = make_data(ct.type, ct.flag, ct.moduli_id, ct.polys, ct.scale);
  const long long ps = ct.poly_stride();
  const int L = params.chains(ct.moduli_id);
  for (int q = 0; q < ct.polys; q++) {
    const int64_t *src = ct.d + q * ps;
    if (ct.is_ntt()) {
      pointwise(kOpReduce, L, ct.moduli_id, src, nullptr, nullptr, out->d + q * ps);
      src = out->d + q * ps;
    }
    pointwise(kOpNegate, L, ct.moduli_id, src, nullptr, nullptr, out->d + q * ps);
  }
  return out;
}

std::unique_ptr<Data> Engine::square(const Data &ct, const Data *rk) {
  // CKKSEngine::square (engine_multiply.cpp:86-101, 175-188) and CKKSCore::square
  // (core.cpp:316-338).
  const std::string fn = rk ? "Square Unit Ciphertext Then Relinearize" : "Square Unit Ciphertext";
  if (ct.polys != 2)
    throw std::runtime_error(fn + ": the input unit ciphertext should have 2 polynomials.");
  if (ct.level() <= 0)
    throw std::runtime_error(fn + ": the input unit ciphertext should have a positive level.");
  if (rk) require_key_level(fn, ct, *rk, true);
  auto r = rescale_any(ct);
  auto x = r->is_ntt() ? std::move(r) : to_ntt(*r);
  // The square's tensor (d1 = x0 x1 doubled with add_reduce) is the product's tensor
  // of x with itself, so with a key the fused tensor-iNTT relinearization serves.
  if (rk) return relinearized_product(*x, *x, *rk);
  auto out = make_data(kUnitCiphertext, x->flag & ~kFlagRescaled, x->moduli_id, 3,
                       x->scale * x->scale);
  const long long ps = x->poly_stride();
  const int L = x->chains, mid = x->moduli_id;
  pointwise(kOpMult, L, mid, x->d, x->d, nullptr, out->d);
  pointwise(kOpMult, L, mid, x->d, x->d + ps, nullptr, out->d + ps);
  pointwise(kOpAddReduce, L, mid, out->d + ps, out->d + ps, nullptr, out->d + ps);
  pointwise(kOpMult, L, mid, x->d + ps, x->d + ps, nullptr, out->d + 2 * ps);
  return out;
}

}  // namespace fhe_b200
