// A caller of the reference's engine interface (AbstractEngine), built twice by
// shim/Makefile: against the reference's CPU engine and against the B200 engine
// through GpuCKKSEngine.  It walks the accelerated path -- keys, encode/encrypt,
// add/subtract/multiply with relinearization and rescale, rotations, conjugation,
// level down, negation, in-place addition, decrypt/decode -- and prints, per step,
// the first slots of the decrypted result and the largest error against the
// plaintext computation, so the two builds' outputs can be compared line by line.
#include <cmath>
#include <complex>
#include <cstdio>
#include <string>
#include <vector>

#include "engine/engine.h"

using namespace desilo::fhe;
using cvec = std::vector<std::complex<double>>;

namespace {

void report(const char *name, const cvec &got, const cvec &want) {
  double err = 0;
  for (size_t i = 0; i < want.size(); i++) err = std::max(err, std::abs(got[i] - want[i]));
  std::printf("%s err %.3e :", name, err);
  for (int i = 0; i < 6; i++) std::printf(" %.9f %.9f", got[i].real(), got[i].imag());
  std::printf("\n");
}

cvec rotated(const cvec &v, int delta) {
  cvec out(v.size());
  const int n = static_cast<int>(v.size());
  for (int i = 0; i < n; i++) out[i] = v[((i - delta) % n + n) % n];
  return out;
}

}  // namespace

int main() {
  AbstractEngine *engine = create_ckks_engine(CKKSConfig{});
  const int slots = engine->get_slot_count();
  cvec m1(slots), m2(slots);
  for (int i = 0; i < slots; i++) {
    m1[i] = {std::sin(0.001 * i), std::cos(0.003 * i) * 0.5};
    m2[i] = {0.25 + 0.5 * std::cos(0.002 * i), -0.1 * std::sin(0.004 * i)};
  }
  SecretKey *sk = engine->create_secret_key();
  PublicKey *pk = engine->create_public_key(sk);
  RelinearizationKey *rk = engine->create_relinearization_key(sk);
  ConjugationKey *ck = engine->create_conjugation_key(sk);
  RotationKey *rot = engine->create_rotation_key(sk);
  FixedRotationKey *fk5 = engine->create_fixed_rotation_key(sk, 5);

  Ciphertext *a = engine->encrypt(m1, pk);
  Ciphertext *b = engine->encrypt(m2, sk);
  auto show = [&](const char *name, Ciphertext *ct, const cvec &want) {
    report(name, engine->decrypt_complex(ct, sk), want);
    delete ct;
  };
  cvec want(slots);

  for (int i = 0; i < slots; i++) want[i] = m1[i];
  show("encrypt_public", engine->clone(a), want);
  for (int i = 0; i < slots; i++) want[i] = m1[i] + m2[i];
  show("add", engine->add(a, b), want);
  for (int i = 0; i < slots; i++) want[i] = m1[i] - m2[i];
  show("subtract_vector", engine->subtract(a, m2), want);
  for (int i = 0; i < slots; i++) want[i] = m1[i] * m2[i];
  {
    Ciphertext *p = engine->multiply(a, b, rk);
    show("multiply_relinearize_rescale", engine->rescale(p), want);
    delete p;
    Ciphertext *t = engine->multiply(a, b);
    Ciphertext *r = engine->relinearize(t, rk);
    show("tensor_relinearize_rescale", engine->rescale(r), want);
    delete t;
    delete r;
  }
  for (int i = 0; i < slots; i++) want[i] = m1[i] * m1[i];
  {
    Ciphertext *s = engine->square(a, rk);
    show("square_rescale", engine->rescale(s), want);
    delete s;
  }
  for (int i = 0; i < slots; i++) want[i] = m1[i] * 0.75;
  show("multiply_scalar", engine->multiply(a, 0.75), want);
  for (int i = 0; i < slots; i++) want[i] = m1[i] * m2[i];
  {
    Ciphertext *p = engine->multiply(a, m2);
    show("multiply_vector_rescale", engine->rescale(p), want);
    delete p;
  }
  show("rotate_key_3", engine->rotate(a, rot, 3), rotated(m1, 3));
  show("rotate_fixed_5", engine->rotate(a, fk5), rotated(m1, 5));
  for (int i = 0; i < slots; i++) want[i] = std::conj(m1[i]);
  show("conjugate", engine->conjugate(a, ck), want);
  for (int i = 0; i < slots; i++) want[i] = m1[i];
  show("level_down", engine->level_down(a, engine->get_max_level() - 2), want);
  for (int i = 0; i < slots; i++) want[i] = -m1[i];
  show("negate", engine->negate(a), want);
  for (int i = 0; i < slots; i++) want[i] = m1[i] + m2[i];
  {
    Ciphertext *c = engine->clone(a);
    engine->add_inplace(c, b);
    show("add_inplace", c, want);
  }
  {
    std::vector<FixedRotationKey *> keys{fk5, rot->fixed_rotation_keys_[1]};
    auto outs = engine->rotate_batch(a, keys);
    show("rotate_batch_5", outs[0], rotated(m1, 5));
    show("rotate_batch_2", outs[1], rotated(m1, 2));
  }

  delete a;
  delete b;
  delete fk5;
  delete rot;
  delete ck;
  delete rk;
  delete pk;
  delete sk;
  delete engine;
  return 0;
}
