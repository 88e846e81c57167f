// The B200 CKKS engine (see engine.hpp).
#include "engine.hpp"

#include <algorithm>
#include <cstring>

namespace fhe_b200 {

// ------------------------------------------------------------------- Data --

size_t Data::words() const {
  return static_cast<size_t>(polys) * chains * static_cast<size_t>(engine->params.n);
}

long long Data::poly_stride() const {
  return static_cast<long long>(chains) * engine->params.n;
}

int Data::level() const {
  int c = chains;
  if (flag & kFlagSpecial) c -= engine->params.special_prime_count;
  return (flag & kFlagRescaled) ? c - 1 : c - 2;
}

const char *Data::type_name() const {
  switch (type) {
    case kSecretKey: return "secret key";
    case kPublicKey: return "public key";
    case kRelinearizationKey: return "relinearization key";
    case kUnitCiphertext: return "unit ciphertext";
    case kUnitPlaintext: return "unit plaintext";
    case kFixedRotationKey: return "fixed rotation key";
    case kConjugationKey: return "conjugation key";
    case kKeySwitchingKey: return "key switching key";
    default: return "data";
  }
}

Data::~Data() {
  if (engine) {
    if (d) engine->free_words(d);
    engine->forget(this);
  }
}

// ----------------------------------------------------------------- Engine --

void Engine::check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation)
      throw std::bad_alloc();
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
  }
}

template <class T>
T *Engine::upload_table(const std::vector<T> &v) {
  const size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
  void *p = nullptr;
  check(cudaMalloc(&p, bytes), "cudaMalloc(table)");
  table_buffers_.push_back(static_cast<int64_t *>(p));
  if (!v.empty()) check(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload table");
  return static_cast<T *>(p);
}

Engine::Engine(const Config &config) : params(config) {
  int device = 0;
  check(cudaGetDevice(&device), "cudaGetDevice");
  check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  stream_ = own_stream_;
  // Keep freed blocks in the stream-ordered pool: key switching allocates and frees
  // the same temporaries every call.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t threshold = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }

  const Parameters &p = params;
  const int P = p.prime_count;
  tables_.q = upload_table(p.q);
  tables_.k = upload_table(p.k);
  tables_.r_squared = upload_table(p.r_squared);
  tables_.n_inverse = upload_table(p.n_inverse);
  tables_.root = upload_table(p.root);
  tables_.root_inverse = upload_table(p.root_inverse);
  std::vector<double> inv_q(P), inv_2q(P);
  for (int i = 0; i < P; i++) {
    inv_q[i] = 1.0 / static_cast<double>(p.q[i]);
    inv_2q[i] = 1.0 / (2.0 * static_cast<double>(p.q[i]));
  }
  tables_.inv_q = upload_table(inv_q);
  tables_.inv_2q = upload_table(inv_2q);
  tables_.log_n = p.log_n;

  std::vector<int64_t> pinv(static_cast<size_t>(std::max(p.special_prime_count, 1)) * P, 0);
  for (int s = 0; s < p.special_prime_count; s++)
    for (size_t i = 0; i < p.p_inverse_mult_r[s].size(); i++) pinv[static_cast<size_t>(s) * P + i] = p.p_inverse_mult_r[s][i];
  std::vector<int64_t> rs(static_cast<size_t>(P) * P, 0);
  for (int from = 0; from + 1 < P; from++)
    for (int to = from + 1; to < P; to++)
      rs[static_cast<size_t>(from) * P + to] = p.rescale_scale[from][to - from - 1];
  ks_.p_inverse_mult_r = upload_table(pinv);
  ks_.rescale_scale = upload_table(rs);
  ks_.prime_count = P;
  ks_.special_count = p.special_prime_count;
}

Engine::~Engine() {
  cudaStreamSynchronize(stream_);
  // Objects still alive lose their device memory and their engine; the C ABI
  // rejects any later use of them.
  for (Data *d : live_) {
    if (d->d) cudaFreeAsync(d->d, stream_);
    d->d = nullptr;
    d->engine = nullptr;
  }
  live_.clear();
  for (auto &p : pending_) {
    cudaEventDestroy(p.start);
    cudaEventDestroy(p.stop);
  }
  for (auto ev : event_pool_) cudaEventDestroy(ev);
  cudaStreamSynchronize(stream_);
  if (own_stream_) cudaStreamSynchronize(own_stream_);
  for (auto &kv : partition_cache_) {
    cudaFree(kv.second.start);
  }
  for (auto *b : table_buffers_) cudaFree(b);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void Engine::synchronize() { check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize"); }

int64_t *Engine::alloc_words(size_t words) {
  void *p = nullptr;
  check(cudaMallocAsync(&p, std::max<size_t>(words, 1) * sizeof(int64_t), stream_), "cudaMallocAsync");
  return static_cast<int64_t *>(p);
}

void Engine::free_words(int64_t *p) {
  if (p) cudaFreeAsync(p, stream_);
}

std::unique_ptr<Data> Engine::make_data(int type, int flag, int moduli_id, int polys,
                                        long double scale) {
  if (moduli_id < 0 || moduli_id >= params.chain_count)
    throw std::invalid_argument("the moduli id is out of range.");
  if (polys <= 0) throw std::invalid_argument("the polynomial count should be positive.");
  auto d = std::make_unique<Data>();
  d->engine = this;
  d->type = type;
  d->flag = flag;
  d->moduli_id = moduli_id;
  d->polys = polys;
  d->chains = params.chains(moduli_id, (flag & kFlagSpecial) != 0);
  d->scale = scale;
  d->d = alloc_words(d->words());
  live_.insert(d.get());
  return d;
}

void Engine::forget(Data *d) { live_.erase(d); }

std::unique_ptr<Data> Engine::upload(int type, int flag, int moduli_id, int polys,
                                     long double scale, const int64_t *host) {
  if (!host) throw std::invalid_argument("the host limb pointer is null.");
  auto d = make_data(type, flag, moduli_id, polys, scale);
  check(cudaMemcpyAsync(d->d, host, d->words() * sizeof(int64_t), cudaMemcpyHostToDevice, stream_),
        "upload limbs");
  return d;
}

void Engine::download(const Data &d, int64_t *host) {
  download_async(d, host);
  synchronize();
}

void Engine::download_async(const Data &d, int64_t *host) {
  if (!host) throw std::invalid_argument("the host limb pointer is null.");
  check(cudaMemcpyAsync(host, d.d, d.words() * sizeof(int64_t), cudaMemcpyDeviceToHost, stream_),
        "download limbs");
}

std::unique_ptr<Data> Engine::clone(const Data &src) {
  auto d = make_data(src.type, src.flag, src.moduli_id, src.polys, src.scale);
  d->delta = src.delta;
  check(cudaMemcpyAsync(d->d, src.d, src.words() * sizeof(int64_t), cudaMemcpyDeviceToDevice, stream_),
        "clone");
  return d;
}

const DevicePartitions &Engine::partitions(int moduli_id, int key_moduli_id) {
  const auto key = std::make_pair(moduli_id, key_moduli_id);
  auto it = partition_cache_.find(key);
  if (it != partition_cache_.end()) return it->second;
  const auto parts = params.partitions(moduli_id, key_moduli_id);
  const int count = static_cast<int>(parts.size());
  const int E = params.chains(moduli_id, true);
  DevicePartitions dp;
  dp.count = count;
  dp.extended = E;
  // One device block: ints first, then the int64 tables.
  const size_t n_int = 3 * static_cast<size_t>(count);
  const size_t int_words = (n_int * sizeof(int) + 7) / 8;
  const size_t words = int_words + static_cast<size_t>(count) * (16 + 256 + 16 * static_cast<size_t>(E));
  std::vector<int64_t> host(words, 0);
  int *ints = reinterpret_cast<int *>(host.data());
  int64_t *inv = host.data() + int_words;
  int64_t *prod = inv + static_cast<size_t>(count) * 16;
  int64_t *prod2 = prod + static_cast<size_t>(count) * 256;
  for (int p = 0; p < count; p++) {
    const auto &pt = parts[p];
    if (pt.size > 16) throw std::invalid_argument("partition larger than 16 limbs.");
    ints[p] = pt.start;
    ints[count + p] = pt.size;
    ints[2 * count + p] = pt.partition_index;
    dp.max_key_index = std::max(dp.max_key_index, pt.partition_index);
    if (pt.partition_index < 0)
      throw std::invalid_argument("the key was created at a lower level than the text.");
    dp.max_size = std::max(dp.max_size, pt.size);
    dp.size_mask |= 1u << pt.size;
    const auto pc = params.partition_constants(moduli_id, pt);
    for (size_t i = 0; i < pc.inverse_r.size(); i++) inv[p * 16 + i] = pc.inverse_r[i];
    for (size_t ci = 0; ci < pc.product_r.size(); ci++)
      for (size_t t2 = 0; t2 < pc.product_r[ci].size(); t2++)
        prod[(p * 16 + ci) * 16 + t2] = pc.product_r[ci][t2];
    for (int ci = 0; ci + 1 < pt.size; ci++)
      for (int j = 0; j < E; j++)
        prod2[(static_cast<size_t>(p) * 16 + ci) * E + j] = pc.product_r_squared[static_cast<size_t>(ci) * E + j];
  }
  void *dev = nullptr;
  check(cudaMalloc(&dev, words * sizeof(int64_t)), "cudaMalloc(partitions)");
  check(cudaMemcpy(dev, host.data(), words * sizeof(int64_t), cudaMemcpyHostToDevice), "upload partitions");
  int *dints = static_cast<int *>(dev);
  dp.start = dints;
  dp.size = dints + count;
  dp.key_index = dints + 2 * count;
  int64_t *d64 = static_cast<int64_t *>(dev) + int_words;
  dp.inverse_r = d64;
  dp.product_r = d64 + static_cast<size_t>(count) * 16;
  dp.product_r_squared = dp.product_r + static_cast<size_t>(count) * 256;
  return partition_cache_.emplace(key, dp).first->second;
}

// --------------------------------------------------------------- transforms --

std::unique_ptr<Data> Engine::to_ntt(const Data &text) {
  if (text.is_ntt()) return clone(text);
  auto out = make_data(text.type, text.flag | kFlagNtt, text.moduli_id, text.polys, text.scale);
  check(timed("to_ntt", [&] { return launch_to_ntt(tables_, params.log_n, text.polys, text.chains, text.moduli_id, text.d,
                      text.poly_stride(), out->d, out->poly_stride(), stream_); }),
        "to_ntt");
  return out;
}

std::unique_ptr<Data> Engine::to_intt(const Data &text) {
  if (!text.is_ntt()) return clone(text);
  auto out = make_data(text.type, text.flag & ~kFlagNtt, text.moduli_id, text.polys, text.scale);
  check(timed("to_intt", [&] { return launch_to_intt(tables_, params.log_n, text.polys, text.chains, text.moduli_id, text.d,
                       text.poly_stride(), out->d, out->poly_stride(), stream_); }),
        "to_intt");
  return out;
}

void Engine::ntt_limbs(int64_t *limbs, int moduli_id, int chains, int polys, long long stride,
                       bool inverse) {
  if (!limbs) throw std::invalid_argument("the device limb pointer is null.");
  if (moduli_id < 0 || chains <= 0 || moduli_id + chains > params.prime_count || polys <= 0)
    throw std::invalid_argument("the limb range is out of the moduli chain.");
  check(timed("ntt_limbs", [&] { return launch_ntt_plain(tables_, params.log_n, polys, chains, moduli_id, limbs, stride, inverse,
                         stream_); }),
        "ntt_limbs");
}

// ------------------------------------------------------------------ rescale --

std::unique_ptr<Data> Engine::core_rescale(const Data &ct) {
  if (ct.flag & kFlagSpecial)
    throw std::invalid_argument("rescale of an extended polynomial is not supported.");
  if (ct.chains < 2) throw std::runtime_error("cannot rescale a single-limb text.");
  auto out = make_data(ct.type, ct.flag | kFlagRescaled, ct.moduli_id + 1, ct.polys,
                       params.rescaled_scale(ct.scale, ct.moduli_id));
  check(timed("rescale", [&] { return launch_rescale(tables_, ks_, params.n, ct.polys, ct.chains, ct.moduli_id, ct.d,
                       ct.poly_stride(), out->d, out->poly_stride(), stream_); }),
        "rescale");
  return out;
}

std::unique_ptr<Data> Engine::rescale(const Data &ct) {
  const std::string fn = "Rescale Unit Ciphertext";
  const std::string prefix = fn + ": the input " + ct.type_name() + " ";
  if (ct.polys != 2 && ct.polys != 3)
    throw std::runtime_error(prefix + "should have either 2 or 3 polynomials.");
  if (ct.level() <= 0) throw std::runtime_error(prefix + "should have a positive level.");
  if (ct.is_rescaled()) return clone(ct);
  if (ct.is_ntt()) {
    auto intt = to_intt(ct);
    auto r = core_rescale(*intt);
    return to_ntt(*r);
  }
  return core_rescale(ct);
}

// ----------------------------------------------------------------- multiply --

// prepare_for_multiply, engine_multiply.cpp:13-28.
std::unique_ptr<Data> Engine::prepare_for_multiply(const Data &text, int level) {
  std::unique_ptr<Data> cur;
  const Data *t = &text;
  if (t->level() > level) {
    cur = to_intt(*t);
    t = cur.get();
  }
  if (t->level() != level)
    throw std::invalid_argument("multiplying texts at different levels is not supported yet.");
  if (!t->is_rescaled()) {
    std::unique_ptr<Data> r;
    if (t->is_ntt()) {
      auto intt = to_intt(*t);
      auto rr = core_rescale(*intt);
      r = to_ntt(*rr);
    } else {
      r = core_rescale(*t);
    }
    cur = std::move(r);
    t = cur.get();
  }
  if (!t->is_ntt()) {
    cur = to_ntt(*t);
    t = cur.get();
  }
  if (!cur) cur = clone(*t);
  return cur;
}

void Engine::require_key_level(const std::string &fn, const Data &text, const Data &key,
                               bool for_multiply) {
  // is_key_compatible (engine_require.cpp:24-32) with the multiply relaxation
  // (engine_require.cpp:787-798).
  const int key_level = key.level();
  bool ok = text.moduli_id >= key.moduli_id;
  if (params.preset.one_more_level && text.moduli_id == 0 && key.moduli_id == 1) ok = true;
  if (!ok && !(for_multiply && text.level() - 1 == key_level))
    throw std::runtime_error(fn + ": the level of the input " + text.type_name() +
                             " is greater than that of the input relinearization key.");
}

static void require_text(const std::string &fn, const Data &t, int index, int count,
                         int polys_required, bool positive_level) {
  std::string prefix = fn + ": the";
  if (count > 1) prefix += index == 0 ? " first" : " second";
  prefix += std::string(" input ") + t.type_name() + " ";
  if (polys_required && t.polys != polys_required)
    throw std::runtime_error(prefix + "should have " + std::to_string(polys_required) +
                             " polynomials.");
  if (positive_level && t.level() <= 0)
    throw std::runtime_error(prefix + "should have a positive level.");
}

std::unique_ptr<Data> Engine::multiply(const Data &a, const Data &b) {
  const std::string fn = "Multiply Unit Ciphertexts";
  require_text(fn, a, 0, 2, 2, true);
  require_text(fn, b, 1, 2, 2, true);
  const int level = std::min(a.level(), b.level());
  auto pa = prepare_for_multiply(a, level);
  auto pb = prepare_for_multiply(b, level);
  const int flag = (pa->flag | pb->flag) & ~kFlagRescaled;
  auto out = make_data(kUnitCiphertext, flag, pa->moduli_id, 3, pa->scale * pb->scale);
  check(timed("tensor", [&] { return launch_tensor(tables_, params.n, pa->chains, pa->moduli_id, pa->d, pb->d, out->d, stream_); }),
        "tensor");
  return out;
}

void Engine::relinearize_tail(const int64_t *t3, int moduli_id, const Data &rk, int mode,
                              int64_t *out) {
  const int n = params.n;
  const int L = params.chains(moduli_id);
  const int E = params.chains(moduli_id, true);
  if (moduli_id < rk.moduli_id)
    throw std::invalid_argument(
        "the key switching key was created at a lower level than the text.");
  const DevicePartitions &dp = partitions(moduli_id, rk.moduli_id);
  if (rk.polys < 2 * (dp.max_key_index + 1))
    throw std::invalid_argument("the relinearization key has too few polynomials.");
  int64_t *digits = alloc_words(static_cast<size_t>(L) * n);
  int64_t *ext = alloc_words(static_cast<size_t>(dp.count) * E * n);
  int64_t *acc = alloc_words(static_cast<size_t>(2) * E * n);
  cudaError_t e = timed("mixed_radix", [&] {
    return launch_mixed_radix(tables_, dp, n, moduli_id, t3 + 2LL * L * n, digits, stream_);
  });
  if (e == cudaSuccess)
    e = timed("mod_up_ntt", [&] {
      return launch_mod_up_ntt(tables_, dp, params.log_n, moduli_id, digits, ext, stream_);
    });
  if (e == cudaSuccess)
    e = timed("key_inner_product", [&] {
      return launch_key_inner_product(tables_, dp, n, moduli_id, ext, rk.d, rk.chains,
                                      moduli_id - rk.moduli_id, acc, stream_);
    });
  if (e == cudaSuccess)
    e = timed("mod_down_intt", [&] {
      return launch_mod_down_intt(tables_, params.log_n, moduli_id, E, acc, stream_);
    });
  if (e == cudaSuccess)
    e = timed("mod_down_epilogue", [&] {
      return launch_mod_down_epilogue(tables_, ks_, n, moduli_id, L, acc, t3, mode, out, stream_);
    });
  free_words(digits);
  free_words(ext);
  free_words(acc);
  check(e, "key switch");
}

std::unique_ptr<Data> Engine::relinearize(const Data &ct, const Data &rk) {
  const std::string fn = "Relinearize Unit Ciphertext";
  require_text(fn, ct, 0, 1, 3, false);
  if (rk.type != kRelinearizationKey && rk.type != kKeySwitchingKey)
    throw std::invalid_argument(fn + ": the key is not a relinearization key.");
  require_key_level(fn, ct, rk, false);
  std::unique_ptr<Data> nt;
  const Data *x = &ct;
  if (!ct.is_ntt()) {
    nt = to_ntt(ct);
    x = nt.get();
  }
  const int m = x->moduli_id;
  const int L = x->chains;
  int64_t *t3 = alloc_words(static_cast<size_t>(3) * L * params.n);
  cudaError_t e = timed("to_intt", [&] {
    return launch_to_intt(tables_, params.log_n, 3, L, m, x->d, x->poly_stride(), t3,
                          static_cast<long long>(L) * params.n, stream_);
  });
  if (e != cudaSuccess) {
    free_words(t3);
    check(e, "relinearize");
  }
  auto out = make_data(kUnitCiphertext, x->flag & ~kFlagNtt, m, 2, x->scale);
  try {
    relinearize_tail(t3, m, rk, 1, out->d);
  } catch (...) {
    free_words(t3);
    throw;
  }
  free_words(t3);
  return out;
}

std::unique_ptr<Data> Engine::multiply_relinearize(const Data &a, const Data &b, const Data &rk) {
  const std::string fn = "Multiply Unit Ciphertexts Then Relinearize";
  require_text(fn, a, 0, 2, 2, true);
  require_text(fn, b, 1, 2, 2, true);
  require_key_level(fn, a, rk, true);
  require_key_level(fn, b, rk, true);
  auto m = multiply(a, b);
  return relinearize(*m, rk);
}

std::unique_ptr<Data> Engine::multiply_relinearize_rescale(const Data &a, const Data &b,
                                                           const Data &rk) {
  const std::string fn = "Multiply Unit Ciphertexts Then Relinearize";
  require_text(fn, a, 0, 2, 2, true);
  require_text(fn, b, 1, 2, 2, true);
  require_key_level(fn, a, rk, true);
  require_key_level(fn, b, rk, true);
  const int level = std::min(a.level(), b.level());
  auto pa = prepare_for_multiply(a, level);
  auto pb = prepare_for_multiply(b, level);
  const int m = pa->moduli_id;
  const int L = pa->chains;
  {
    // The tensor of the prepared inputs is at `level - 1`; rescaling it needs a
    // positive level (engine_rescale.cpp:48).
    const int tensor_level = L - 2;
    if (tensor_level <= 0)
      throw std::runtime_error(
          "Rescale Unit Ciphertext: the input unit ciphertext should have a positive level.");
  }
  int64_t *t3 = alloc_words(static_cast<size_t>(3) * L * params.n);
  cudaError_t e = timed("tensor_to_intt", [&] {
    return launch_tensor_to_intt(tables_, params.log_n, L, m, pa->d, pb->d, t3, stream_);
  });
  if (e != cudaSuccess) {
    free_words(t3);
    check(e, "tensor");
  }
  const int flag = ((pa->flag | pb->flag) & ~kFlagRescaled & ~kFlagNtt) | kFlagRescaled;
  const long double scale = params.rescaled_scale(pa->scale * pb->scale, m);
  auto out = make_data(kUnitCiphertext, flag, m + 1, 2, scale);
  try {
    relinearize_tail(t3, m, rk, 2, out->d);
  } catch (...) {
    free_words(t3);
    throw;
  }
  free_words(t3);
  return out;
}

// ---------------------------------------------------------------- profiling --

void Engine::set_profiling(bool on) { profiling_ = on; }

cudaEvent_t Engine::take_event() {
  if (!event_pool_.empty()) {
    cudaEvent_t e = event_pool_.back();
    event_pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  check(cudaEventCreate(&e), "cudaEventCreate");
  return e;
}

void Engine::collect_timings() {
  if (pending_.empty()) return;
  synchronize();
  for (auto &p : pending_) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
      auto &st = stats_[p.name];
      st.first += 1;
      st.second += ms;
    }
    event_pool_.push_back(p.start);
    event_pool_.push_back(p.stop);
  }
  pending_.clear();
}

std::string Engine::profile_report() {
  collect_timings();
  std::string out;
  for (const auto &kv : stats_) {
    char line[160];
    snprintf(line, sizeof(line), "%s %llu %.6f\n", kv.first.c_str(),
             static_cast<unsigned long long>(kv.second.first), kv.second.second);
    out += line;
  }
  return out;
}

void Engine::profile_reset() {
  collect_timings();
  stats_.clear();
}

}  // namespace fhe_b200
