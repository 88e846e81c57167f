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
    case kDecomposed: return "decomposed unit ciphertext";
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
    if (d) engine->release(d, copy_pending);
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

Engine::Engine(const Config &config) : params(config) {
  int device = 0;
  check(cudaGetDevice(&device), "cudaGetDevice");
  check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  stream_ = own_stream_;
  check(cudaStreamCreateWithFlags(&upload_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaStreamCreateWithFlags(&download_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaEventCreateWithFlags(&upload_done_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&compute_done_, cudaEventDisableTiming), "cudaEventCreate");
  set_concurrency(concurrency_);
  check(cudaMalloc(&device_error_, sizeof(int)), "cudaMalloc(error flag)");
  check(cudaMemset(device_error_, 0, sizeof(int)), "clear error flag");
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
  {
    // The same twiddles reduced to [0, q), for the transforms whose result only
    // matters modulo q (ntt.cuh, kValueOnly).
    const size_t per = static_cast<size_t>(p.n) - 1;
    std::vector<int64_t> rc(p.root), ric(p.root_inverse);
    for (int i = 0; i < P; i++) {
      const int64_t qi = static_cast<int64_t>(p.q[i]);
      for (size_t j = 0; j < per; j++) {
        rc[i * per + j] = guard(rc[i * per + j], qi);
        ric[i * per + j] = guard(ric[i * per + j], qi);
      }
    }
    tables_.root_reduced = upload_table(rc);
    tables_.root_inverse_reduced = upload_table(ric);
    // Plain twiddles and their Shoup quotients for shoup_mult.
    std::vector<int64_t> rs(2 * rc.size()), ris(2 * ric.size());
    for (int i = 0; i < P; i++) {
      const uint64_t qi = p.q[i];
      using u128 = unsigned __int128;
      auto mulmod = [&](uint64_t a, uint64_t b) { return static_cast<uint64_t>(static_cast<u128>(a) * b % qi); };
      uint64_t r_inverse = 1, base = (uint64_t(1) << 62) % qi;  // R^-1 = R^(q-2) mod q
      for (uint64_t e = qi - 2; e > 0; e >>= 1) {
        if (e & 1) r_inverse = mulmod(r_inverse, base);
        base = mulmod(base, base);
      }
      auto pair = [&](int64_t mont, int64_t *out) {
        const uint64_t w = mulmod(static_cast<uint64_t>(mont), r_inverse);
        out[0] = static_cast<int64_t>(w);
        out[1] = static_cast<int64_t>((static_cast<u128>(w) << 64) / qi);
      };
      for (size_t j = 0; j < per; j++) {
        pair(rc[i * per + j], &rs[2 * (i * per + j)]);
        pair(ric[i * per + j], &ris[2 * (i * per + j)]);
      }
    }
    tables_.root_shoup = upload_table(rs);
    tables_.root_inverse_shoup = upload_table(ris);
    // The reduced exit's constant N^-1 R^-1 (n_inverse = N^-1 R) and its Shoup quotient.
    std::vector<int64_t> es(2 * static_cast<size_t>(P));
    for (int i = 0; i < P; i++) {
      const uint64_t qi = p.q[i];
      using u128 = unsigned __int128;
      auto mulmod = [&](uint64_t a, uint64_t b) { return static_cast<uint64_t>(static_cast<u128>(a) * b % qi); };
      uint64_t r_inverse = 1, base = (uint64_t(1) << 62) % qi;
      for (uint64_t e = qi - 2; e > 0; e >>= 1) {
        if (e & 1) r_inverse = mulmod(r_inverse, base);
        base = mulmod(base, base);
      }
      const uint64_t c = mulmod(mulmod(static_cast<uint64_t>(p.n_inverse[i]) % qi, r_inverse), r_inverse);
      es[2 * i] = static_cast<int64_t>(c);
      es[2 * i + 1] = static_cast<int64_t>((static_cast<u128>(c) << 64) / qi);
    }
    tables_.exit_shoup = upload_table(es);
  }
  std::vector<double> inv_q(P), inv_2q(P);
  for (int i = 0; i < P; i++) {
    inv_q[i] = 1.0 / static_cast<double>(p.q[i]);
    inv_2q[i] = 1.0 / (2.0 * static_cast<double>(p.q[i]));
  }
  tables_.inv_q = upload_table(inv_q);
  tables_.inv_2q = upload_table(inv_2q);
  tables_.log_n = p.log_n;
  if (tc_ntt_supported(p.log_n)) {
    const TcNttHost h = make_tc_ntt_tables(p);
    tc_ntt_.bmat = upload_table(h.bmat);
    tc_ntt_.psi_pow = upload_table(h.psi_pow);
  }

  std::vector<int64_t> pinv(static_cast<size_t>(std::max(p.special_prime_count, 1)) * P, 0);
  for (int s = 0; s < p.special_prime_count; s++)
    for (size_t i = 0; i < p.p_inverse_mult_r[s].size(); i++) pinv[static_cast<size_t>(s) * P + i] = p.p_inverse_mult_r[s][i];
  std::vector<int64_t> rs(static_cast<size_t>(P) * P, 0);
  for (int from = 0; from + 1 < P; from++)
    for (int to = from + 1; to < P; to++)
      rs[static_cast<size_t>(from) * P + to] = p.rescale_scale[from][to - from - 1];
  std::vector<int64_t> ppr(P, 0);
  for (size_t i = 0; i < p.p_product_mult_r.size(); i++) ppr[i] = p.p_product_mult_r[i];
  ks_.p_inverse_mult_r = upload_table(pinv);
  ks_.rescale_scale = upload_table(rs);
  {
    // Shoup pairs of the rescale constants: C = rescale_scale R^-1 mod q_to.
    using u128 = unsigned __int128;
    std::vector<int64_t> rsh(2 * rs.size(), 0);
    for (int to = 1; to < P; to++) {
      const uint64_t qt = p.q[to];
      auto mulmod = [&](uint64_t a, uint64_t b) { return static_cast<uint64_t>(static_cast<u128>(a) * b % qt); };
      uint64_t r_inverse = 1, base = (uint64_t(1) << 62) % qt;
      for (uint64_t e = qt - 2; e > 0; e >>= 1) {
        if (e & 1) r_inverse = mulmod(r_inverse, base);
        base = mulmod(base, base);
      }
      for (int from = 0; from < to; from++) {
        const size_t at = static_cast<size_t>(from) * P + to;
        const uint64_t c = mulmod(static_cast<uint64_t>(rs[at]) % qt, r_inverse);
        rsh[2 * at] = static_cast<int64_t>(c);
        rsh[2 * at + 1] = static_cast<int64_t>((static_cast<u128>(c) << 64) / qt);
      }
    }
    ks_.rescale_shoup = upload_table(rsh);
    // The rescale and the enter as one product: q_from^-1 R mod q_to, the plain value
    // of rescale_scale; and R mod q for the rounder.
    std::vector<int64_t> resh(2 * rs.size(), 0), rmod(P, 0);
    for (int to = 0; to < P; to++) {
      const uint64_t qt = p.q[to];
      rmod[to] = static_cast<int64_t>((uint64_t(1) << 62) % qt);
      for (int from = 0; from < to; from++) {
        const size_t at = static_cast<size_t>(from) * P + to;
        const uint64_t c = static_cast<uint64_t>(rs[at]) % qt;
        resh[2 * at] = static_cast<int64_t>(c);
        resh[2 * at + 1] = static_cast<int64_t>((static_cast<u128>(c) << 64) / qt);
      }
    }
    ks_.rescale_enter_shoup = upload_table(resh);
    ks_.r_mod = upload_table(rmod);
    // P mod q and its Shoup quotient (the tensor addend of the key inner product):
    // p_product_mult_r R^-1.
    std::vector<int64_t> psh(2 * static_cast<size_t>(P), 0);
    for (int i = 0; i < P; i++) {
      const uint64_t qi = p.q[i];
      auto mulmod = [&](uint64_t a, uint64_t b) { return static_cast<uint64_t>(static_cast<u128>(a) * b % qi); };
      uint64_t r_inverse = 1, base = (uint64_t(1) << 62) % qi;
      for (uint64_t e = qi - 2; e > 0; e >>= 1) {
        if (e & 1) r_inverse = mulmod(r_inverse, base);
        base = mulmod(base, base);
      }
      const uint64_t c = mulmod(static_cast<uint64_t>(ppr[i]) % qi, r_inverse);
      psh[2 * i] = static_cast<int64_t>(c);
      psh[2 * i + 1] = static_cast<int64_t>((static_cast<u128>(c) << 64) / qi);
    }
    ks_.p_shoup = upload_table(psh);
  }
  ks_.p_product_mult_r = upload_table(ppr);
  ks_.prime_count = P;
  ks_.special_count = p.special_prime_count;
  seed(nullptr, nullptr);
}

Engine::~Engine() {
  cudaStreamSynchronize(upload_stream_);
  cudaStreamSynchronize(download_stream_);
  cudaStreamSynchronize(stream_);
  for (auto &kv : graph_cache_)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
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
  for (auto &kv : signed_perm_cache_) cudaFree(kv.second);
  for (auto &kv : ntt_perm_cache_) cudaFree(kv.second);
  for (auto *b : table_buffers_) cudaFree(b);
  if (device_error_) cudaFree(device_error_);
  for (auto w : workers_) {
    cudaStreamSynchronize(w);
    cudaStreamDestroy(w);
  }
  for (auto ev : worker_done_) cudaEventDestroy(ev);
  if (fork_) cudaEventDestroy(fork_);
  cudaEventDestroy(upload_done_);
  cudaEventDestroy(compute_done_);
  cudaStreamDestroy(upload_stream_);
  cudaStreamDestroy(download_stream_);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void Engine::synchronize() {
  check(cudaStreamSynchronize(upload_stream_), "cudaStreamSynchronize");
  check(cudaStreamSynchronize(download_stream_), "cudaStreamSynchronize");
  check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
  int flag = 0;
  check(cudaMemcpy(&flag, device_error_, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
  if (flag) {
    check(cudaMemset(device_error_, 0, sizeof(int)), "clear error flag");
    throw CudaError("a tensor-core wait ran out; the results since the last check are unspecified");
  }
}

const ModDownTcTables *Engine::mod_down_tc(int moduli_id) {
  const int L = params.chains(moduli_id), K = params.special_prime_count;
  if (!mod_down_tc_supported(K, L, params.n)) return nullptr;
  auto it = mod_down_tc_cache_.find(moduli_id);
  if (it != mod_down_tc_cache_.end()) return &it->second;
  const ModDownTcHost h = make_mod_down_tc_tables(params.q, params.p_inverse_mult_r, moduli_id, L, K);
  ModDownTcTables tc;
  tc.b = upload_table(h.b);
  tc.c_r = upload_table(h.c_r);
  tc.c_shoup = upload_table(h.c_shoup);
  tc.rounds = h.rounds;
  tc.kb = h.kb;
  return &mod_down_tc_cache_.emplace(moduli_id, tc).first->second;
}

void Engine::set_tensor_cores(int mode) {
  if (mode != kTensorCoresOff && mode != kTensorCoresOn && mode != kTensorCoresAuto)
    throw std::invalid_argument("the tensor core mode should be 0 (off), 1 (on) or 2 (auto).");
  tensor_cores_ = mode;
}

void Engine::set_tensor_core_wait_limit(long long limit) {
  if (limit > static_cast<long long>(UINT32_MAX))
    throw std::invalid_argument("the tensor core wait limit should be below 2^32.");
  tc_wait_limit_ = limit < 0 ? kTcDefaultWaitLimit : static_cast<uint32_t>(limit);
}

bool Engine::use_tensor_cores(int min_special) const {
  return tensor_cores_ == kTensorCoresOn ||
         (tensor_cores_ == kTensorCoresAuto && params.special_prime_count >= min_special);
}

const ModUpTcTables *Engine::mod_up_tc(int moduli_id) {
  const auto parts = params.partitions(moduli_id, moduli_id);
  int max_size = 0;
  for (const auto &pt : parts) max_size = std::max(max_size, pt.size);
  if (!mod_up_tc_supported(max_size, params.n)) return nullptr;
  auto it = mod_up_tc_cache_.find(moduli_id);
  if (it != mod_up_tc_cache_.end()) return &it->second;
  std::vector<PartitionConstants> constants;
  for (const auto &pt : parts) constants.push_back(params.partition_constants(moduli_id, pt));
  const ModUpTcHost h = make_mod_up_tc_tables(params.q, params.r_squared, moduli_id,
                                              params.chains(moduli_id, true), parts, constants);
  ModUpTcTables tc;
  tc.b = upload_table(h.b);
  tc.b_offset = upload_table(h.b_offset);
  tc.rounds = h.rounds;
  return &mod_up_tc_cache_.emplace(moduli_id, tc).first->second;
}

cudaError_t Engine::mod_up(const DevicePartitions &dp, int moduli_id, const int64_t *digits,
                           int64_t *ext, bool skip_own) {
  if (skip_own && use_tc_ntt()) return cudaErrorInvalidValue;
  const ModUpTcTables *tc =
      use_tensor_cores(kTensorCoreModUpMinSpecial) ? mod_up_tc(moduli_id) : nullptr;
  if (!tc)
    return timed("mod_up_ntt", [&] {
      return launch_mod_up_ntt(tables_, dp, params.log_n, moduli_id, digits, ext, stream_,
                               skip_own);
    });
  // Profiled as two families, so the tensor-pipe contraction's time is its own.
  const cudaError_t e = timed("mod_up_contract_tc", [&] {
    return launch_mod_up_contract_tc(tables_, dp, *tc, params.n, moduli_id, digits, ext,
                                     tc_status(), stream_, skip_own);
  });
  if (e != cudaSuccess) return e;
  return timed("mod_up_ntt_tc", [&] {
    if (use_tc_ntt())  // the extended limbs only matter modulo q: the tensor-core NTT
      return launch_tc_ntt(tc_ntt_, tables_, false, dp.count, dp.extended, moduli_id, ext,
                           static_cast<long long>(dp.extended) * params.n, tc_status(), stream_);
    return launch_extended_ntt(tables_, dp, params.log_n, moduli_id, ext, stream_, skip_own);
  });
}

int64_t *Engine::own_limbs_ext(int moduli_id, const Data &rk) {
  if (use_tc_ntt() || rk.moduli_id > moduli_id) return nullptr;
  const DevicePartitions &dp = partitions(moduli_id, rk.moduli_id);
  return alloc_words(static_cast<size_t>(dp.count) * dp.extended * params.n);
}

cudaError_t Engine::mod_down_transform(int moduli_id, int extended, int64_t *acc, int polys) {
  if (use_tc_ntt())
    return timed("mod_down_intt_tc", [&] {
      return launch_tc_ntt(tc_ntt_, tables_, true, polys, extended, moduli_id, acc,
                           static_cast<long long>(extended) * params.n, tc_status(), stream_);
    });
  return timed("mod_down_intt", [&] {
    return launch_mod_down_intt(tables_, params.log_n, moduli_id, extended, acc, stream_, polys);
  });
}

cudaError_t Engine::mod_down_epilogue(int moduli_id, int limbs, const int64_t *acc,
                                      const EpilogueOps &ops, int64_t *out) {
  const ModDownTcTables *tc =
      use_tensor_cores(kTensorCoreMinSpecial) ? mod_down_tc(moduli_id) : nullptr;
  if (tc)
    return timed("mod_down_epilogue_tc", [&] {
      return launch_mod_down_epilogue_tc(tables_, ks_, *tc, params.n, moduli_id, limbs, acc, ops,
                                         out, tc_status(), stream_);
    });
  return timed("mod_down_epilogue", [&] {
    return launch_mod_down_epilogue_ops(tables_, ks_, params.n, moduli_id, limbs, acc, ops, out,
                                        stream_);
  });
}

void Engine::upload_bytes(void *dst, const void *src, size_t bytes, const char *what) {
  check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), what);
  synchronize();
}

int64_t *Engine::alloc_words(size_t words) {
  void *p = nullptr;
  check(cudaMallocAsync(&p, std::max<size_t>(words, 1) * sizeof(int64_t), stream_), "cudaMallocAsync");
  return static_cast<int64_t *>(p);
}

void Engine::free_words(int64_t *p) {
  if (p) cudaFreeAsync(p, stream_);
}

void Engine::release(int64_t *p, bool copy_pending) {
  if (!p) return;
  if (!copy_pending) {
    cudaFreeAsync(p, stream_);
    return;
  }
  // Behind the download and behind every kernel queued so far.
  order_download_after_compute();
  cudaFreeAsync(p, download_stream_);
}

void Engine::order_download_after_compute() {
  check(cudaEventRecord(compute_done_, stream_), "cudaEventRecord");
  check(cudaStreamWaitEvent(download_stream_, compute_done_, 0), "cudaStreamWaitEvent");
}

void Engine::order_compute_after_upload() {
  check(cudaEventRecord(upload_done_, upload_stream_), "cudaEventRecord");
  check(cudaStreamWaitEvent(stream_, upload_done_, 0), "cudaStreamWaitEvent");
}

std::unique_ptr<Data> Engine::make_data(int type, int flag, int moduli_id, int polys,
                                        long double scale, cudaStream_t alloc_stream) {
  if (moduli_id < 0 || moduli_id >= params.chain_count)
    throw std::invalid_argument("the moduli id is out of range.");
  if (polys <= 0) throw std::invalid_argument("the polynomial count should be positive.");
  auto d = std::make_unique<Data>();
  d->engine = this;
  d->serial = ++serial_;
  d->type = type;
  d->flag = flag;
  d->moduli_id = moduli_id;
  d->polys = polys;
  d->chains = params.chains(moduli_id, (flag & kFlagSpecial) != 0);
  d->scale = scale;
  if (alloc_stream) {
    void *p = nullptr;
    check(cudaMallocAsync(&p, std::max<size_t>(d->words(), 1) * sizeof(int64_t), alloc_stream),
          "cudaMallocAsync");
    d->d = static_cast<int64_t *>(p);
  } else {
    d->d = alloc_words(d->words());
  }
  live_.insert(d.get());
  return d;
}

void Engine::forget(Data *d) { live_.erase(d); }

std::unique_ptr<Data> Engine::upload(int type, int flag, int moduli_id, int polys,
                                     long double scale, const int64_t *host) {
  if (!host) throw std::invalid_argument("the host limb pointer is null.");
  auto d = make_data(type, flag, moduli_id, polys, scale, upload_stream_);
  check(cudaMemcpyAsync(d->d, host, d->words() * sizeof(int64_t), cudaMemcpyHostToDevice,
                        upload_stream_),
        "upload limbs");
  order_compute_after_upload();
  return d;
}

void Engine::download(const Data &d, int64_t *host) {
  download_async(d, host);
  synchronize();
}

void Engine::download_async(const Data &d, int64_t *host) {
  if (!host) throw std::invalid_argument("the host limb pointer is null.");
  order_download_after_compute();
  check(cudaMemcpyAsync(host, d.d, d.words() * sizeof(int64_t), cudaMemcpyDeviceToHost,
                        download_stream_),
        "download limbs");
  d.copy_pending = true;
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
    if (p < 8) dp.key_index_first[p] = pt.partition_index;
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
  upload_bytes(dev, host.data(), words * sizeof(int64_t), "upload partitions");
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

void Engine::mont_mult_limbs(const int64_t *a, const int64_t *b, int64_t *y, int moduli_id, int chains,
                             int polys, long long stride) {
  if (!a || !b || !y) throw std::invalid_argument("a device limb pointer is null.");
  if (moduli_id < 0 || chains <= 0 || moduli_id + chains > params.prime_count || polys <= 0 ||
      stride < static_cast<long long>(chains) * params.n)
    throw std::invalid_argument("the limb range is out of the moduli chain.");
  if (stride == static_cast<long long>(chains) * params.n) {
    pointwise(kOpMult, polys * chains, moduli_id, a, b, nullptr, y, chains);  // one launch
    return;
  }
  for (int p = 0; p < polys; p++)
    pointwise(kOpMult, chains, moduli_id, a + p * stride, b + p * stride, nullptr, y + p * stride);
}

// ------------------------------------------------------------------ rescale --

std::unique_ptr<Data> Engine::core_rescale(const Data &ct) {
  // rescale_once_ (core_rescale.cpp:5-25); with the special primes, their limbs are
  // rescaled too (the prime tables run on past the chain).
  if (ct.chains < 2) throw std::runtime_error("cannot rescale a single-limb text.");
  auto out = make_data(ct.type, ct.flag | kFlagRescaled, ct.moduli_id + 1, ct.polys,
                       params.rescaled_scale(ct.scale, ct.moduli_id));
  check(timed("rescale", [&] { return launch_rescale(tables_, ks_, params.n, ct.polys, ct.chains, ct.moduli_id, ct.d,
                       ct.poly_stride(), out->d, out->poly_stride(), stream_); }),
        "rescale");
  return out;
}

std::unique_ptr<Data> Engine::rescale_to_ntt(const Data &ct, const ExactLimbs &exact) {
  // to_ntt(core_rescale(ct)) of a coefficient-form text in one pass.
  if (ct.chains < 2) throw std::runtime_error("cannot rescale a single-limb text.");
  if (ct.is_ntt()) throw std::invalid_argument("rescale to NTT: the text is in NTT form.");
  auto out = make_data(ct.type, ct.flag | kFlagRescaled | kFlagNtt, ct.moduli_id + 1, ct.polys,
                       params.rescaled_scale(ct.scale, ct.moduli_id));
  check(timed("rescale_to_ntt", [&] {
          return launch_rescale_to_ntt(tables_, ks_, params.log_n, ct.polys, out->chains,
                                       ct.moduli_id, ct.d, ct.poly_stride(), out->d,
                                       out->poly_stride(), stream_, exact);
        }),
        "rescale to NTT");
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
std::unique_ptr<Data> Engine::prepare_for_multiply(const Data &text, int level, const Data *rk) {
  std::unique_ptr<Data> cur;
  const Data *t = &text;
  if (t->level() > level) {
    cur = to_intt(*t);
    t = cur.get();
  }
  if (t->level() != level) {
    cur = level_down_any(*t, level);
    t = cur.get();
  }
  if (!t->is_rescaled()) {
    // rescale_, then the NTT form the product needs: one fused pass.  Before a
    // relinearization only the limbs it reads exactly need the reference's words;
    // they are limbs of the second polynomial (a1 b1 forms the tensor's third).
    const ExactLimbs exact = rk ? relinearize_exact_limbs(t->moduli_id + 1, *rk, 1)
                                : ExactLimbs{ExactLimbs::kAllExact, 0};
    if (t->is_ntt()) {
      auto intt = to_intt(*t);
      cur = rescale_to_ntt(*intt, exact);
    } else {
      cur = rescale_to_ntt(*t, exact);
    }
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
                               bool for_multiply, const char *key_name) {
  // is_key_compatible (engine_require.cpp:24-32) with the multiply relaxation
  // (engine_require.cpp:787-798).
  const int key_level = key.level();
  bool ok = text.moduli_id >= key.moduli_id;
  if (params.preset.one_more_level && text.moduli_id == 0 && key.moduli_id == 1) ok = true;
  if (!ok && !(for_multiply && text.level() - 1 == key_level))
    throw std::runtime_error(fn + ": the level of the input " + text.type_name() +
                             " is greater than that of the input " + key_name + ".");
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

void Engine::key_switch_pipeline(const int64_t *c1, int moduli_id, const Data &key,
                                 const int64_t *rotate_c0, const EpilogueOps &ops, int64_t *out,
                                 const int64_t *decomposed, int64_t *own_ext,
                                 const TensorAddend *addend) {
  const int n = params.n;
  const int L = params.chains(moduli_id);
  const int E = params.chains(moduli_id, true);
  if (moduli_id < key.moduli_id)
    throw std::invalid_argument(
        "the key switching key was created at a lower level than the text.");
  const DevicePartitions &dp = partitions(moduli_id, key.moduli_id);
  if (key.polys < 2 * (dp.max_key_index + 1))
    throw std::invalid_argument("the key switching key has too few polynomials.");
  // A decomposition made earlier (hoisted rotations) replaces the ModUp: its partitions
  // have the same starts and sizes, only the key index depends on the key's level.
  int64_t *digits = alloc_words(static_cast<size_t>(L) * n);
  const bool skip_own = own_ext != nullptr && !decomposed;
  int64_t *alloc_ext =
      decomposed || skip_own ? nullptr : alloc_words(static_cast<size_t>(dp.count) * E * n);
  int64_t *work_ext = skip_own ? own_ext : alloc_ext;
  const int64_t *ext = decomposed ? decomposed : work_ext;
  int64_t *acc = alloc_words(static_cast<size_t>(2) * E * n);
  cudaError_t e = cudaSuccess;
  if (!decomposed) {
    e = timed("mixed_radix", [&] {
      return launch_mixed_radix(tables_, dp, n, moduli_id, c1, digits, stream_);
    });
    if (e == cudaSuccess) e = mod_up(dp, moduli_id, digits, work_ext, skip_own);
  }
  if (e == cudaSuccess)
    e = timed("key_inner_product", [&] {
      return launch_key_inner_product(tables_, dp, n, moduli_id, ext, key.d, key.chains,
                                      moduli_id - key.moduli_id, acc, stream_,
                                      addend ? *addend : TensorAddend{});
    });
  if (e == cudaSuccess && rotate_c0 != nullptr)
    e = timed("rotate_base", [&] {
      // `digits` is free again and serves as the NTT's intermediate buffer.
      return launch_rotate_base(tables_, ks_, params.log_n, moduli_id, L, rotate_c0, digits, acc,
                                stream_);
    });
  if (e == cudaSuccess) e = mod_down_transform(moduli_id, E, acc, 2);
  if (e == cudaSuccess) e = mod_down_epilogue(moduli_id, L, acc, ops, out);
  free_words(digits);
  free_words(alloc_ext);
  free_words(acc);
  check(e, "key switch");
}

void Engine::relinearize_tail(const int64_t *t3, int moduli_id, const Data &rk, int mode,
                              int64_t *out, int64_t *own_ext, const TensorAddend *addend) {
  EpilogueOps ops;
  ops.rescale = mode == 2;
  const long long L = params.chains(moduli_id);
  if (addend) {
    // The first two polynomials enter through the key inner product; t3 holds the
    // third alone.
    key_switch_pipeline(t3, moduli_id, rk, nullptr, ops, out, nullptr, own_ext, addend);
    return;
  }
  ops.base = t3;
  ops.base_polys = mode == 0 ? 0 : 2;
  key_switch_pipeline(t3 + 2 * L * params.n, moduli_id, rk, nullptr, ops, out, nullptr, own_ext);
}

bool Engine::fold_tensor(int moduli_id, const Data &rk) {
  if (!value_transforms_) return false;
  if (partitions(moduli_id, rk.moduli_id).count > 8) return false;
  // The exact sum takes operands below 2^61: words in [0, 2q) for q below 2^60.  And
  // P d carries d only where P is invertible: a chain whose first prime is also a
  // special prime (P = 0 modulo it, at the top level) keeps the addend in ModDown's
  // store, where the reference adds it.
  const int L = params.chains(moduli_id);
  for (int i = 0; i < L; i++)
    if (params.q[moduli_id + i] >= (uint64_t(1) << 60) ||
        params.p_product_mult_r[moduli_id + i] == 0)
      return false;
  return true;
}

TensorAddend Engine::tensor_addend(const Data &pa, const Data &pb) const {
  TensorAddend add;
  add.a = pa.d;
  add.b = pb.d;
  add.a_stride = pa.poly_stride();
  add.b_stride = pb.poly_stride();
  add.p_shoup = ks_.p_shoup;
  add.p_mont = ks_.p_product_mult_r;
  add.limbs = pa.chains;
  return add;
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
  // With the fold, c0 and c1 enter the key inner product as P c0, P c1 and only c2 is
  // transformed back.
  const bool fold = fold_tensor(m, rk);
  int64_t *t3 = alloc_words(static_cast<size_t>(fold ? 1 : 3) * L * params.n);
  cudaError_t e = timed("to_intt", [&] {
    return launch_to_intt(tables_, params.log_n, fold ? 1 : 3, L, m,
                          x->d + (fold ? 2 * x->poly_stride() : 0), x->poly_stride(), t3,
                          static_cast<long long>(L) * params.n, stream_);
  });
  if (e != cudaSuccess) {
    free_words(t3);
    check(e, "relinearize");
  }
  auto out = make_data(kUnitCiphertext, x->flag & ~kFlagNtt, m, 2, x->scale);
  // The NTT-form third polynomial is at hand: its limbs are ModUp's own limbs.
  int64_t *own_ext = own_limbs_ext(m, rk);
  try {
    if (own_ext) {
      const long long n = params.n;
      const int E = params.chains(m, true);
      const auto parts = params.partitions(m, rk.moduli_id);
      for (size_t p = 0; p < parts.size(); p++)
        check(cudaMemcpyAsync(own_ext + (static_cast<long long>(p) * E + parts[p].start) * n,
                              x->d + 2 * x->poly_stride() + parts[p].start * n,
                              static_cast<size_t>(parts[p].size) * n * sizeof(int64_t),
                              cudaMemcpyDeviceToDevice, stream_),
              "copy own limbs");
    }
    TensorAddend add;
    add.a = x->d;
    add.a_stride = x->poly_stride();
    add.p_shoup = ks_.p_shoup;
    add.p_mont = ks_.p_product_mult_r;
    add.limbs = L;
    relinearize_tail(t3, m, rk, 1, out->d, own_ext, fold ? &add : nullptr);
  } catch (...) {
    free_words(t3);
    free_words(own_ext);
    throw;
  }
  free_words(t3);
  free_words(own_ext);
  return out;
}

std::unique_ptr<Data> Engine::multiply_relinearize(const Data &a, const Data &b, const Data &rk) {
  const std::string fn = "Multiply Unit Ciphertexts Then Relinearize";
  require_text(fn, a, 0, 2, 2, true);
  require_text(fn, b, 1, 2, 2, true);
  require_key_level(fn, a, rk, true);
  require_key_level(fn, b, rk, true);
  const int level = std::min(a.level(), b.level());
  auto pa = prepare_for_multiply(a, level, &rk);
  auto pb = prepare_for_multiply(b, level, &rk);
  return relinearized_product(*pa, *pb, rk);
}

ExactLimbs Engine::relinearize_exact_limbs(int moduli_id, const Data &rk, int poly) {
  // Relinearization reduces its output to [0, q) (ModDown's store) and reads the
  // tensor's first two polynomials as addends below 2q, so only their values matter.
  // Of the third it reads each partition's limbs through Garner's digits (rns_to_mrs,
  // core_key_switch.cpp:21-56): the first limb as the first digit itself, word for
  // word; limb j > 0 as guard(x_j + 2q_j - Y, 2q_j) followed by a Montgomery product
  // and a reduction to [0, q_j), where Y is the first limb's word or a digit already
  // reduced.  That result depends on x_j only modulo q_j when 0 <= Y <= 2q_j: the
  // first limb's word is at most q_first (to_intt_'s exit), and the later Y are below
  // q_j when q_first <= 2q_j (with every prime below 2^60, the Montgomery products
  // before them are below 1.5 q_j).  So a partition whose first prime is at most
  // twice each of its others needs its first limb exact; any other partition needs
  // all of them.
  ExactLimbs all{ExactLimbs::kAllExact, 0};
  if (!value_transforms_) return all;
  const int L = params.chains(moduli_id);
  for (int i = 0; i < L; i++)
    if (params.q[moduli_id + i] >= (uint64_t(1) << 60)) return all;
  uint64_t mask = 0;
  for (const Partition &pt : params.partitions(moduli_id, rk.moduli_id)) {
    const uint64_t q_first = params.q[moduli_id + pt.start];
    bool bounded = true;
    for (int j = 1; j < pt.size; j++)
      if (q_first > 2 * params.q[moduli_id + pt.start + j]) bounded = false;
    const int exact_count = bounded ? 1 : pt.size;
    for (int j = 0; j < exact_count; j++) {
      const int limb = pt.start + j;
      if (limb >= 64) return all;
      mask |= uint64_t(1) << limb;
    }
  }
  return ExactLimbs{poly, mask};
}

std::unique_ptr<Data> Engine::relinearized_product(const Data &pa, const Data &pb, const Data &rk) {
  // multiply (core.cpp:284-314) then relinearize (core.cpp:713-741) of prepared
  // NTT-form inputs: the tensor's NTT-form polynomials are formed on the way into
  // the inverse NTT (all three) or, with the fold, into the key inner product (d0,
  // d1) and a streaming pass before d2's inverse NTT.
  const int m = pa.moduli_id;
  const int L = pa.chains;
  // With the fold, only the third polynomial is transformed; the first two go to the
  // key inner product.
  const bool fold = fold_tensor(m, rk);
  int64_t *t3 = alloc_words(static_cast<size_t>(fold ? 1 : 3) * L * params.n);
  // The tensor's NTT-form third polynomial also lands in ModUp's own limbs.
  int64_t *own_ext = own_limbs_ext(m, rk);
  const DevicePartitions *dp = own_ext ? &partitions(m, rk.moduli_id) : nullptr;
  const ExactLimbs exact = relinearize_exact_limbs(m, rk, fold ? 0 : 2);
  cudaError_t e = timed("tensor_to_intt", [&] {
    return launch_tensor_to_intt(tables_, params.log_n, L, m, pa.d, pb.d, t3, stream_, own_ext, dp,
                                 exact, fold);
  });
  if (e != cudaSuccess) {
    free_words(t3);
    free_words(own_ext);
    check(e, "tensor");
  }
  const int flag = (pa.flag | pb.flag) & ~kFlagRescaled & ~kFlagNtt;
  auto out = make_data(kUnitCiphertext, flag, m, 2, pa.scale * pb.scale);
  try {
    const TensorAddend add = tensor_addend(pa, pb);
    relinearize_tail(t3, m, rk, 1, out->d, own_ext, fold ? &add : nullptr);
  } catch (...) {
    free_words(t3);
    free_words(own_ext);
    throw;
  }
  free_words(t3);
  free_words(own_ext);
  return out;
}

std::unique_ptr<Data> Engine::multiply_relinearize_rescale(const Data &a, const Data &b,
                                                           const Data &rk) {
  const std::string fn = "Multiply Unit Ciphertexts Then Relinearize";
  require_text(fn, a, 0, 2, 2, true);
  require_text(fn, b, 1, 2, 2, true);
  require_key_level(fn, a, rk, true);
  require_key_level(fn, b, rk, true);
  const int level = std::min(a.level(), b.level());
  auto pa = prepare_for_multiply(a, level, &rk);
  auto pb = prepare_for_multiply(b, level, &rk);
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
  const bool fold = fold_tensor(m, rk);
  int64_t *t3 = alloc_words(static_cast<size_t>(fold ? 1 : 3) * L * params.n);
  // The tensor's NTT-form third polynomial also lands in ModUp's own limbs.
  int64_t *own_ext = own_limbs_ext(m, rk);
  const DevicePartitions *dp = own_ext ? &partitions(m, rk.moduli_id) : nullptr;
  const ExactLimbs exact = relinearize_exact_limbs(m, rk, fold ? 0 : 2);
  cudaError_t e = timed("tensor_to_intt", [&] {
    return launch_tensor_to_intt(tables_, params.log_n, L, m, pa->d, pb->d, t3, stream_, own_ext,
                                 dp, exact, fold);
  });
  if (e != cudaSuccess) {
    free_words(t3);
    free_words(own_ext);
    check(e, "tensor");
  }
  const int flag = ((pa->flag | pb->flag) & ~kFlagRescaled & ~kFlagNtt) | kFlagRescaled;
  const long double scale = params.rescaled_scale(pa->scale * pb->scale, m);
  auto out = make_data(kUnitCiphertext, flag, m + 1, 2, scale);
  try {
    const TensorAddend add = tensor_addend(*pa, *pb);
    relinearize_tail(t3, m, rk, 2, out->d, own_ext, fold ? &add : nullptr);
  } catch (...) {
    free_words(t3);
    free_words(own_ext);
    throw;
  }
  free_words(t3);
  free_words(own_ext);
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

// --------------------------------------------------------------- level down --

// CKKSCore::level_down_after_rescale (core.cpp:743-778) for rescaled text in any
// form and CKKSCore::level_down (core.cpp:786-838) for coefficient-form text:
// multiply by the level-down multiplier, then (not rescaled) rescale by the first
// prime and keep the destination's limbs.
std::unique_ptr<Data> Engine::core_level_down(const Data &text, int level) {
  const int n = params.n;
  const int dst_mid = params.moduli_id(level);
  const int out_chains = params.chains(dst_mid);
  auto to_scalars = [](const std::vector<int64_t> &v, int count) {
    if (count > kMaxScalarLimbs || static_cast<int>(v.size()) < count)
      throw std::invalid_argument("level down: too many limbs.");
    LimbScalars s{};
    for (int i = 0; i < count; i++) s.v[i] = v[i];
    return s;
  };
  if (text.is_rescaled()) {
    const LimbScalars s = to_scalars(params.level_down_multiplier_after_rescale(text.level(), level), out_chains);
    auto out = make_data(text.type, text.flag & ~kFlagRescaled, dst_mid, text.polys,
                         params.level_down_scale(level));
    check(timed("level_down", [&] {
            return launch_scalar_enter(tables_, n, text.polys, out_chains, dst_mid, text.d,
                                       text.poly_stride(), dst_mid - text.moduli_id, s, out->d,
                                       out->poly_stride(), stream_);
          }),
          "level_down");
    return out;
  }
  const int src_mid = text.moduli_id;
  const int L = text.chains;
  const int next_mid = params.moduli_id(text.level() - 1);
  const LimbScalars s = to_scalars(params.level_down_multiplier(text.level(), level), L);
  const long long in_stride = static_cast<long long>(L) * n;
  const long long mid_stride = static_cast<long long>(L - 1) * n;
  int64_t *entered = alloc_words(static_cast<size_t>(text.polys) * in_stride);
  int64_t *rescaled = alloc_words(static_cast<size_t>(text.polys) * mid_stride);
  auto out = make_data(text.type, text.flag, dst_mid, text.polys, params.level_down_scale(level));
  cudaError_t e = timed("level_down", [&] {
    return launch_scalar_enter(tables_, n, text.polys, L, src_mid, text.d, text.poly_stride(), 0, s,
                               entered, in_stride, stream_);
  });
  if (e == cudaSuccess)
    e = timed("rescale", [&] {
      return launch_rescale(tables_, ks_, n, text.polys, L, src_mid, entered, in_stride, rescaled,
                            mid_stride, stream_);
    });
  if (e == cudaSuccess) {
    const int offset = dst_mid - next_mid;
    e = cudaMemcpy2DAsync(out->d, out->poly_stride() * sizeof(int64_t),
                          rescaled + static_cast<long long>(offset) * n, mid_stride * sizeof(int64_t),
                          static_cast<size_t>(out_chains) * n * sizeof(int64_t), text.polys,
                          cudaMemcpyDeviceToDevice, stream_);
  }
  free_words(entered);
  free_words(rescaled);
  check(e, "level_down");
  return out;
}

// CKKSEngine::level_down_ (engine_level_down.cpp:5-36).
std::unique_ptr<Data> Engine::level_down_any(const Data &text, int level) {
  if (text.level() == level) return clone(text);
  if (text.is_rescaled()) return core_level_down(text, level);
  if (text.is_ntt()) {
    auto intt = to_intt(text);
    auto down = core_level_down(*intt, level);
    return to_ntt(*down);
  }
  return core_level_down(text, level);
}

std::unique_ptr<Data> Engine::level_down(const Data &text, int level) {
  const bool cipher = text.type == kUnitCiphertext;
  const std::string fn = cipher ? "Level Down Unit Ciphertext" : "Level Down Unit Plaintext";
  if (cipher && text.polys != 2 && text.polys != 3)
    throw std::runtime_error(fn + ": the input " + text.type_name() +
                             " should have either 2 or 3 polynomials.");
  if (level < 0 || level > text.level())
    throw std::runtime_error(fn + ": the target level cannot be reached.");
  return level_down_any(text, level);
}

// ------------------------------------------------- rotation and conjugation --

int Engine::normalized_delta(int delta, bool normalize_by_slot_count) const {
  // CKKSEngine::to_normalized_delta (engine.cpp:227-235) with positive_modulo.
  const int m = normalize_by_slot_count ? params.slot_count : params.n / 2;
  return (m + delta % m) % m;
}

const int32_t *Engine::device_signed_permutation(int delta) {
  auto it = signed_perm_cache_.find(delta);
  if (it != signed_perm_cache_.end()) return it->second;
  const auto host = signed_permutation(params.n, delta);
  void *p = nullptr;
  check(cudaMalloc(&p, host.size() * sizeof(int32_t)), "cudaMalloc(permutation)");
  upload_bytes(p, host.data(), host.size() * sizeof(int32_t), "upload permutation");
  return signed_perm_cache_.emplace(delta, static_cast<int32_t *>(p)).first->second;
}

const int32_t *Engine::device_ntt_permutation(int delta) {
  auto it = ntt_perm_cache_.find(delta);
  if (it != ntt_perm_cache_.end()) return it->second;
  const auto host = ntt_permutation(params.n, delta);
  void *p = nullptr;
  check(cudaMalloc(&p, host.size() * sizeof(int32_t)), "cudaMalloc(permutation)");
  upload_bytes(p, host.data(), host.size() * sizeof(int32_t), "upload permutation");
  return ntt_perm_cache_.emplace(delta, static_cast<int32_t *>(p)).first->second;
}

// CKKSCore::rotate (core.cpp:939-963): key switch of c1 with the b * P term, ModDown,
// then the key's signed coefficient permutation.
std::unique_ptr<Data> Engine::core_rotate(const Data &ct, const Data &key, const Data *decomposed) {
  auto out = make_data(kUnitCiphertext, ct.flag, ct.moduli_id, 2, ct.scale);
  EpilogueOps ops;
  ops.signed_perm = device_signed_permutation(key.delta);
  key_switch_pipeline(ct.d + ct.poly_stride(), ct.moduli_id, key, ct.d, ops, out->d,
                      decomposed ? decomposed->d : nullptr);
  return out;
}

std::vector<std::unique_ptr<Data>> Engine::rotate_batch(const Data &ct,
                                                        const std::vector<const Data *> &keys) {
  // CKKSEngine::rotate_batch(ct, fixed rotation keys) (engine_rotate.cpp:262-300):
  // the input is decomposed once (core_key_switch.cpp:434-466) and every key reuses
  // the decomposition (core.cpp:939-952).
  const std::string fn = "Batch Rotate Ciphertext With Fixed Rotation Keys";
  require_text(fn, ct, 0, 1, 2, false);
  for (const Data *k : keys) {
    if (!k || k->type != kFixedRotationKey)
      throw std::invalid_argument(fn + ": the key is not a fixed rotation key.");
    require_key_level(fn, ct, *k, false, "fixed rotation key");
  }
  std::unique_ptr<Data> hold;
  const Data *x = &ct;
  if (params.preset.one_more_level && ct.moduli_id == 0) {
    hold = level_down_any(ct, ct.level() - 1);
    x = hold.get();
  }
  if (x->is_ntt()) {
    hold = to_intt(*x);
    x = hold.get();
  }
  std::vector<std::unique_ptr<Data>> out;
  if (keys.empty()) return out;
  auto decomposed = decompose(*x);
  for (const Data *k : keys) out.push_back(core_rotate(*x, *k, decomposed.get()));
  return out;
}

std::unique_ptr<Data> Engine::rotate(const Data &ct, const Data &key) {
  const std::string fn = "Rotate Unit Ciphertext With Fixed Rotation Key";
  require_text(fn, ct, 0, 1, 2, false);
  if (key.type != kFixedRotationKey)
    throw std::invalid_argument(fn + ": the key is not a fixed rotation key.");
  require_key_level(fn, ct, key, false, "fixed rotation key");
  std::unique_ptr<Data> hold;
  const Data *x = &ct;
  if (params.preset.one_more_level && ct.moduli_id == 0) {
    hold = level_down_any(ct, ct.level() - 1);
    x = hold.get();
  }
  if (x->is_ntt()) {
    hold = to_intt(*x);
    x = hold.get();
  }
  return core_rotate(*x, key);
}

std::unique_ptr<Data> Engine::rotate(const Data &ct, const std::vector<const Data *> &keys,
                                     int delta, bool normalize_by_slot_count) {
  const std::string fn = "Rotate Unit Ciphertext With Rotation Key";
  require_text(fn, ct, 0, 1, 2, false);
  for (const Data *k : keys) {
    if (k == nullptr || k->type != kFixedRotationKey)
      throw std::invalid_argument(fn + ": the key is not a fixed rotation key.");
    require_key_level(fn, ct, *k, false, "rotation key");
  }
  const int nd = normalized_delta(delta, normalize_by_slot_count);
  if (nd == 0) return to_intt(ct);
  std::unique_ptr<Data> cur;
  for (const Data *k : keys) {
    if ((nd & k->delta) == 0) continue;
    auto next = rotate(cur ? *cur : ct, *k);
    cur = std::move(next);
  }
  if (!cur)
    throw std::invalid_argument(fn + ": no fixed rotation key matches the delta.");
  return cur;
}

std::unique_ptr<Data> Engine::rotate_plain(const Data &pt, int delta) {
  // CKKSEngine::rotate(UnitPlaintext*, int) (engine_rotate.cpp:10-24).
  const int nd = normalized_delta(delta);
  auto out = make_data(pt.type, pt.flag, pt.moduli_id, pt.polys, pt.scale);
  out->delta = pt.delta;
  if (pt.is_ntt()) {
    check(timed("permute", [&] {
            return launch_permute_gather(params.n, pt.polys, pt.chains, pt.d, pt.poly_stride(),
                                         device_ntt_permutation(nd), out->d, out->poly_stride(),
                                         stream_);
          }),
          "rotate");
  } else {
    check(timed("permute", [&] {
            return launch_permute_signed(tables_, params.n, pt.polys, pt.chains, pt.moduli_id, pt.d,
                                         pt.poly_stride(), device_signed_permutation(nd), out->d,
                                         out->poly_stride(), stream_);
          }),
          "rotate");
  }
  return out;
}

std::unique_ptr<Data> Engine::conjugate_plain(const Data &pt) {
  // conjugate_intt_form / conjugate_ntt_form (core.cpp:1020-1033): delta -1.
  auto out = make_data(pt.type, pt.flag, pt.moduli_id, pt.polys, pt.scale);
  if (pt.is_ntt()) {
    check(timed("permute", [&] {
            return launch_permute_gather(params.n, pt.polys, pt.chains, pt.d, pt.poly_stride(),
                                         device_ntt_permutation(-1), out->d, out->poly_stride(),
                                         stream_);
          }),
          "conjugate");
  } else {
    check(timed("permute", [&] {
            return launch_permute_signed(tables_, params.n, pt.polys, pt.chains, pt.moduli_id, pt.d,
                                         pt.poly_stride(), device_signed_permutation(-1), out->d,
                                         out->poly_stride(), stream_);
          }),
          "conjugate");
  }
  return out;
}

std::unique_ptr<Data> Engine::conjugate(const Data &ct, const Data &key) {
  // CKKSEngine::conjugate (engine_conjugate.cpp:53-73) and CKKSCore::conjugate
  // (core.cpp:1035-1056): permute both polynomials, key switch the permuted c1 and
  // add the permuted c0.
  const std::string fn = "Conjugate Unit Ciphertext";
  require_text(fn, ct, 0, 1, 2, false);
  if (key.type != kConjugationKey)
    throw std::invalid_argument(fn + ": the key is not a conjugation key.");
  require_key_level(fn, ct, key, false, "conjugation key");
  std::unique_ptr<Data> hold;
  const Data *x = &ct;
  if (params.preset.one_more_level && ct.moduli_id == 0) {
    hold = level_down_any(ct, ct.level() - 1);
    x = hold.get();
  }
  if (x->is_ntt()) {
    hold = to_intt(*x);
    x = hold.get();
  }
  const int n = params.n;
  const long long ps = x->poly_stride();
  int64_t *permuted = alloc_words(static_cast<size_t>(2) * ps);
  cudaError_t e = timed("permute", [&] {
    return launch_permute_signed(tables_, n, 2, x->chains, x->moduli_id, x->d, ps,
                                 device_signed_permutation(-1), permuted, ps, stream_);
  });
  if (e != cudaSuccess) {
    free_words(permuted);
    check(e, "conjugate");
  }
  auto out = make_data(kUnitCiphertext, x->flag, x->moduli_id, 2, x->scale);
  EpilogueOps ops;
  ops.base = permuted;
  ops.base_polys = 1;
  try {
    key_switch_pipeline(permuted + ps, x->moduli_id, key, nullptr, ops, out->d);
  } catch (...) {
    free_words(permuted);
    throw;
  }
  free_words(permuted);
  return out;
}

std::unique_ptr<Data> Engine::switch_key(const Data &ct, const Data &key) {
  const std::string fn = "Switch Key";
  require_text(fn, ct, 0, 1, 2, false);
  if (key.type != kKeySwitchingKey)
    throw std::invalid_argument(fn + ": the key is not a key switching key.");
  require_key_level(fn, ct, key, false, "key switching key");
  std::unique_ptr<Data> hold;
  const Data *x = &ct;
  if (x->is_ntt()) {
    hold = to_intt(*x);
    x = hold.get();
  }
  auto out = make_data(x->type, x->flag, x->moduli_id, 2, x->scale);
  EpilogueOps ops;
  ops.base = x->d;
  ops.base_polys = 1;
  key_switch_pipeline(x->d + x->poly_stride(), x->moduli_id, key, nullptr, ops, out->d);
  return out;
}

}  // namespace fhe_b200
