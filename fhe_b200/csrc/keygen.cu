// Randomness, key generation, encryption and decryption on the device
// (DESILO FHE src/random/random.cpp, random_number_generator.cpp,
// ckks/core_key.cpp, ckks/core.cpp:35-200, ckks/core_random.cpp).
//
// The reference draws every random word from one ChaCha20 stream (20 rounds,
// 64-bit block counter in words 12-13, the 2-word nonce in 14-15); each block
// gives four samples, so sample i of a draw comes from block counter0 + i / 4.
// That makes the stream parallel by block: one thread per block reproduces the
// reference's samples exactly, and the engine advances its counter on the host.
#include <random>

#include "engine.hpp"

namespace fhe_b200 {

namespace {

#include "cdt_table.inc"

constexpr int kThreads = 256;
constexpr int kCdtDepth = 5;   // ceil(log2(6 * 3.2))
constexpr int kCdtSize = 31;   // 2^depth - 1 nodes

__constant__ unsigned long long c_cdt[2 * kCdtSize];

inline unsigned grid_for(long long work) {
  long long b = (work + kThreads - 1) / kThreads;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

__device__ __forceinline__ uint32_t rotl(uint32_t x, int s) { return (x << s) | (x >> (32 - s)); }

#define FHE_QR(a, b, c, d)    \
  x[a] += x[b];               \
  x[d] = rotl(x[d] ^ x[a], 16); \
  x[c] += x[d];               \
  x[b] = rotl(x[b] ^ x[c], 12); \
  x[a] += x[b];               \
  x[d] = rotl(x[d] ^ x[a], 8);  \
  x[c] += x[d];               \
  x[b] = rotl(x[b] ^ x[c], 7)

// chacha20 (random.cpp:76-92): ten double rounds, then the state added back.
__device__ void chacha_block(const RngState &st, unsigned long long counter, uint32_t out[16]) {
  uint32_t in[16];
  in[0] = 1634760805u;
  in[1] = 857760878u;
  in[2] = 2036477234u;
  in[3] = 1797285236u;
  for (int i = 0; i < 8; i++) in[4 + i] = st.seed[i];
  in[12] = static_cast<uint32_t>(counter);
  in[13] = static_cast<uint32_t>(counter >> 32);
  in[14] = st.nonce[0];
  in[15] = st.nonce[1];
  uint32_t x[16];
  for (int i = 0; i < 16; i++) x[i] = in[i];
  for (int r = 0; r < 10; r++) {
    FHE_QR(0, 4, 8, 12);
    FHE_QR(1, 5, 9, 13);
    FHE_QR(2, 6, 10, 14);
    FHE_QR(3, 7, 11, 15);
    FHE_QR(0, 5, 10, 15);
    FHE_QR(1, 6, 11, 12);
    FHE_QR(2, 7, 8, 13);
    FHE_QR(3, 4, 9, 14);
  }
  for (int i = 0; i < 16; i++) out[i] = x[i] + in[i];
}
#undef FHE_QR

// rand_int (random.cpp:94-131): floor((max * x_high + floor(max * x_low / 2^64)) / 2^64)
// for the 128-bit word (x_high, x_low) of each lane, plus shift.
__device__ __forceinline__ int64_t uniform_sample(const uint32_t *w, uint64_t max_value, int64_t shift) {
  const uint64_t x_low = (static_cast<uint64_t>(w[0]) << 32) | w[1];
  const uint64_t x_high = (static_cast<uint64_t>(w[2]) << 32) | w[3];
  const uint64_t alpha = __umul64hi(max_value, x_low);
  const uint64_t lo = max_value * x_high;
  const uint64_t hi = __umul64hi(max_value, x_high);
  const uint64_t sum = lo + alpha;
  return static_cast<int64_t>(hi + (sum < lo ? 1 : 0)) + shift;
}

// Rows of N uniform samples: row j draws blocks counter0 + j N/4 .. with bound
// q[prime_base + j] (assign_a, core_random.cpp:32-45) or `fixed_max` when nonzero.
__global__ void rng_uniform_kernel(RngState st, unsigned long long counter0, int log_n, int rows,
                                   const uint64_t *q, int prime_base, uint64_t fixed_max,
                                   int64_t shift, int64_t *out, long long row_stride) {
  const long long blocks_per_row = 1LL << (log_n - 2);
  const long long b = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (b >= blocks_per_row * rows) return;
  const int row = static_cast<int>(b / blocks_per_row);
  const long long bi = b - row * blocks_per_row;
  uint32_t w[16];
  chacha_block(st, counter0 + static_cast<unsigned long long>(b), w);
  const uint64_t max_value = fixed_max ? fixed_max : q[prime_base + row];
  int64_t *o = out + row * row_stride + 4 * bi;
  for (int lane = 0; lane < 4; lane++) o[lane] = uniform_sample(w + 4 * lane, max_value, shift);
}

// discrete_gaussian (random.cpp:133-170): sign bit from the high word, then a walk
// down the CDT tree comparing (x_high >> 1, x_low) with each node.
__global__ void rng_gaussian_kernel(RngState st, unsigned long long counter0, int log_n,
                                    int64_t *out) {
  const long long b = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (b >= (1LL << (log_n - 2))) return;
  uint32_t w[16];
  chacha_block(st, counter0 + static_cast<unsigned long long>(b), w);
  for (int lane = 0; lane < 4; lane++) {
    const uint32_t *l = w + 4 * lane;
    const uint64_t x_low = (static_cast<uint64_t>(l[0]) << 32) | l[1];
    uint64_t x_high = (static_cast<uint64_t>(l[2]) << 32) | l[3];
    const int64_t sign_bit = static_cast<int64_t>(x_high & 1);
    x_high >>= 1;
    int jump = 1, current = 0, counter = 0;
    for (int depth = 0; depth < kCdtDepth; depth++) {
      const uint64_t th = c_cdt[counter + current + kCdtSize];
      const uint64_t tl = c_cdt[counter + current];
      const int ge = (x_high > th) || (x_high == th && x_low >= tl);
      current = 2 * current + ge;
      counter += jump;
      jump *= 2;
    }
    out[4 * b + lane] = (sign_bit * 2 - 1) * static_cast<int64_t>(current);
  }
}

// assign_sparse_ternary_chain (random_number_generator.cpp:62-92): hamming_weight + 1
// uniform indices below N from consecutive blocks, the first fixing the count of
// -1 entries, then the sequential swaps.  One thread: the swaps depend on order.
__global__ void rng_sparse_ternary_kernel(RngState st, unsigned long long counter0, int n,
                                          int hamming_weight, int64_t *out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  auto index_at = [&](int i) -> int64_t {
    uint32_t w[16];
    chacha_block(st, counter0 + static_cast<unsigned long long>(i / 4), w);
    return uniform_sample(w + 4 * (i % 4), static_cast<uint64_t>(n), 0);
  };
  const int64_t negative_count = index_at(0) % hamming_weight;
  for (int i = 0; i < n; i++) out[i] = i < negative_count ? -1 : (i < hamming_weight ? 1 : 0);
  for (int i = 0; i < hamming_weight; i++) {
    const int64_t j = index_at(i + 1);
    const int64_t t = out[i];
    out[i] = out[j];
    out[j] = t;
  }
}

// tile_unsigned_reduce_2q_to_q (single.cpp:315-326): one signed chain onto `limbs`.
__global__ void tile_kernel(PrimeTables t, int log_n, int limbs, int prime_base, const int64_t *x,
                            int64_t *y, long long y_stride) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= (static_cast<long long>(limbs) << log_n)) return;
  const int j = static_cast<int>(i >> log_n);
  const int c = static_cast<int>(i & ((1LL << log_n) - 1));
  const int64_t q = static_cast<int64_t>(t.q[prime_base + j]);
  const int64_t v = x[c];
  y[j * y_stride + c] = v < 0 ? v + q : guard(v, q);
}

// make_signed (unit.cpp:36-42, unsigned comparison with q/2) of one chain modulo
// q_src, then tile_unsigned_reduce_2q_to_q onto `limbs` (make_signed_tile, core.cpp:
// 1085-1108).
__global__ void signed_tile_kernel(PrimeTables t, int log_n, int limbs, int prime_base,
                                   const int64_t *x, int64_t q_src, int64_t *y, long long y_stride) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= (static_cast<long long>(limbs) << log_n)) return;
  const int j = static_cast<int>(i >> log_n);
  const int c = static_cast<int>(i & ((1LL << log_n) - 1));
  const int64_t v = x[c];
  const int64_t s = static_cast<uint64_t>(v) <= static_cast<uint64_t>(q_src >> 1) ? v : v - q_src;
  const int64_t q = static_cast<int64_t>(t.q[prime_base + j]);
  y[j * y_stride + c] = s < 0 ? s + q : guard(s, q);
}

// One word of y[j] = op(a[j], b[j]): word i (global index over the limbs) of limb j.
__device__ __forceinline__ int64_t pointwise_word(int op, long long i, int log_n, int j, int64_t ai,
                                                  int64_t bi, const LimbScalars &c, uint64_t q,
                                                  uint64_t k) {
  const int64_t qs = static_cast<int64_t>(q), q2 = qs << 1;
  int64_t v = 0;
  switch (op) {
    case kOpMult: v = mont_mult_lazy(ai, bi, q, k); break;
    case kOpAddReduce: v = guard(guard(ai + bi, q2), qs); break;
    case kOpSubReduce: v = guard(guard(ai + q2 - bi, q2), qs); break;
    case kOpReduce: v = guard(ai, qs); break;
    case kOpEnter: v = mont_mult_lazy(ai, c.v[j], q, k); break;
    case kOpNegate: v = qs - ai; break;
    case kOpAddScalarFirst: v = guard(ai + ((i & ((1LL << log_n) - 1)) == 0 ? c.v[j] : 0), qs); break;
    case kOpEnterReduce: v = guard(mont_mult_lazy(ai, c.v[j], q, k), qs); break;
    case kOpMonomial: {
      const int64_t m = c.v[j];
      v = (i & ((1LL << log_n) - 1)) == (1LL << (log_n - 1)) ? (m < 0 ? m + qs : guard(m, qs)) : 0;
      break;
    }
  }
  return v;
}

__device__ __forceinline__ bool pointwise_reads_a(int op) { return op != kOpMonomial; }
__device__ __forceinline__ bool pointwise_reads_b(int op) {
  return op == kOpMult || op == kOpAddReduce || op == kOpSubReduce;
}

// y[j] = op(a[j], b[j]) over `limbs` limbs of N words; a, b, y are [limbs][N]
// views (any may alias).  W consecutive words per thread: W = 4 moves them as
// 16-byte vectors (every pointer 16-byte aligned), which keeps enough loads in
// flight to stream at HBM speed; W = 1 serves unaligned views.
// Limb j runs modulo prime prime_base + j % period (period = limbs but for batches of
// polynomials laid out back to back).
template <int W>
__global__ void pointwise_kernel(PrimeTables t, int op, int log_n, int limbs, int period,
                                 int prime_base, const int64_t *a, const int64_t *b, LimbScalars c,
                                 int64_t *y) {
  const long long i0 = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) * W;
  if (i0 >= (static_cast<long long>(limbs) << log_n)) return;
  const int j = static_cast<int>(i0 >> log_n) % period;  // W <= N: the words share a limb
  const int prime = prime_base + j;
  const uint64_t q = t.q[prime], k = t.k[prime];
  int64_t av[W] = {}, bv[W] = {}, yv[W];
  if (W == 4) {
    if (pointwise_reads_a(op)) {
      const longlong2 x0 = reinterpret_cast<const longlong2 *>(a + i0)[0];
      const longlong2 x1 = reinterpret_cast<const longlong2 *>(a + i0)[1];
      av[0] = x0.x; av[1] = x0.y; av[2 % W] = x1.x; av[3 % W] = x1.y;
    }
    if (pointwise_reads_b(op)) {
      const longlong2 x0 = reinterpret_cast<const longlong2 *>(b + i0)[0];
      const longlong2 x1 = reinterpret_cast<const longlong2 *>(b + i0)[1];
      bv[0] = x0.x; bv[1] = x0.y; bv[2 % W] = x1.x; bv[3 % W] = x1.y;
    }
  } else {
    if (pointwise_reads_a(op)) av[0] = a[i0];
    if (pointwise_reads_b(op)) bv[0] = b[i0];
  }
#pragma unroll
  for (int w = 0; w < W; w++) yv[w] = pointwise_word(op, i0 + w, log_n, j, av[w], bv[w], c, q, k);
  if (W == 4) {
    reinterpret_cast<longlong2 *>(y + i0)[0] = make_longlong2(yv[0], yv[1 % W]);
    reinterpret_cast<longlong2 *>(y + i0)[1] = make_longlong2(yv[2 % W], yv[3 % W]);
  } else {
    y[i0] = yv[0];
  }
}

}  // namespace

// ------------------------------------------------------------------ host --

void Engine::seed(const uint32_t *seed_words, const uint8_t *nonce) {
  // RandomNumberGenerator(1, N, seed, nonce) (random_number_generator.cpp:9-55):
  // missing parts come from the system's random device.
  std::random_device rd;
  for (int i = 0; i < 8; i++) rng_.seed[i] = seed_words ? seed_words[i] : rd();
  for (int i = 0; i < 2; i++) rng_.nonce[i] = nonce ? nonce[i] : (rd() & 0xff);
  rng_counter_ = 0;
}

void Engine::ensure_rng_tables() {
  if (cdt_uploaded_) return;
  static_assert(sizeof(kCdtTree) == 2 * kCdtSize * sizeof(unsigned long long), "CDT tree size");
  check(cudaMemcpyToSymbolAsync(c_cdt, kCdtTree, sizeof(kCdtTree), 0, cudaMemcpyHostToDevice,
                                stream_),
        "upload CDT tree");
  synchronize();
  cdt_uploaded_ = true;
}

void Engine::draw_uniform(int64_t *out, long long row_stride, int rows, int prime_base,
                          uint64_t fixed_max, int64_t shift) {
  const long long blocks = (static_cast<long long>(params.n) >> 2) * rows;
  note_launch();
  rng_uniform_kernel<<<grid_for(blocks), kThreads, 0, stream_>>>(
      rng_, rng_counter_, params.log_n, rows, tables_.q, prime_base, fixed_max, shift, out,
      row_stride);
  rng_counter_ += static_cast<unsigned long long>(blocks);
  check(cudaGetLastError(), "random draw");
}

void Engine::draw_gaussian(int64_t *out) {
  ensure_rng_tables();
  const long long blocks = static_cast<long long>(params.n) >> 2;
  note_launch();
  rng_gaussian_kernel<<<grid_for(blocks), kThreads, 0, stream_>>>(rng_, rng_counter_, params.log_n,
                                                                  out);
  rng_counter_ += static_cast<unsigned long long>(blocks);
  check(cudaGetLastError(), "gaussian draw");
}

void Engine::tile(const int64_t *chain, int limbs, int prime_base, int64_t *y, long long y_stride) {
  note_launch();
  tile_kernel<<<grid_for(static_cast<long long>(limbs) << params.log_n), kThreads, 0, stream_>>>(
      tables_, params.log_n, limbs, prime_base, chain, y, y_stride);
  check(cudaGetLastError(), "tile");
}

void Engine::signed_tile(const int64_t *chain, int64_t q_src, int limbs, int prime_base,
                         int64_t *y, long long y_stride) {
  note_launch();
  signed_tile_kernel<<<grid_for(static_cast<long long>(limbs) << params.log_n), kThreads, 0,
                       stream_>>>(tables_, params.log_n, limbs, prime_base, chain, q_src, y,
                                  y_stride);
  check(cudaGetLastError(), "signed tile");
}

void Engine::pointwise(int op, int limbs, int prime_base, const int64_t *a, const int64_t *b,
                       const int64_t *constants, int64_t *y, int period) {
  if (period <= 0 || period > limbs) period = limbs;
  // The per-limb constants (one per prime of the period) travel by value in the
  // launch (no copy, no wait).
  LimbScalars c{};
  if (constants) {
    if (period > kMaxScalarLimbs) throw std::invalid_argument("pointwise: too many limbs.");
    for (int j = 0; j < period; j++) c.v[j] = constants[j];
  }
  const long long words = static_cast<long long>(limbs) << params.log_n;
  const bool aligned = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) |
                         reinterpret_cast<uintptr_t>(y)) & 15) == 0;
  check(timed("pointwise", [&] {
          note_launch();
          if (aligned && params.n >= 4)
            pointwise_kernel<4><<<grid_for(words / 4), kThreads, 0, stream_>>>(
                tables_, op, params.log_n, limbs, period, prime_base, a, b, c, y);
          else
            pointwise_kernel<1><<<grid_for(words), kThreads, 0, stream_>>>(
                tables_, op, params.log_n, limbs, period, prime_base, a, b, c, y);
          return cudaGetLastError();
        }),
        "pointwise");
}

void Engine::ntt_in_place(int64_t *x, int limbs, int prime_base, long long stride, int polys) {
  check(launch_to_ntt(tables_, params.log_n, polys, limbs, prime_base, x, stride, x, stride, stream_),
        "to_ntt");
}

void Engine::intt_in_place(int64_t *x, int limbs, int prime_base, long long stride, int polys) {
  check(launch_to_intt(tables_, params.log_n, polys, limbs, prime_base, x, stride, x, stride,
                       stream_),
        "to_intt");
}

static void validate_level(const std::string &fn, int level, int max_level) {
  if (level < 0 || level > max_level)
    throw std::runtime_error(fn + ": the target level cannot be reached with the current engine "
                                  "parameters.");
}

static void validate_key_level(const std::string &fn, const Data &key, int level) {
  if (key.level() < level)
    throw std::runtime_error(fn + ": the target level cannot be reached with the provided keys.");
}

std::unique_ptr<Data> Engine::create_secret_key(int level) {
  // CKKSCore::create_secret_key (core_key.cpp:9-28): uniform ternary, tiled, NTT.
  validate_level("Create Secret Key", level, params.max_level());
  const int mid = params.moduli_id(level);
  auto sk = make_data(kSecretKey, kFlagNtt | kFlagSpecial, mid, 1, 1.0L);
  int64_t *chain = alloc_words(params.n);
  draw_uniform(chain, 0, 1, 0, 3, -1);
  tile(chain, sk->chains, mid, sk->d, params.n);
  free_words(chain);
  ntt_in_place(sk->d, sk->chains, mid, sk->poly_stride(), 1);
  return sk;
}

std::unique_ptr<Data> Engine::create_secret_key(const int64_t *secret, int count, int level) {
  // create_secret_key(std::vector<int64_t>&) (core_key.cpp:30-50), zero-padded to N.
  const std::string fn = "Create Custom Secret Key";
  validate_level(fn, level, params.max_level());
  if (count < 0 || count > params.n || (count > 0 && secret == nullptr))
    throw std::runtime_error(fn + ": the input secret does not fit the coefficient count.");
  const int mid = params.moduli_id(level);
  auto sk = make_data(kSecretKey, kFlagNtt | kFlagSpecial, mid, 1, 1.0L);
  std::vector<int64_t> host(params.n, 0);
  for (int i = 0; i < count; i++) host[i] = secret[i];
  int64_t *chain = alloc_words(params.n);
  check(cudaMemcpyAsync(chain, host.data(), params.n * sizeof(int64_t), cudaMemcpyHostToDevice,
                        stream_),
        "upload secret");
  tile(chain, sk->chains, mid, sk->d, params.n);
  free_words(chain);
  ntt_in_place(sk->d, sk->chains, mid, sk->poly_stride(), 1);
  synchronize();  // the host vector is released on return
  return sk;
}

std::unique_ptr<Data> Engine::create_sparse_secret_key(int hamming_weight, int level) {
  // create_sparse_secret_key (core_key.cpp:52-77; engine default weight 128).
  if (hamming_weight > params.n)
    throw std::runtime_error(
        "Create Sparse Secret Key: the given hamming weight is bigger than the coefficient count.");
  validate_level("Create Sparse Secret Key", level, params.max_level());
  const int mid = params.moduli_id(level);
  auto sk = make_data(kSecretKey, kFlagNtt | kFlagSparse | kFlagSpecial, mid, 1, 1.0L);
  int64_t *chain = alloc_words(params.n);
  note_launch();
  rng_sparse_ternary_kernel<<<1, 1, 0, stream_>>>(rng_, rng_counter_, params.n, hamming_weight,
                                                   chain);
  check(cudaGetLastError(), "sparse ternary");
  rng_counter_ += static_cast<unsigned long long>((hamming_weight + 1 + 3) / 4);
  tile(chain, sk->chains, mid, sk->d, params.n);
  free_words(chain);
  ntt_in_place(sk->d, sk->chains, mid, sk->poly_stride(), 1);
  return sk;
}

std::unique_ptr<Data> Engine::create_public_key(const Data &sk, int level) {
  // CKKSCore::create_public_key (core_key.cpp:79-109).
  const std::string fn = "Create Public Key";
  if (sk.type != kSecretKey) throw std::invalid_argument(fn + ": the key is not a secret key.");
  validate_level(fn, level, params.max_level());
  validate_key_level(fn, sk, level);
  const int mid = params.moduli_id(level);
  const int L = params.chains(mid);
  const long long ps = static_cast<long long>(L) * params.n;
  auto pk = make_data(kPublicKey, kFlagNtt, mid, 2, 1.0L);
  int64_t *chain = alloc_words(params.n);
  int64_t *error = alloc_words(static_cast<size_t>(ps));
  draw_gaussian(chain);
  tile(chain, L, mid, error, params.n);
  ntt_in_place(error, L, mid, ps, 1);
  int64_t *b = pk->d, *a = pk->d + ps;
  draw_uniform(a, params.n, L, mid, 0, 0);
  const int64_t *s = sk.d + static_cast<long long>(mid - sk.moduli_id) * params.n;
  pointwise(kOpMult, L, mid, a, s, nullptr, b);
  pointwise(kOpSubReduce, L, mid, error, b, nullptr, b);
  free_words(chain);
  free_words(error);
  return pk;
}

std::unique_ptr<Data> Engine::create_key_switching_key(const Data &from, const Data &to, int level,
                                                       int type) {
  // CKKSCore::create_key_switching_key (core_key.cpp:111-166).
  const int mid = params.moduli_id(level);
  const int L = params.chains(mid);
  const int P = params.chains(mid, true);
  const int n = params.n;
  const auto parts = params.partitions(mid, mid);
  const long long ps = static_cast<long long>(P) * n;
  auto ksk = make_data(type, kFlagNtt | kFlagSpecial, mid, 2 * static_cast<int>(parts.size()), 1.0L);
  std::vector<int64_t> ppr(L);
  for (int j = 0; j < L; j++) ppr[j] = params.p_product_mult_r[mid + j];
  int64_t *p_from = alloc_words(static_cast<size_t>(L) * n);
  int64_t *chain = alloc_words(n);
  int64_t *error = alloc_words(static_cast<size_t>(ps));
  pointwise(kOpEnter, L, mid, from.d + static_cast<long long>(mid - from.moduli_id) * n, nullptr,
            ppr.data(), p_from);
  const int64_t *s_to = to.d + static_cast<long long>(mid - to.moduli_id) * n;
  for (size_t pi = 0; pi < parts.size(); pi++) {
    int64_t *b = ksk->d + static_cast<long long>(2 * pi) * ps;
    int64_t *a = b + ps;
    draw_gaussian(chain);
    tile(chain, P, mid, error, n);
    ntt_in_place(error, P, mid, ps, 1);
    draw_uniform(a, n, P, mid, 0, 0);
    pointwise(kOpMult, P, mid, a, s_to, nullptr, b);
    pointwise(kOpSubReduce, P, mid, error, b, nullptr, b);
    const int start = parts[pi].start, size = parts[pi].size;
    pointwise(kOpAddReduce, size, mid + start, p_from + static_cast<long long>(start) * n,
              b + static_cast<long long>(start) * n, nullptr, b + static_cast<long long>(start) * n);
  }
  free_words(p_from);
  free_words(chain);
  free_words(error);
  return ksk;
}

static void validate_switching_key_level(const std::string &fn, const Parameters &p, const Data &sk,
                                         int level) {
  validate_level(fn, level, p.max_level());
  validate_key_level(fn, sk, level);
  if (level < 0 || level > p.max_key_switching_level())
    throw std::runtime_error(fn + ": the target level cannot be reached with the current engine "
                                  "parameters.");
}

std::unique_ptr<Data> Engine::create_relinearization_key(const Data &sk, int level) {
  // create_relinearization_key (core_key.cpp:168-190): switch from s^2 to s.
  const std::string fn = "Create Relinearization Key";
  if (sk.type != kSecretKey) throw std::invalid_argument(fn + ": the key is not a secret key.");
  validate_switching_key_level(fn, params, sk, level);
  auto squared = make_data(kSecretKey, sk.flag, sk.moduli_id, 1, 1.0L);
  pointwise(kOpMult, sk.chains, sk.moduli_id, sk.d, sk.d, nullptr, squared->d);
  return create_key_switching_key(*squared, sk, level, kRelinearizationKey);
}

std::unique_ptr<Data> Engine::rotated_secret_key(const Data &sk, int ntt_delta) {
  // CKKSCore::rotate(key, delta, invert_delta) (core_key.cpp:195-227): an NTT-form
  // gather of every limb.
  auto out = make_data(kSecretKey, sk.flag, sk.moduli_id, 1, 1.0L);
  check(launch_permute_gather(params.n, 1, sk.chains, sk.d, sk.poly_stride(),
                              device_ntt_permutation(ntt_delta), out->d, out->poly_stride(),
                              stream_),
        "rotate secret key");
  return out;
}

std::unique_ptr<Data> Engine::create_fixed_rotation_key(const Data &sk, int delta, int level) {
  // create_fixed_rotation_key (core_key.cpp:229-242): key switching from s to the
  // secret rotated by N/2 - delta; `delta` is already normalised.
  const std::string fn = "Create Fixed Rotation Key";
  if (sk.type != kSecretKey) throw std::invalid_argument(fn + ": the key is not a secret key.");
  validate_switching_key_level(fn, params, sk, level);
  auto rotated = rotated_secret_key(sk, params.n / 2 - delta);
  auto key = create_key_switching_key(sk, *rotated, level, kFixedRotationKey);
  key->delta = delta;
  return key;
}

std::vector<std::unique_ptr<Data>> Engine::create_rotation_keys(const Data &sk, int level) {
  // create_rotation_key (core_key.cpp:258-268): one fixed key per power of two below N/2.
  const std::string fn = "Create Rotation Key";
  if (sk.type != kSecretKey) throw std::invalid_argument(fn + ": the key is not a secret key.");
  validate_switching_key_level(fn, params, sk, level);
  std::vector<std::unique_ptr<Data>> keys;
  for (int delta = 1; delta < params.n / 2; delta <<= 1) {
    auto rotated = rotated_secret_key(sk, params.n / 2 - delta);
    auto key = create_key_switching_key(sk, *rotated, level, kFixedRotationKey);
    key->delta = delta;
    keys.push_back(std::move(key));
  }
  return keys;
}

std::unique_ptr<Data> Engine::create_conjugation_key(const Data &sk, int level) {
  // create_conjugation_key (core_key.cpp:244-256): switch from conj(s) to s.
  const std::string fn = "Create Conjugation Key";
  if (sk.type != kSecretKey) throw std::invalid_argument(fn + ": the key is not a secret key.");
  validate_switching_key_level(fn, params, sk, level);
  auto conjugated = rotated_secret_key(sk, -1);
  return create_key_switching_key(*conjugated, sk, level, kConjugationKey);
}

std::unique_ptr<Data> Engine::encrypt(const Data &pt, const Data &key) {
  if (pt.type != kUnitPlaintext || pt.polys != 1)
    throw std::invalid_argument("Encrypt: the input is not a unit plaintext.");
  if (pt.is_ntt()) throw std::invalid_argument("Encrypt: the input plaintext is in NTT form.");
  const int mid = pt.moduli_id;
  const int L = params.chains(mid);
  const int n = params.n;
  const long long ps = static_cast<long long>(L) * n;
  auto ct = make_data(kUnitCiphertext, pt.flag & ~kFlagSpecial, mid, 2, pt.scale);
  int64_t *c0 = ct->d, *c1 = ct->d + ps;
  int64_t *chain = alloc_words(n);
  if (key.type == kPublicKey) {
    // CKKSCore::encrypt(pt, pk) (core.cpp:35-85).
    if (key.moduli_id > mid)
      throw std::runtime_error("Encrypt: the level of the input plaintext is greater than that of "
                               "the input public key.");
    int64_t *e0 = alloc_words(static_cast<size_t>(ps));
    int64_t *e1 = alloc_words(static_cast<size_t>(ps));
    int64_t *u = alloc_words(static_cast<size_t>(ps));
    draw_gaussian(chain);
    tile(chain, L, mid, e0, n);
    draw_gaussian(chain);
    tile(chain, L, mid, e1, n);
    draw_uniform(chain, 0, 1, 0, 2, 0);
    pointwise(kOpAddReduce, L, mid, pt.d, e0, nullptr, e0);
    tile(chain, L, mid, u, n);
    ntt_in_place(u, L, mid, ps, 1);
    const long long off = static_cast<long long>(mid - key.moduli_id) * n;
    const long long kps = key.poly_stride();
    pointwise(kOpMult, L, mid, u, key.d + off, nullptr, c0);
    pointwise(kOpMult, L, mid, u, key.d + kps + off, nullptr, c1);
    intt_in_place(ct->d, L, mid, ps, 2);
    pointwise(kOpAddReduce, L, mid, c0, e0, nullptr, c0);
    pointwise(kOpAddReduce, L, mid, c1, e1, nullptr, c1);
    free_words(e0);
    free_words(e1);
    free_words(u);
  } else if (key.type == kSecretKey) {
    // CKKSCore::encrypt(pt, sk) (core.cpp:87-122).
    if (key.moduli_id > mid)
      throw std::runtime_error("Encrypt: the level of the input plaintext is greater than that of "
                               "the input secret key.");
    int64_t *e = alloc_words(static_cast<size_t>(ps));
    draw_gaussian(chain);
    tile(chain, L, mid, e, n);
    pointwise(kOpAddReduce, L, mid, pt.d, e, nullptr, e);
    draw_uniform(c1, n, L, mid, 0, 0);
    const int64_t *s = key.d + static_cast<long long>(mid - key.moduli_id) * n;
    pointwise(kOpMult, L, mid, c1, s, nullptr, c0);
    pointwise(kOpReduce, L, mid, c0, nullptr, nullptr, c0);
    intt_in_place(ct->d, L, mid, ps, 2);
    pointwise(kOpSubReduce, L, mid, e, c0, nullptr, c0);
    free_words(e);
  } else {
    free_words(chain);
    throw std::invalid_argument("Encrypt: the key is neither a public key nor a secret key.");
  }
  free_words(chain);
  return ct;
}

std::unique_ptr<Data> Engine::decrypt(const Data &ct, const Data &sk) {
  // CKKSEngine::decrypt_to_unit_plaintext (engine_decrypt.cpp:99-126) with
  // CKKSCore::decrypt_duo / decrypt_trio (core.cpp:124-200).
  const std::string fn = "Decrypt Unit Ciphertext To Unit Plaintext";
  if (ct.polys != 2 && ct.polys != 3)
    throw std::runtime_error(fn + ": the input " + std::string(ct.type_name()) +
                             " should have either 2 or 3 polynomials.");
  if (sk.type != kSecretKey) throw std::invalid_argument(fn + ": the key is not a secret key.");
  if (ct.moduli_id < sk.moduli_id)
    throw std::runtime_error(fn + ": the level of the input " + std::string(ct.type_name()) +
                             " is greater than that of the input secret key.");
  std::unique_ptr<Data> hold;
  const Data *x = &ct;
  if (x->is_rescaled()) {
    hold = level_down_any(*x, x->level() - 1);
    x = hold.get();
  }
  const int mid = x->moduli_id;
  const int L = x->chains;
  const int n = params.n;
  const long long ps = static_cast<long long>(L) * n;
  const int64_t *s = sk.d + static_cast<long long>(mid - sk.moduli_id) * n;
  auto pt = make_data(kUnitPlaintext, x->flag & kFlagComplex, mid, 1, x->scale);
  if (x->polys == 2) {
    if (x->is_ntt()) {
      hold = to_intt(*x);
      x = hold.get();
    }
    check(launch_to_ntt(tables_, params.log_n, 1, L, mid, x->d + ps, ps, pt->d, ps, stream_),
          "to_ntt");
    pointwise(kOpMult, L, mid, pt->d, s, nullptr, pt->d);
    intt_in_place(pt->d, L, mid, ps, 1);
    pointwise(kOpAddReduce, L, mid, x->d, pt->d, nullptr, pt->d);
    return pt;
  }
  // Three polynomials, NTT form: (c0 + c1 s + c2 s^2), each product brought back
  // with iNTT and N^-1 enter-exit before the sums (decrypt_trio).
  if (!x->is_ntt()) {
    hold = to_ntt(*x);
    x = hold.get();
  }
  int64_t *s2 = alloc_words(static_cast<size_t>(ps));
  int64_t *t0 = alloc_words(static_cast<size_t>(ps));
  int64_t *t2 = alloc_words(static_cast<size_t>(ps));
  pointwise(kOpMult, L, mid, s, s, nullptr, s2);
  pointwise(kOpMult, L, mid, x->d + ps, s, nullptr, pt->d);
  intt_in_place(pt->d, L, mid, ps, 1);
  check(launch_to_intt(tables_, params.log_n, 1, L, mid, x->d, ps, t0, ps, stream_), "to_intt");
  pointwise(kOpAddReduce, L, mid, t0, pt->d, nullptr, pt->d);
  pointwise(kOpMult, L, mid, x->d + 2 * ps, s2, nullptr, t2);
  intt_in_place(t2, L, mid, ps, 1);
  pointwise(kOpAddReduce, L, mid, pt->d, t2, nullptr, pt->d);
  free_words(s2);
  free_words(t0);
  free_words(t2);
  return pt;
}

}  // namespace fhe_b200
