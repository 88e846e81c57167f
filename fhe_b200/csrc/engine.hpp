// The B200 CKKS engine: HBM-resident objects and the CKKS operations of the
// reference's CKKSEngine (DESILO FHE, src/ckks/engine.h) executed by the device
// kernels of kernels.cu / ntt.cuh.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <complex>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "kernels.cuh"
#include "params.hpp"

namespace fhe_b200 {

// An NVTX range for the lifetime of the object (a no-op unless an Nsight tool is
// attached): C-ABI calls and kernel families show up by name on profiler timelines.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

enum DataFlag : int {
  kFlagNone = 0,
  kFlagComplex = 1,
  kFlagNtt = 2,
  kFlagRescaled = 4,
  kFlagSparse = 8,
  kFlagSpecial = 16,
};

enum DataType : int {
  kDecomposed = 0,  // DecomposedUnitCiphertext: [partitions][L+K][N], NTT form
  kSecretKey = 1,
  kPublicKey = 2,
  kRelinearizationKey = 3,
  kUnitCiphertext = 4,
  kUnitPlaintext = 5,
  kFixedRotationKey = 6,
  kConjugationKey = 7,
  kKeySwitchingKey = 8,
};

class CudaError : public std::runtime_error {
 public:
  explicit CudaError(const std::string &what) : std::runtime_error(what) {}
};

class Engine;

// Element-wise operations of Engine::pointwise over [limbs][N] views.
enum PointwiseOp : int {
  kOpMult = 0,            // mont_mult(a, b)
  kOpAddReduce = 1,       // mont_add_reduce_2q_to_q(a, b)
  kOpSubReduce = 2,       // mont_sub_reduce_2q_to_q: a - b
  kOpReduce = 3,          // reduce_2q_to_q(a)
  kOpEnter = 4,           // mont_enter(a, c[limb])
  kOpNegate = 5,          // negate_make_unsigned: q - a
  kOpAddScalarFirst = 6,  // add_scalar (c[limb] on coefficient 0) then reduce_2q_to_q
  kOpEnterReduce = 7,     // mont_enter(a, c[limb]) then reduce_2q_to_q
  kOpMonomial = 8,        // c[limb] X^(N/2), signed c tiled per limb (encode_imaginary)
};

// The ChaCha20 key and nonce of the engine's random stream (RandomNumberGenerator,
// random_number_generator.cpp:9-55); the block counter is kept by the engine.
// Operations replayed as CUDA graphs (the first element of a graph key).
enum GraphOp : uint64_t { kGraphBootstrap = 1, kGraphMultiplyRotate = 2 };

struct RngState {
  uint32_t seed[8];
  uint32_t nonce[2];
};

// One HBM-resident object (key, ciphertext or plaintext).
struct Data {
  Engine *engine = nullptr;
  int type = 0;
  int flag = 0;
  int moduli_id = 0;
  int polys = 0;
  int chains = 0;  // limbs per polynomial
  int delta = 0;
  long double scale = 1.0L;
  int64_t *d = nullptr;
  uint64_t serial = 0;  // unique per engine, never reused (keys captured graphs)
  mutable bool copy_pending = false;  // a download may still read d

  size_t words() const;
  long long poly_stride() const;
  int level() const;  // data.h:21-32
  bool is_ntt() const { return flag & kFlagNtt; }
  bool is_rescaled() const { return flag & kFlagRescaled; }
  const char *type_name() const;
  ~Data();
};

// One stage of the baby-step giant-step linear transform of bootstrapping
// (PlainMatrix, data/plain_matrix.h; made by make_bootstrap_stage,
// engine_bootstrap.cpp:8-67): the rotation steps and the twiddle diagonals, encoded
// with the special primes, rescaled and in NTT form.
struct BootstrapStage {
  int level = 0;
  int inner = 0;
  int outer = 0;
  std::vector<int> inner_deltas;  // inner_deltas[0] == 0
  std::vector<int> outer_deltas;
  std::vector<std::pair<int, std::vector<int>>> process_order;  // delta -> outer indices
  std::map<int, std::map<int, std::unique_ptr<Data>>> diagonals;  // [outer][inner]
};

// BootstrapKey (data/bootstrap.h:24-44): fixed rotation keys per normalised delta
// (with their NTT-form permutation, made on use), the coefficients-to-slots and
// slots-to-coefficients stages, and the small bootstrap key.
struct BootstrapKey {
  uint64_t serial = 0;  // unique per engine, never reused
  int stage_count = 0;
  int inner_loop_shift = 0;
  std::map<int, std::unique_ptr<Data>> rotation_keys;
  std::vector<BootstrapStage> coeff_to_slot;
  std::vector<BootstrapStage> slot_to_coeff;
  std::unique_ptr<Data> to_sparse;
  std::unique_ptr<Data> to_dense;
  size_t bytes() const;
};


class Engine {
 public:
  explicit Engine(const Config &config);
  ~Engine();
  Engine(const Engine &) = delete;
  Engine &operator=(const Engine &) = delete;

  const Parameters params;

  cudaStream_t stream() const { return stream_; }
  // Work queued on the previous stream finishes first, so results made there are
  // ready for the new one.
  void set_stream(cudaStream_t s) {
    synchronize();
    stream_ = s ? s : own_stream_;
  }
  void synchronize();

  // Device memory from the stream-ordered pool.
  int64_t *alloc_words(size_t words);
  void free_words(int64_t *p);
  // Frees an object's words; after a pending download, in order behind it.
  void release(int64_t *p, bool copy_pending);

  std::unique_ptr<Data> make_data(int type, int flag, int moduli_id, int polys, long double scale,
                                  cudaStream_t alloc_stream = nullptr);
  std::unique_ptr<Data> upload(int type, int flag, int moduli_id, int polys, long double scale,
                               const int64_t *host);
  // The wire format of serialize.cu: header (parameters, shape, scale) and limbs.
  size_t serialized_size(const Data &d) const;
  void serialize(const Data &d, void *buffer, size_t capacity);
  std::unique_ptr<Data> deserialize(const void *buffer, size_t size);
  void download(const Data &d, int64_t *host);
  void download_async(const Data &d, int64_t *host);
  std::unique_ptr<Data> clone(const Data &d);
  void forget(Data *d);  // called by ~Data

  // Engine-level operations (reference semantics, see fhe_b200.h).
  std::unique_ptr<Data> multiply(const Data &a, const Data &b);
  std::unique_ptr<Data> multiply_relinearize(const Data &a, const Data &b, const Data &rk);
  std::unique_ptr<Data> multiply_relinearize_rescale(const Data &a, const Data &b, const Data &rk);
  std::unique_ptr<Data> relinearize(const Data &ct, const Data &rk);
  std::unique_ptr<Data> rescale(const Data &ct);
  std::unique_ptr<Data> to_ntt(const Data &text);
  std::unique_ptr<Data> to_intt(const Data &text);
  std::unique_ptr<Data> level_down(const Data &text, int level);
  // Ciphertext rotation by one fixed rotation key (engine_rotate.cpp:52-74) and by
  // a set of power-of-two keys selected by the bits of `delta` (:106-139).
  std::unique_ptr<Data> rotate(const Data &ct, const Data &fixed_rotation_key);
  std::unique_ptr<Data> rotate(const Data &ct, const std::vector<const Data *> &keys, int delta,
                               bool normalize_by_slot_count = true);
  // Hoisted rotations of one ciphertext by several fixed keys (rotate_batch with fixed
  // rotation keys, engine_rotate.cpp:262-300): one decomposition for all keys.
  std::vector<std::unique_ptr<Data>> rotate_batch(const Data &ct,
                                                  const std::vector<const Data *> &keys);
  // Plaintext rotation and conjugation (no key): engine_rotate.cpp:10-24.
  std::unique_ptr<Data> rotate_plain(const Data &pt, int delta);
  std::unique_ptr<Data> conjugate_plain(const Data &pt);
  std::unique_ptr<Data> conjugate(const Data &ct, const Data &conjugation_key);
  // CKKSCore::switch_key (core.cpp:1058-1083): coefficient-form input.
  std::unique_ptr<Data> switch_key(const Data &ct, const Data &key_switching_key);
  int normalized_delta(int delta, bool normalize_by_slot_count = true) const;  // engine.h:370
  // CKKSCore::encode (core_encode.cpp:33-150) of up to slot_count values (im null:
  // real input) at `level`; CKKSCore::decode / decode_complex_plaintext
  // (core_decode.cpp) into host arrays of slot_count doubles.
  std::unique_ptr<Data> encode(const double *re, const double *im, int count, int level,
                               bool include_special = false);
  void decode(const Data &pt, double *re, double *im);

  // Randomness and keys (core_key.cpp, core.cpp:35-200).  seed: 8 words and a
  // 2-byte nonce (null: from the system random device), block counter reset.
  void seed(const uint32_t *seed_words, const uint8_t *nonce);
  unsigned long long random_counter() const { return rng_counter_; }
  std::unique_ptr<Data> create_secret_key(int level);
  std::unique_ptr<Data> create_secret_key(const int64_t *secret, int count, int level);
  std::unique_ptr<Data> create_sparse_secret_key(int hamming_weight, int level);
  std::unique_ptr<Data> create_public_key(const Data &sk, int level);
  std::unique_ptr<Data> create_relinearization_key(const Data &sk, int level);
  std::unique_ptr<Data> create_fixed_rotation_key(const Data &sk, int delta, int level);
  std::vector<std::unique_ptr<Data>> create_rotation_keys(const Data &sk, int level);
  std::unique_ptr<Data> create_conjugation_key(const Data &sk, int level);
  std::unique_ptr<Data> encrypt(const Data &pt, const Data &key);  // public or secret key
  std::unique_ptr<Data> decrypt(const Data &ct, const Data &sk);

  // Ciphertext arithmetic (engine_add.cpp, engine_subtract.cpp, engine_multiply.cpp,
  // engine_negate.cpp): operands are brought to a common level, rescale state and
  // form first (match_form / prepare_for_multiply), then the core operation.
  std::unique_ptr<Data> add(const Data &a, const Data &b);
  std::unique_ptr<Data> subtract(const Data &a, const Data &b);
  std::unique_ptr<Data> add_plain(const Data &ct, const Data &pt);
  std::unique_ptr<Data> subtract_plain(const Data &ct, const Data &pt);
  std::unique_ptr<Data> subtract_from_plain(const Data &pt, const Data &ct);
  std::unique_ptr<Data> add_scalar(const Data &ct, double value);
  std::unique_ptr<Data> subtract_scalar(const Data &ct, double value);
  std::unique_ptr<Data> multiply_plain(const Data &ct, const Data &pt);
  std::unique_ptr<Data> multiply_scalar(const Data &ct, double value);
  std::unique_ptr<Data> multiply_integer(const Data &ct, int64_t value);
  std::unique_ptr<Data> negate(const Data &ct);
  std::unique_ptr<Data> square(const Data &ct, const Data *rk);

  // Bootstrapping with a rotation key (engine_bootstrap.cpp:712-754) and its parts.
  std::pair<std::unique_ptr<Data>, std::unique_ptr<Data>> create_small_bootstrap_key(const Data &sk);
  std::unique_ptr<Data> bootstrap(const Data &ct, const Data &rk, const Data &ck,
                                  const std::vector<const Data *> &rotation_keys,
                                  const Data &to_sparse, const Data &to_dense, int stage_count);
  std::unique_ptr<Data> mod_raise(const Data &ct, const Data &to_sparse, const Data &to_dense);
  std::unique_ptr<Data> multiply_imaginary(const Data &ct, int64_t value);
  std::unique_ptr<Data> weighted_sum(const std::vector<const Data *> &basis,
                                     const std::vector<double> &weights);
  std::vector<std::unique_ptr<Data>> rotate_batch(const Data &ct,
                                                  const std::vector<const Data *> &keys,
                                                  const std::vector<int> &deltas);
  void add_inplace(Data &a, const Data &b);

  // Bootstrapping with a bootstrap key (engine_bootstrap.cpp:804-838): hoisted
  // baby-step giant-step transforms in the special-prime-extended NTT domain.
  std::unique_ptr<BootstrapKey> create_bootstrap_key(const Data &sk, int stage_count,
                                                     const std::string &size);
  std::unique_ptr<Data> bootstrap(const Data &ct, const Data &rk, const Data &ck,
                                  const BootstrapKey &bk);
  // After one direct run of an input shape, bootstrap(ct, rk, ck, bootstrap key) is
  // captured once as a CUDA graph and replayed (one launch instead of ~10^4); on by
  // default, off while profiling.  Same words either way.
  void set_graphs(bool on) { graphs_ = on; }
  // The inner loop of a bootstrap key's linear transforms as one fused kernel (on by
  // default) or as the per-rotation key products, gathers and diagonal sums; same
  // words either way.
  void set_fused_bsgs(bool on) { fused_bsgs_ = on; }
  // Multiply-then-relinearize transforms its inputs and the tensor value-only except
  // the limbs whose words relinearization reads exactly (ExactLimbs); on by default,
  // off for every limb exact.  Same words either way.
  void set_value_transforms(bool on) { value_transforms_ = on; }
  // Runs a batch of independent multiply-relinearize-rescale operations, each followed
  // by a rotation with its own fixed key (the batched serving step; no reference
  // counterpart), replayed as one CUDA graph after its first run.
  std::vector<std::unique_ptr<Data>> multiply_rotate_batch(
      const std::vector<const Data *> &a, const std::vector<const Data *> &b, const Data &rk,
      const std::vector<const Data *> &rotation_keys);
  // The independent operations of a batch run on up to this many streams at once
  // (1 to kMaxConcurrency; default 4; 1 runs them in order on the engine's stream).
  // Each operation's kernels stay in order on its stream, so the words are the same;
  // the streams fill the SMs left idle by one operation's last wave of CTAs.
  static constexpr int kMaxConcurrency = 8;
  void set_concurrency(int streams);
  int concurrency() const { return concurrency_; }
  // multiply_relinearize_rescale of every pair (a[i], b[i]), concurrently.
  std::vector<std::unique_ptr<Data>> multiply_relinearize_rescale_batch(
      const std::vector<const Data *> &a, const std::vector<const Data *> &b, const Data &rk);
  // bootstrap(ct, rk, ck, bk) of every ciphertext, concurrently.
  std::vector<std::unique_ptr<Data>> bootstrap_batch(const std::vector<const Data *> &cts,
                                                     const Data &rk, const Data &ck,
                                                     const BootstrapKey &bk);
  // Captured graphs held, and input shapes whose capture failed (run directly).
  std::pair<int, int> graph_counts() const {
    return {static_cast<int>(graph_cache_.size()), static_cast<int>(graph_failed_.size())};
  }
  // CKKSEngine::rotate(UnitCiphertext*, BootstrapKey*, delta, normalize)
  // (engine_rotate.cpp:192-206).
  std::unique_ptr<Data> rotate(const Data &ct, const BootstrapKey &bk, int delta,
                               bool normalize_by_slot_count = true);
  // CKKSCore::decompose (core_key_switch.cpp:434-466): every partition's ModUp of
  // polynomial 1 of a coefficient-form text.
  std::unique_ptr<Data> decompose(const Data &ct);
  // CKKSEngine::ntt_rotate (engine_rotate.cpp:223-259) on an extended NTT-form text.
  std::unique_ptr<Data> ntt_rotate(const Data &ct, const Data &decomposed, const BootstrapKey &bk,
                                   int delta);
  // CKKSCore::attach_special_prime_chains / remove_special_prime_chains
  // (core.cpp:1127-1195).
  std::unique_ptr<Data> attach_special_primes(const Data &text);
  std::unique_ptr<Data> remove_special_primes(const Data &text);

  void ntt_limbs(int64_t *limbs, int moduli_id, int chains, int polys, long long stride,
                 bool inverse);
  // SingleProcessor::mont_mult (single.h:27) on device limbs: y = REDC(a b) per word,
  // `polys` x `chains` limbs at moduli_id, [poly][chain][N] with the given stride.
  void mont_mult_limbs(const int64_t *a, const int64_t *b, int64_t *y, int moduli_id, int chains,
                       int polys, long long stride);

  // Per-kernel-family device time, measured with CUDA events on the engine's
  // stream around each launch while profiling is on.
  void set_profiling(bool on);
  std::string profile_report();  // "name launches total_ms" lines; synchronizes
  void profile_reset();

  // Where the ModDown base conversion runs; every mode gives the same words.
  //   kTensorCoresOff: CUDA cores; kTensorCoresOn: the INT8 tensor pipe wherever the
  //   shape allows it; kTensorCoresAuto (default): each conversion on the tensor pipe
  //   from the number of special primes where it measured faster (ModDown and ModUp
  //   from 4: the tensor form's cost per output is mostly fixed, the CUDA-core form's
  //   grows with K).
  enum TensorCoreMode : int { kTensorCoresOff = 0, kTensorCoresOn = 1, kTensorCoresAuto = 2 };
  static constexpr int kTensorCoreMinSpecial = 4;
  static constexpr int kTensorCoreModUpMinSpecial = 4;
  void set_tensor_cores(int mode);
  int tensor_cores() const { return tensor_cores_; }
  // Diagnostics: how many times the tensor-core kernels poll for each MMA round
  // before they give up, set the error flag that synchronize() reports, drain their
  // MMAs and return (0: give up at once; negative: the default).  Applies to
  // kernels launched afterwards.
  void set_tensor_core_wait_limit(long long limit);

  const PrimeTables &tables() const { return tables_; }
  const KeySwitchTables &key_switch_tables() const { return ks_; }
  const DevicePartitions &partitions(int moduli_id, int key_moduli_id);

 private:
  cudaStream_t own_stream_ = nullptr;
  cudaStream_t stream_ = nullptr;
  // Host uploads and downloads run on streams of their own (one per direction),
  // ordered against the compute stream by events, so the copies of one ciphertext
  // overlap the kernels of its neighbours.
  cudaStream_t upload_stream_ = nullptr;
  cudaStream_t download_stream_ = nullptr;
  cudaEvent_t upload_done_ = nullptr;
  cudaEvent_t compute_done_ = nullptr;
  void order_download_after_compute();  // the download stream waits for the compute so far
  void order_compute_after_upload();    // the compute stream waits for the uploads so far
  std::vector<int64_t *> table_buffers_;
  PrimeTables tables_{};
  KeySwitchTables ks_{};
  std::map<std::pair<int, int>, DevicePartitions> partition_cache_;
  int tensor_cores_ = kTensorCoresAuto;
  uint64_t serial_ = 0;
  // CUDA graphs of multi-kernel operations (graphs.cu): key = the operation, the
  // serial numbers of its constant operands, the kernel-form switches, the shapes of
  // its inputs and the stream.
  struct GraphShape {
    int type, flag, moduli_id, polys;
    long double scale;
  };
  struct CapturedGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<std::unique_ptr<Data>> in, out;  // the graph reads `in`, writes `out`
    unsigned long long launches = 0;
  };
  bool graphs_ = true;
  bool fused_bsgs_ = true;
  bool value_transforms_ = true;
  // Streams of batch items (graphs.cu): item i of a batch runs on worker i % count,
  // forked from and joined back into the engine's stream by events.
  int concurrency_ = 4;
  std::vector<cudaStream_t> workers_;
  std::vector<cudaEvent_t> worker_done_;
  cudaEvent_t fork_ = nullptr;
  void run_concurrent(int count, const std::function<void(int)> &item);
  std::map<std::vector<uint64_t>, std::vector<GraphShape>> graph_seen_;
  std::map<std::vector<uint64_t>, CapturedGraph> graph_cache_;
  std::set<std::vector<uint64_t>> graph_failed_;
  using GraphBody =
      std::function<std::vector<std::unique_ptr<Data>>(const std::vector<const Data *> &)>;
  // Runs `body` on `inputs` directly the first time its key is seen (checking the
  // inputs and filling every table a capture must not build), captures it once as
  // a CUDA graph over private copies of the inputs the second time, and replays the
  // graph from then on.  A capture that fails leaves the key on the direct path.
  std::vector<std::unique_ptr<Data>> run_captured(std::vector<uint64_t> key,
                                                  const std::vector<const Data *> &inputs,
                                                  const GraphBody &body);
  std::unique_ptr<Data> bootstrap_direct(const Data &ct, const Data &rk, const Data &ck,
                                         const BootstrapKey &bk);
  std::map<int, ModDownTcTables> mod_down_tc_cache_;  // moduli id -> tables
  std::map<int, ModUpTcTables> mod_up_tc_cache_;      // moduli id -> tables
  const ModUpTcTables *mod_up_tc(int moduli_id);
  bool use_tensor_cores(int min_special) const;
  // ModUp of every partition's digits into NTT-form extended limbs, in the selected form.
  cudaError_t mod_up(const DevicePartitions &dp, int moduli_id, const int64_t *digits,
                     int64_t *ext, bool skip_own = false);
  int *device_error_ = nullptr;  // set by a kernel whose bounded wait ran out
  uint32_t tc_wait_limit_ = kTcDefaultWaitLimit;
  TcNttTables tc_ntt_{};  // set when the ring degree has a tensor-core NTT
  // The value-only transforms run on the tensor pipe only when the tensor cores are
  // forced on: the CUDA-core form measured faster (see ntt_tc.cu), so AUTO keeps it.
  bool use_tc_ntt() const { return tc_ntt_.bmat != nullptr && tensor_cores_ == kTensorCoresOn; }
  // ModDown's inverse transform of `polys` extended polynomials at moduli_id, in
  // place, reduced to [0, q): on the tensor pipe when the tensor cores are in use and
  // the ring degree has a tensor-core NTT, else on the CUDA cores (same words).
  cudaError_t mod_down_transform(int moduli_id, int extended, int64_t *acc, int polys);
  TcStatus tc_status() const {
    TcStatus st;
    st.error = device_error_;
    st.wait_limit = tc_wait_limit_;
    return st;
  }
  const ModDownTcTables *mod_down_tc(int moduli_id);
  // The ModDown epilogue in the selected form.
  cudaError_t mod_down_epilogue(int moduli_id, int limbs, const int64_t *acc,
                                const EpilogueOps &ops, int64_t *out);
  RngState rng_{};
  unsigned long long rng_counter_ = 0;
  bool cdt_uploaded_ = false;
  void ensure_rng_tables();
  void draw_uniform(int64_t *out, long long row_stride, int rows, int prime_base, uint64_t fixed_max,
                    int64_t shift);
  void draw_gaussian(int64_t *out);
  void tile(const int64_t *chain, int limbs, int prime_base, int64_t *y, long long y_stride);
  // constants: host array of `limbs` per-limb values (or null), passed by value;
  // limb j runs modulo prime prime_base + j % period (period 0: limbs).
  void pointwise(int op, int limbs, int prime_base, const int64_t *a, const int64_t *b,
                 const int64_t *constants, int64_t *y, int period = 0);
  void ntt_in_place(int64_t *x, int limbs, int prime_base, long long stride, int polys);
  void intt_in_place(int64_t *x, int limbs, int prime_base, long long stride, int polys);
  std::unique_ptr<Data> create_key_switching_key(const Data &from, const Data &to, int level,
                                                 int type);
  std::unique_ptr<Data> rotated_secret_key(const Data &sk, int ntt_delta);
  std::unique_ptr<Data> rescale_any(const Data &text);  // CKKSEngine::rescale_
  void signed_tile(const int64_t *chain, int64_t q_src, int limbs, int prime_base, int64_t *y,
                   long long y_stride);
  std::unique_ptr<Data> apply_butterfly(const Data &ct, bool to_slot, int stage_count, int stage,
                                        const std::vector<const Data *> &keys, int rotate_count);
  // Host twiddles per (direction, stage count) and device diagonals prepared for the
  // product (rescaled, NTT form) per (direction, stage count, stage, outer, inner, level).
  std::map<std::pair<bool, int>, std::vector<std::vector<std::vector<std::complex<double>>>>>
      twiddle_cache_;
  std::map<std::tuple<bool, int, int, int, int, int>, std::unique_ptr<Data>> diagonal_cache_;
  const std::vector<std::vector<std::vector<std::complex<double>>>> &bootstrap_twiddles(
      bool to_slot, int stage_count);
  std::pair<std::unique_ptr<Data>, std::unique_ptr<Data>> coeff_to_slot(
      const Data &ct, const Data &conjugation_key, const std::vector<const Data *> &keys,
      int stage_count);
  std::unique_ptr<Data> slot_to_coeff(const Data &real_part, const Data &imaginary_part,
                                      const std::vector<const Data *> &keys, int stage_count);
  std::unique_ptr<Data> chebyshev_ps(const std::vector<const Data *> &baby, const Data &giant,
                                     const Data *rk,
                                     const std::vector<std::vector<double>> &coefficients);
  std::unique_ptr<Data> sine(const Data &ct, const Data &rk);
  std::unique_ptr<Data> round_to_integer(const Data &ct, const Data &rk);
  std::unique_ptr<Data> make_signed_tile(const Data &ct);
  void make_bootstrap_stage(BootstrapStage &stage,
                            const std::vector<std::vector<std::complex<double>>> &twiddles,
                            int rotate_count, int level, int inner_loop_shift);
  void require_bootstrap_stage_count(const std::string &fn, int stage_count,
                                     int inner_loop_shift) const;
  std::unique_ptr<Data> mod_down_then_decompose(Data &ct);  // clobbers polynomial 1
  std::unique_ptr<Data> remove_special_primes_in_place(Data &text);  // clobbers text
  std::unique_ptr<Data> core_ntt_rotate(const Data &ct, const Data &decomposed, const Data &key,
                                        int delta);
  std::unique_ptr<Data> apply_butterfly(const Data &ct, const BootstrapKey &bk,
                                        const BootstrapStage &stage);
  // Every outer group's sum of the stage's inner loop (bsgs.cu), in process order;
  // empty when the stage falls outside the fused kernel's limits.
  std::vector<std::unique_ptr<Data>> bsgs_inner_sums(const Data &x, const Data &decomposed,
                                                     const BootstrapKey &bk,
                                                     const BootstrapStage &stage);
  // ModUp of every partition of one coefficient-form polynomial (L limbs at
  // moduli_id) into `out` ([partitions][L+K][N]).
  void decompose_into(const int64_t *x, int moduli_id, int64_t *out);
  // ModDown (core_key_switch.cpp:110-160) of `polys` NTT-form extended polynomials
  // (clobbered) into coefficient-form polynomials of L limbs.
  void mod_down_polys(int64_t *extended, int moduli_id, int polys, int64_t *out);
  struct Matched;
  Matched match_texts(const Data &a, const Data &b, bool b_is_plain);
  std::vector<int64_t> add_multiplier(double value, int level) const;
  std::vector<int64_t> mult_multiplier(double value, int level) const;

  std::map<int, int32_t *> signed_perm_cache_;  // delta -> signed permutation [N]
  std::map<int, int32_t *> ntt_perm_cache_;     // delta -> NTT-form gather indices [N]
  const int32_t *device_signed_permutation(int delta);
  const int32_t *device_ntt_permutation(int delta);
  std::set<Data *> live_;

  struct PendingTiming {
    const char *name;
    cudaEvent_t start;
    cudaEvent_t stop;
  };
  bool profiling_ = false;
  std::vector<PendingTiming> pending_;
  std::vector<cudaEvent_t> event_pool_;
  std::map<std::string, std::pair<uint64_t, double>> stats_;
  cudaEvent_t take_event();
  void collect_timings();
  template <class F>
  cudaError_t timed(const char *name, F &&launch) {
    const NvtxRange range(name);
    if (!profiling_) return launch();
    PendingTiming p{name, take_event(), take_event()};
    cudaEventRecord(p.start, stream_);
    const cudaError_t e = launch();
    cudaEventRecord(p.stop, stream_);
    pending_.push_back(p);
    return e;
  }

  void check(cudaError_t e, const char *what);
  // Copies a host table to the device on the engine's stream and waits for it.  A
  // plain cudaMemcpy is not enough: from pageable memory it may return before the
  // DMA lands, and it runs on the legacy stream, which a non-blocking stream does
  // not wait for.  Waiting also makes the table visible to every other stream.
  void upload_bytes(void *dst, const void *src, size_t bytes, const char *what);
  // Device copy of a host table, freed with the engine.
  template <class T>
  T *upload_table(const std::vector<T> &v) {
    const size_t bytes = (v.empty() ? 1 : v.size()) * sizeof(T);
    void *p = nullptr;
    check(cudaMalloc(&p, bytes), "cudaMalloc(table)");
    table_buffers_.push_back(static_cast<int64_t *>(p));
    if (!v.empty()) upload_bytes(p, v.data(), v.size() * sizeof(T), "upload table");
    return static_cast<T *>(p);
  }

  // Codec tables on the device (built on first encode/decode).
  struct DeviceCodec {
    int codec = 0;
    int log_codec = 0;
    const int32_t *pre = nullptr;
    const int32_t *post = nullptr;
    const double2 *fft = nullptr;    // (cos, sin) of the forward twiddles
    const double2 *ifft = nullptr;
    const double2 *twist = nullptr;  // apply_twister factors
    const double2 *skew = nullptr;   // apply_skewer factors
  };
  DeviceCodec codec_;
  const DeviceCodec &codec();
  void fft_on_device(double2 *y, const double2 *twiddle, int log_codec);

  // Core steps.
  std::unique_ptr<Data> core_rescale(const Data &ct);          // coefficient form
  // With rk, the product is relinearized with rk: the prepared text's words then
  // only matter where relinearize_exact_limbs says so.
  std::unique_ptr<Data> prepare_for_multiply(const Data &text, int level,
                                             const Data *rk = nullptr);
  // to_ntt(core_rescale(text)); limbs outside `exact` value-only.
  std::unique_ptr<Data> rescale_to_ntt(const Data &text,
                                       const ExactLimbs &exact = ExactLimbs{ExactLimbs::kAllExact, 0});
  std::unique_ptr<Data> relinearized_product(const Data &pa, const Data &pb, const Data &rk);
  // The limbs of polynomial `poly` of a product at moduli_id that relinearization
  // with rk reads word for word (ExactLimbs), or every limb exact when the switch is
  // off or the bound that makes the others value-only does not hold.
  ExactLimbs relinearize_exact_limbs(int moduli_id, const Data &rk, int poly);
  // Hybrid key switch of the coefficient-form polynomial c1 at moduli_id (L limbs):
  // decompose, ModUp, key product, optional rotation term b * P (rotate_c0 = the
  // coefficient-form c0), ModDown and the epilogue operations `ops` into `out`.
  // own_ext: a caller-owned extended buffer [count][E][N] whose partitions' own limbs
  // already hold NTT-form words of c1 (see own_limbs_ext); ModUp then skips them.
  void key_switch_pipeline(const int64_t *c1, int moduli_id, const Data &key,
                           const int64_t *rotate_c0, const EpilogueOps &ops, int64_t *out,
                           const int64_t *decomposed = nullptr, int64_t *own_ext = nullptr,
                           const TensorAddend *addend = nullptr);
  // Key switch tail shared by relinearize variants; t3 is [3][L][N] coefficient
  // form at moduli_id (poly 2 is switched), or with an addend the switched polynomial
  // alone, the first two entering through the key inner product (TensorAddend).
  void relinearize_tail(const int64_t *t3, int moduli_id, const Data &rk, int mode, int64_t *out,
                        int64_t *own_ext = nullptr, const TensorAddend *addend = nullptr);
  // Whether a product at moduli_id relinearized with rk folds its first two tensor
  // polynomials into the key inner product (value transforms on, at most 8
  // partitions, every prime below 2^60 and none of them special).
  bool fold_tensor(int moduli_id, const Data &rk);
  TensorAddend tensor_addend(const Data &pa, const Data &pb) const;
  // ModUp's extended limbs of a partition's own primes are the input limbs' values,
  // so when the input's NTT form exists their NTT needs no work: an extended buffer
  // for relinearizing at moduli_id with rk, to be filled with those NTT-form words,
  // or null when ModUp's transform runs on the tensor pipe (which covers every limb).
  int64_t *own_limbs_ext(int moduli_id, const Data &rk);
  void require_key_level(const std::string &fn, const Data &text, const Data &key,
                         bool for_multiply, const char *key_name = "relinearization key");
  std::unique_ptr<Data> core_level_down(const Data &text, int level);  // coefficient form
  std::unique_ptr<Data> level_down_any(const Data &text, int level);   // level_down_ (any form)
  std::unique_ptr<Data> core_rotate(const Data &ct, const Data &key,
                                    const Data *decomposed = nullptr);   // coefficient form
};

// Thread-local last error of the C ABI.
void set_last_error(const std::string &message);

}  // namespace fhe_b200
