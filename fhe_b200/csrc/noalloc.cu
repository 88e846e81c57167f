// Relinearization that allocates nothing per call.
//
// Some callers of this library cannot allocate device memory while they work:
// code running inside a CUDA graph capture, real-time pipelines with a fixed
// memory budget, or hosts whose allocator policy forbids cudaMalloc after
// start-up.  For them, fhe_relinearize_noalloc runs the same key-switching kernels
// as fhe_relinearize but takes its temporaries (the iNTT'd ciphertext, the
// mixed-radix digits, the extended partitions, the key-product accumulators and the
// partition constants) from one file-scope device array of kNoAllocScratchWords
// words instead of the stream-ordered pool.  Inputs and outputs are caller-owned
// device buffers.
//
// Set-up: the first call on each device resolves the device address of the array
// with cudaGetSymbolAddress while that device is current; that first call should
// therefore come before any stream capture.  Every later call on the device reuses
// the address.  All calls share the one array and it keeps the last call's
// contents; everything a call reads is written by the same call first.  Calls that
// overlap on the GPU (different streams, or different host threads on one device)
// race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/fhe_b200.h"
#include "engine.hpp"

struct fhe_engine {
  fhe_b200::Engine *impl;
};

namespace fhe_b200 {
namespace {

// 4 Mi words = 32 MiB of scratch, held by every GPU that loads the library.
constexpr size_t kNoAllocScratchWords = size_t(1) << 22;
// Partition constants staged on the host: dnum <= 64 partitions.
constexpr int kMaxPartitions = 64;
constexpr size_t kConstantWords = 1 << 17;

__device__ __align__(256) int64_t g_noalloc_scratch[kNoAllocScratchWords];

constexpr int kMaxDevices = 64;
int64_t *g_scratch_address[kMaxDevices] = {};
std::mutex g_setup_mutex;
int64_t g_host_constants[kConstantWords];  // host staging, no heap

int64_t *scratch_address() {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
    throw std::runtime_error("no usable CUDA device for the no-alloc scratch.");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_address[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      throw std::runtime_error(std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                               cudaGetErrorString(e));
    }
    g_scratch_address[device] = static_cast<int64_t *>(p);
  }
  return g_scratch_address[device];
}

// Partition constants of (moduli_id, key_moduli_id) written into the host staging
// buffer in the DevicePartitions layout (ints, then inverse_r, product_r,
// product_r_squared), following ckks/parameters.cpp:334-360 and
// ckks/precomputed.cpp:326-382 without any heap allocation.
size_t stage_partitions(const Parameters &p, int moduli_id, int key_moduli_id,
                        DevicePartitions &dp, int starts[], int sizes[], int indices[]) {
  const int K = p.special_prime_count;
  const int L = p.chains(moduli_id);
  const int E = p.chains(moduli_id, true);
  const int pc = p.partition_count(moduli_id);
  if (pc > kMaxPartitions) throw std::invalid_argument("too many partitions for the no-alloc path.");
  int index = p.partition_count(key_moduli_id) - pc;
  int count = 0;
  for (int start = L - pc * K; start < L; start += K, index++) {
    const int lo = start > 0 ? start : 0;
    const int hi = start + K < L ? start + K : L;
    if (index < 0) throw std::invalid_argument("the key was created at a lower level than the text.");
    if (hi - lo > 16) throw std::invalid_argument("partition larger than 16 limbs.");
    starts[count] = lo;
    sizes[count] = hi - lo;
    indices[count] = index;
    count++;
  }
  const size_t int_words = (3 * static_cast<size_t>(count) * sizeof(int) + 7) / 8;
  const size_t words = int_words + static_cast<size_t>(count) * (16 + 256 + 16 * static_cast<size_t>(E));
  if (words > kConstantWords) throw std::invalid_argument("partition constants exceed the no-alloc staging.");
  std::memset(g_host_constants, 0, words * sizeof(int64_t));
  int *ints = reinterpret_cast<int *>(g_host_constants);
  int64_t *inv = g_host_constants + int_words;
  int64_t *prod = inv + static_cast<size_t>(count) * 16;
  int64_t *prod2 = prod + static_cast<size_t>(count) * 256;
  const uint64_t *qq = p.q.data() + moduli_id;
  const int64_t *r2 = p.r_squared.data() + moduli_id;
  constexpr int64_t kR = int64_t(1) << 62;
  dp.count = count;
  dp.extended = E;
  dp.max_size = 0;
  dp.size_mask = 0;
  dp.max_key_index = 0;
  for (int part = 0; part < count; part++) {
    const int st = starts[part], sz = sizes[part];
    ints[part] = st;
    ints[count + part] = sz;
    ints[2 * count + part] = indices[part];
    dp.max_size = dp.max_size > sz ? dp.max_size : sz;
    dp.size_mask |= 1u << sz;
    dp.max_key_index = dp.max_key_index > indices[part] ? dp.max_key_index : indices[part];
    auto product_mod = [&](int cnt, int64_t m) {
      int64_t acc = 1;
      for (int z = 0; z < cnt; z++)
        acc = mod_mul(acc, static_cast<int64_t>(qq[st + z] % static_cast<uint64_t>(m)), m);
      return acc;
    };
    for (int ci = 1; ci < sz; ci++) {
      const int64_t chain_q = static_cast<int64_t>(qq[st + ci]);
      const int64_t inverse = mod_invert(product_mod(ci, chain_q), chain_q);
      inv[part * 16 + ci - 1] = (chain_q & 1) == 0 ? inverse : mod_mul(inverse, kR, chain_q);
      for (int mi = ci + 1; mi < sz; mi++) {
        const int64_t mq = static_cast<int64_t>(qq[st + mi]);
        const int64_t v = product_mod(ci, mq);
        prod[(part * 16 + ci - 1) * 16 + (mi - ci - 1)] = (mq & 1) == 0 ? v : mod_mul(v, kR, mq);
      }
      for (int mi = 0; mi < E; mi++) {
        const int64_t mq = static_cast<int64_t>(qq[mi]);
        const int64_t v = product_mod(ci, mq);
        prod2[(static_cast<size_t>(part) * 16 + ci - 1) * E + mi] =
            (mq & 1) == 0 ? v : mod_mul(v, r2[mi], mq);
      }
    }
  }
  return words;
}

}  // namespace
}  // namespace fhe_b200

extern "C" int fhe_relinearize_noalloc(fhe_engine *engine, const int64_t *ct_device, int moduli_id,
                                       const int64_t *key_device, int key_moduli_id, int key_polys,
                                       int64_t *out_device) {
  using namespace fhe_b200;
  if (!engine || !engine->impl) {
    set_last_error("null handle: engine");
    return FHE_ERR_NULL_HANDLE;
  }
  if (!ct_device || !key_device || !out_device) {
    set_last_error("Relinearize Without Allocation: a device buffer pointer is null.");
    return FHE_ERR_NULL_HANDLE;
  }
  try {
    Engine &e = *engine->impl;
    const Parameters &p = e.params;
    // Messages are only built on the error paths, so the working path touches no heap.
    static const char fn[] = "Relinearize Without Allocation";
    if (moduli_id < 0 || moduli_id >= p.chain_count - 1 || key_moduli_id < 0 ||
        key_moduli_id > moduli_id)
      throw std::invalid_argument(std::string(fn) +
                                  ": the moduli ids of the text and key are not compatible.");
    const int n = p.n;
    const int L = p.chains(moduli_id);
    const int E = p.chains(moduli_id, true);
    int starts[kMaxPartitions], sizes[kMaxPartitions], indices[kMaxPartitions];
    DevicePartitions dp;
    // The host staging buffer is shared: stage and copy under the lock (a copy from
    // pageable memory returns once the buffer may be reused).
    std::unique_lock<std::mutex> staging(g_setup_mutex, std::defer_lock);
    int64_t *scratch = scratch_address();
    staging.lock();
    const size_t const_words = stage_partitions(p, moduli_id, key_moduli_id, dp, starts, sizes, indices);
    if (key_polys < 2 * (dp.max_key_index + 1))
      throw std::invalid_argument(std::string(fn) + ": the key switching key has too few polynomials.");
    const size_t const_region = (const_words + 31) & ~size_t(31);  // keep 256-byte alignment
    const size_t t3_words = static_cast<size_t>(3) * L * n;
    const size_t digit_words = static_cast<size_t>(L) * n;
    const size_t ext_words = static_cast<size_t>(dp.count) * E * n;
    const size_t acc_words = static_cast<size_t>(2) * E * n;
    const size_t need = const_region + t3_words + digit_words + ext_words + acc_words;
    if (need > kNoAllocScratchWords)
      throw std::invalid_argument(std::string(fn) + ": needs " + std::to_string(need) +
                                  " scratch words, more than the fixed " +
                                  std::to_string(kNoAllocScratchWords) + " (N x limbs too large).");
    cudaStream_t s = e.stream();
    cudaError_t rc = cudaMemcpyAsync(scratch, g_host_constants, const_words * sizeof(int64_t),
                                     cudaMemcpyHostToDevice, s);
    staging.unlock();
    const size_t int_words = (3 * static_cast<size_t>(dp.count) * sizeof(int) + 7) / 8;
    int *dints = reinterpret_cast<int *>(scratch);
    dp.start = dints;
    dp.size = dints + dp.count;
    dp.key_index = dints + 2 * dp.count;
    dp.inverse_r = scratch + int_words;
    dp.product_r = dp.inverse_r + static_cast<size_t>(dp.count) * 16;
    dp.product_r_squared = dp.product_r + static_cast<size_t>(dp.count) * 256;
    int64_t *t3 = scratch + const_region;
    int64_t *digits = t3 + t3_words;
    int64_t *ext = digits + digit_words;
    int64_t *acc = ext + ext_words;
    const PrimeTables &t = e.tables();
    const long long ps = static_cast<long long>(L) * n;
    if (rc == cudaSuccess) rc = launch_to_intt(t, p.log_n, 3, L, moduli_id, ct_device, ps, t3, ps, s);
    if (rc == cudaSuccess) rc = launch_mixed_radix(t, dp, n, moduli_id, t3 + 2 * ps, digits, s);
    if (rc == cudaSuccess) rc = launch_mod_up_ntt(t, dp, p.log_n, moduli_id, digits, ext, s);
    if (rc == cudaSuccess)
      rc = launch_key_inner_product(t, dp, n, moduli_id, ext, key_device, p.chains(key_moduli_id, true),
                                    moduli_id - key_moduli_id, acc, s);
    if (rc == cudaSuccess) rc = launch_mod_down_intt(t, p.log_n, moduli_id, E, acc, s);
    if (rc == cudaSuccess)
      rc = launch_mod_down_epilogue(t, e.key_switch_tables(), n, moduli_id, L, acc, t3, 1, out_device, s);
    if (rc != cudaSuccess) {
      cudaGetLastError();
      throw CudaError(std::string("relinearize (no-alloc): ") + cudaGetErrorString(rc));
    }
    set_last_error("");
    return FHE_OK;
  } catch (const std::invalid_argument &ex) {
    set_last_error(ex.what());
    return FHE_ERR_INVALID_ARGUMENT;
  } catch (const CudaError &ex) {
    set_last_error(ex.what());
    return FHE_ERR_CUDA;
  } catch (const std::exception &ex) {
    set_last_error(ex.what());
    return FHE_ERR_RUNTIME;
  }
}
