// Relinearization that allocates nothing per call.
//
// Some callers of this library cannot allocate device memory while they work:
// applications whose own allocator reserves the GPU's memory up front and hands
// libraries a fixed budget, real-time loops where the implicit device
// synchronisation of cudaMalloc/cudaFree (or an out-of-memory failure in mid-run)
// is not acceptable, and code running where CUDA allocation calls are not allowed,
// such as stream callbacks.  For them, fhe_relinearize_noalloc runs the same
// key-switching kernels as fhe_relinearize but takes its temporaries (the iNTT'd
// ciphertext, the mixed-radix digits, the extended partitions, the key-product
// accumulators and the partition constants) from one file-scope device array of
// kNoAllocScratchWords words instead of the stream-ordered pool.  Inputs and
// outputs are caller-owned device buffers.
//
// Set-up: the first call on each device resolves the device address of the array
// with cudaGetSymbolAddress while that device is current; that first call should
// therefore come before any stream capture.  Every later call on the device reuses
// the address.  All calls share the one array and it keeps the last call's
// contents; everything a call reads is written by the same call first (the
// partition constants are computed on the device from the call's own arguments,
// so no host buffer is read after the call returns).  Calls that overlap on the
// GPU (different streams, or different host threads on one device) race on the
// array and must be serialised by the caller.
#include <cuda_runtime.h>

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
// dnum <= 64 partitions.
constexpr int kMaxPartitions = 64;

__device__ __align__(256) int64_t g_noalloc_scratch[kNoAllocScratchWords];

constexpr int kMaxDevices = 64;
int64_t *g_scratch_address[kMaxDevices] = {};
std::mutex g_setup_mutex;

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

// The partition ranges of (moduli_id, key_moduli_id), passed to the device by value
// (ckks/parameters.cpp:334-360: partitions of K limbs counted from the top, the
// lowest one cut short; the key's partition index counts from its own top).
struct PartitionLayout {
  int count;
  int extended;
  int moduli_id;
  int start[kMaxPartitions];
  int size[kMaxPartitions];
  int key_index[kMaxPartitions];
};

// a * b mod m on the signed 128-bit product (arithmetic.cpp:33-38).
__device__ int64_t device_mod_mul(int64_t a, int64_t b, int64_t m) {
  return static_cast<int64_t>((static_cast<__int128>(a) * b) % m);
}

// Extended Euclid on signed 64-bit values; 0 when no inverse exists
// (arithmetic.cpp:9-31).
__device__ int64_t device_mod_invert(int64_t x, int64_t modulus) {
  int64_t a = x, b = modulus, ra = 1, rb = 0;
  while (b > 0) {
    const int64_t quotient = a / b;
    int64_t t = a;
    a = b;
    b = t - quotient * b;
    t = ra;
    ra = rb;
    rb = t - quotient * rb;
  }
  if (a != 1) return 0;
  return ra >= 0 ? ra : ra + modulus;
}

// Garner constants of one partition per CTA, in the DevicePartitions layout (ints,
// then inverse_r [16], product_r [16][16], product_r_squared [16][E] per partition),
// following ckks/precomputed.cpp:326-382; unused entries are written as zero.  The
// product of the partition's leading primes is carried as residues modulo each
// prime that needs it.
__global__ void noalloc_partition_constants_kernel(PartitionLayout lay, const uint64_t *q,
                                                   const int64_t *r_squared, int *ints,
                                                   int64_t *inverse_r, int64_t *product_r,
                                                   int64_t *product_r_squared) {
  constexpr int64_t kR = int64_t(1) << 62;
  const int part = blockIdx.x;
  const int E = lay.extended;
  const uint64_t *qq = q + lay.moduli_id;
  const int64_t *r2 = r_squared + lay.moduli_id;
  const int st = lay.start[part], sz = lay.size[part];
  if (threadIdx.x == 0) {
    ints[part] = st;
    ints[lay.count + part] = sz;
    ints[2 * lay.count + part] = lay.key_index[part];
  }
  auto product_mod = [&](int cnt, int64_t m) {
    int64_t acc = 1;
    for (int z = 0; z < cnt; z++)
      acc = device_mod_mul(acc, static_cast<int64_t>(qq[st + z] % static_cast<uint64_t>(m)), m);
    return acc;
  };
  const int entries = 16 + 256 + 16 * E;
  for (int idx = threadIdx.x; idx < entries; idx += blockDim.x) {
    int64_t value = 0;
    if (idx < 16) {
      const int ci = idx + 1;
      if (ci < sz) {
        const int64_t chain_q = static_cast<int64_t>(qq[st + ci]);
        const int64_t inverse = device_mod_invert(product_mod(ci, chain_q), chain_q);
        value = (chain_q & 1) == 0 ? inverse : device_mod_mul(inverse, kR, chain_q);
      }
      inverse_r[part * 16 + idx] = value;
    } else if (idx < 16 + 256) {
      const int r = idx - 16;
      const int ci = r / 16 + 1, mi = ci + 1 + r % 16;
      if (mi < sz) {
        const int64_t mq = static_cast<int64_t>(qq[st + mi]);
        const int64_t v = product_mod(ci, mq);
        value = (mq & 1) == 0 ? v : device_mod_mul(v, kR, mq);
      }
      product_r[part * 256 + r] = value;
    } else {
      const int r = idx - 16 - 256;
      const int ci = r / E + 1, mi = r % E;
      if (ci < sz) {
        const int64_t mq = static_cast<int64_t>(qq[mi]);
        const int64_t v = product_mod(ci, mq);
        value = (mq & 1) == 0 ? v : device_mod_mul(v, r2[mi], mq);
      }
      product_r_squared[static_cast<size_t>(part) * 16 * E + r] = value;
    }
  }
}

// Partition ranges of (moduli_id, key_moduli_id) and the host-side fields of
// DevicePartitions, without any heap allocation.
void plan_partitions(const Parameters &p, int moduli_id, int key_moduli_id, PartitionLayout &lay,
                     DevicePartitions &dp) {
  const int K = p.special_prime_count;
  const int L = p.chains(moduli_id);
  const int pc = p.partition_count(moduli_id);
  if (pc > kMaxPartitions) throw std::invalid_argument("too many partitions for the no-alloc path.");
  int index = p.partition_count(key_moduli_id) - pc;
  int count = 0;
  for (int start = L - pc * K; start < L; start += K, index++) {
    const int lo = start > 0 ? start : 0;
    const int hi = start + K < L ? start + K : L;
    if (index < 0) throw std::invalid_argument("the key was created at a lower level than the text.");
    if (hi - lo > 16) throw std::invalid_argument("partition larger than 16 limbs.");
    lay.start[count] = lo;
    lay.size[count] = hi - lo;
    lay.key_index[count] = index;
    count++;
  }
  lay.count = count;
  lay.extended = p.chains(moduli_id, true);
  lay.moduli_id = moduli_id;
  dp.count = count;
  dp.extended = lay.extended;
  dp.max_size = 0;
  dp.size_mask = 0;
  dp.max_key_index = 0;
  for (int part = 0; part < count; part++) {
    dp.max_size = dp.max_size > lay.size[part] ? dp.max_size : lay.size[part];
    dp.size_mask |= 1u << lay.size[part];
    dp.max_key_index = dp.max_key_index > lay.key_index[part] ? dp.max_key_index : lay.key_index[part];
    if (part < 8) dp.key_index_first[part] = lay.key_index[part];
  }
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
    PartitionLayout lay;
    DevicePartitions dp;
    plan_partitions(p, moduli_id, key_moduli_id, lay, dp);
    if (key_polys < 2 * (dp.max_key_index + 1))
      throw std::invalid_argument(std::string(fn) + ": the key switching key has too few polynomials.");
    const size_t int_words = (3 * static_cast<size_t>(dp.count) * sizeof(int) + 7) / 8;
    const size_t const_words = int_words + static_cast<size_t>(dp.count) * (16 + 256 + 16 * static_cast<size_t>(E));
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
    int64_t *scratch = scratch_address();
    cudaStream_t s = e.stream();
    int *dints = reinterpret_cast<int *>(scratch);
    dp.start = dints;
    dp.size = dints + dp.count;
    dp.key_index = dints + 2 * dp.count;
    dp.inverse_r = scratch + int_words;
    dp.product_r = dp.inverse_r + static_cast<size_t>(dp.count) * 16;
    dp.product_r_squared = dp.product_r + static_cast<size_t>(dp.count) * 256;
    const PrimeTables &t = e.tables();
    note_launch();
    noalloc_partition_constants_kernel<<<dp.count, 256, 0, s>>>(lay, t.q, t.r_squared, dints,
                                                                dp.inverse_r, dp.product_r,
                                                                dp.product_r_squared);
    cudaError_t rc = cudaGetLastError();
    int64_t *t3 = scratch + const_region;
    int64_t *digits = t3 + t3_words;
    int64_t *ext = digits + digit_words;
    int64_t *acc = ext + ext_words;
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
