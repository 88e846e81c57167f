// Device kernels of rotation, conjugation and level_down: the b * P term that
// rotation adds in the NTT domain, signed coefficient permutations, NTT-form
// gathers and per-limb Montgomery scalars (contracts in kernels.cuh).
#include "kernels.cuh"
#include "ntt.cuh"

namespace fhe_b200 {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(long long work) {
  long long b = (work + kThreads - 1) / kThreads;
  if (b > (1LL << 30)) b = 1LL << 30;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

// mont_enter(mont_enter(c0, P mod q * R), R^2) on the way into the forward NTT
// (create_key_switcher_for_rotate, core_key_switch.cpp:550-576).
struct ScaledEnterLoad {
  const int64_t *src;
  const int64_t *p_product_mult_r;  // indexed by prime
  const int64_t *r_squared;
  const uint64_t *q;
  const uint64_t *k;
  __device__ __forceinline__ int64_t operator()(int, int limb, int prime, int gi, int n) const {
    const uint64_t qq = q[prime], kk = k[prime];
    const int64_t x = src[static_cast<long long>(limb) * n + gi];
    return mont_mult_lazy(mont_mult_lazy(x, p_product_mult_r[prime], qq, kk), r_squared[prime], qq, kk);
  }
};

// dst = reduce_2q_to_q(reduce(dst + v, 2q)) (mont_add_reduce_2q_to_q on the
// accumulator of the key product).
struct AccumulateStore {
  int64_t *dst;
  const uint64_t *q;
  __device__ __forceinline__ void operator()(int, int limb, int prime, int gi, int n, int64_t v) const {
    const int64_t qs = static_cast<int64_t>(q[prime]);
    int64_t *p = dst + static_cast<long long>(limb) * n + gi;
    *p = guard(guard(*p + v, qs << 1), qs);
  }
};

// One thread per word of polys x limbs x N; grid-stride.
__global__ void permute_signed_kernel(PrimeTables t, int log_n, int polys, int limbs,
                                      int prime_base, const int64_t *x, long long xs,
                                      const int32_t *perm, int64_t *y, long long ys) {
  const long long per_poly = static_cast<long long>(limbs) << log_n;
  const long long total = per_poly * polys;
  const int n = 1 << log_n;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int poly = static_cast<int>(i / per_poly);
    const long long r = i - poly * per_poly;
    const int j = static_cast<int>(r >> log_n);
    const int c = static_cast<int>(r & (n - 1));
    const int64_t qs = static_cast<int64_t>(t.q[prime_base + j]);
    const int32_t pc = perm[c];
    int64_t v = x[poly * xs + r];
    if (pc < 0) v = -v;
    v = v < 0 ? v + qs : guard(v, qs);  // make_unsigned_reduce_2q_to_q
    y[poly * ys + (static_cast<long long>(j) << log_n) + (pc < 0 ? ~pc : pc)] = v;
  }
}

__global__ void permute_gather_kernel(int log_n, int polys, int limbs, const int64_t *x,
                                      long long xs, const int32_t *perm, int64_t *y, long long ys) {
  const long long per_poly = static_cast<long long>(limbs) << log_n;
  const long long total = per_poly * polys;
  const int n = 1 << log_n;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int poly = static_cast<int>(i / per_poly);
    const long long r = i - poly * per_poly;
    const long long row = r & ~static_cast<long long>(n - 1);
    y[poly * ys + r] = x[poly * xs + row + perm[r & (n - 1)]];
  }
}

__global__ void scalar_enter_kernel(PrimeTables t, int log_n, int polys, int limbs, int prime_base,
                                    const int64_t *x, long long xs, int x_limb_offset,
                                    LimbScalars s, int64_t *y, long long ys) {
  const long long per_poly = static_cast<long long>(limbs) << log_n;
  const long long total = per_poly * polys;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int poly = static_cast<int>(i / per_poly);
    const long long r = i - poly * per_poly;
    const int j = static_cast<int>(r >> log_n);
    const int prime = prime_base + j;
    const uint64_t q = t.q[prime], k = t.k[prime];
    const int64_t v = x[poly * xs + (static_cast<long long>(x_limb_offset) << log_n) + r];
    y[poly * ys + r] = guard(mont_mult_lazy(v, s.v[j], q, k), static_cast<int64_t>(q));
  }
}

__global__ void ntt_rotate_finish_kernel(PrimeTables t, int log_n, int limbs, int prime_base,
                                         const int64_t *x0, const int64_t *acc,
                                         const int32_t *perm, int64_t *y) {
  const long long per_poly = static_cast<long long>(limbs) << log_n;
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= 2 * per_poly) return;
  const int poly = i >= per_poly ? 1 : 0;
  const long long r = i - poly * per_poly;
  const int j = static_cast<int>(r >> log_n);
  const long long src = (static_cast<long long>(j) << log_n) + perm[r & ((1LL << log_n) - 1)];
  int64_t v = acc[poly * per_poly + src];
  if (poly == 0) v = guard(x0[src] + v, static_cast<int64_t>(t.q[prime_base + j] << 1));
  y[i] = v;
}

// W consecutive words per thread (W = 2: 16-byte accesses, every pointer and stride
// 16-byte aligned), the terms' loads issued four at a time ahead of their products,
// so the diagonal streams keep enough loads in flight.
template <int W>
__global__ void diagonal_mac_kernel(PrimeTables t, int log_n, int limbs, int prime_base,
                                    MacTerms terms, long long x_stride, bool accumulate,
                                    int64_t *y, long long y_stride) {
  const long long per_poly = static_cast<long long>(limbs) << log_n;
  const long long i = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) * W;
  if (i >= 2 * per_poly) return;
  const int poly = i >= per_poly ? 1 : 0;  // W <= N: the words share a polynomial and limb
  const long long r = i - poly * per_poly;
  const int prime = prime_base + static_cast<int>(r >> log_n);
  const uint64_t q = t.q[prime], k = t.k[prime];
  const int64_t qs = static_cast<int64_t>(q), q2 = qs << 1;
  auto load = [&](const int64_t *p, int64_t (&v)[W]) {
    if (W == 2) {
      const longlong2 x = *reinterpret_cast<const longlong2 *>(p);
      v[0] = x.x;
      v[1 % W] = x.y;
    } else {
      v[0] = *p;
    }
  };
  int first = 0;
  int64_t acc[W];
  if (accumulate) {
    load(y + poly * y_stride + r, acc);
  } else {
    int64_t x[W], d[W];
    load(terms.x[0] + poly * x_stride + r, x);
    load(terms.d[0] + r, d);
#pragma unroll
    for (int w = 0; w < W; w++) acc[w] = mont_mult_lazy(x[w], d[w], q, k);
    first = 1;
  }
  constexpr int kAhead = 4;
  for (int m0 = first; m0 < terms.count; m0 += kAhead) {
    int64_t x[kAhead][W], d[kAhead][W];
#pragma unroll
    for (int u = 0; u < kAhead; u++) {
      if (m0 + u < terms.count) {
        load(terms.x[m0 + u] + poly * x_stride + r, x[u]);
        load(terms.d[m0 + u] + r, d[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < kAhead; u++) {
      if (m0 + u < terms.count) {
#pragma unroll
        for (int w = 0; w < W; w++)
          acc[w] = guard(guard(acc[w] + mont_mult_lazy(x[u][w], d[u][w], q, k), q2), qs);
      }
    }
  }
  if (W == 2) {
    *reinterpret_cast<longlong2 *>(y + poly * y_stride + r) = make_longlong2(acc[0], acc[1 % W]);
  } else {
    y[poly * y_stride + r] = acc[0];
  }
}

}  // namespace

cudaError_t launch_rotate_base(const PrimeTables &t, const KeySwitchTables &ks, int log_n,
                               int moduli_id, int limbs, const int64_t *c0, int64_t *work,
                               int64_t *acc0, cudaStream_t s) {
  ScaledEnterLoad ld{c0, ks.p_product_mult_r, t.r_squared, t.q, t.k};
  AccumulateStore st{acc0, t.q};
  // Value-only: the accumulated key product reaches the output through ModDown.
  return forward_ntt<ScaledEnterLoad, AccumulateStore, kNttValueOnly>(
      log_n, 1, limbs, moduli_id, t, ld, st, work, static_cast<long long>(limbs) << log_n, s);
}

cudaError_t launch_permute_signed(const PrimeTables &t, int n, int polys, int limbs,
                                  int prime_base, const int64_t *x, long long x_stride,
                                  const int32_t *signed_perm, int64_t *y, long long y_stride,
                                  cudaStream_t s) {
  if (x == y) return cudaErrorInvalidValue;  // a scatter cannot run in place
  const int log_n = __builtin_ctz(static_cast<unsigned>(n));
  note_launch();
  permute_signed_kernel<<<grid_for(static_cast<long long>(polys) * limbs * n), kThreads, 0, s>>>(
      t, log_n, polys, limbs, prime_base, x, x_stride, signed_perm, y, y_stride);
  return cudaGetLastError();
}

cudaError_t launch_permute_gather(int n, int polys, int limbs, const int64_t *x,
                                  long long x_stride, const int32_t *perm, int64_t *y,
                                  long long y_stride, cudaStream_t s) {
  if (x == y) return cudaErrorInvalidValue;
  const int log_n = __builtin_ctz(static_cast<unsigned>(n));
  note_launch();
  permute_gather_kernel<<<grid_for(static_cast<long long>(polys) * limbs * n), kThreads, 0, s>>>(
      log_n, polys, limbs, x, x_stride, perm, y, y_stride);
  return cudaGetLastError();
}

cudaError_t launch_scalar_enter(const PrimeTables &t, int n, int polys, int limbs,
                                int prime_base, const int64_t *x, long long x_stride,
                                int x_limb_offset, const LimbScalars &s, int64_t *y,
                                long long y_stride, cudaStream_t st) {
  if (limbs > kMaxScalarLimbs) return cudaErrorInvalidValue;
  const int log_n = __builtin_ctz(static_cast<unsigned>(n));
  note_launch();
  scalar_enter_kernel<<<grid_for(static_cast<long long>(polys) * limbs * n), kThreads, 0, st>>>(
      t, log_n, polys, limbs, prime_base, x, x_stride, x_limb_offset, s, y, y_stride);
  return cudaGetLastError();
}

cudaError_t launch_ntt_rotate_finish(const PrimeTables &t, int log_n, int limbs, int prime_base,
                                     const int64_t *x0, const int64_t *acc, const int32_t *perm,
                                     int64_t *y, cudaStream_t s) {
  note_launch();
  ntt_rotate_finish_kernel<<<grid_for((2LL * limbs) << log_n), kThreads, 0, s>>>(
      t, log_n, limbs, prime_base, x0, acc, perm, y);
  return cudaGetLastError();
}

cudaError_t launch_diagonal_mac(const PrimeTables &t, int log_n, int limbs, int prime_base,
                                const MacTerms &terms, long long x_stride, bool accumulate,
                                int64_t *y, long long y_stride, cudaStream_t s) {
  if (terms.count < 1 || terms.count > kMaxMacTerms) return cudaErrorInvalidValue;
  uintptr_t bits = reinterpret_cast<uintptr_t>(y) | static_cast<uintptr_t>(x_stride * 8) |
                   static_cast<uintptr_t>(y_stride * 8);
  for (int m = 0; m < terms.count; m++)
    bits |= reinterpret_cast<uintptr_t>(terms.x[m]) | reinterpret_cast<uintptr_t>(terms.d[m]);
  note_launch();
  if ((bits & 15) == 0 && log_n >= 1)
    diagonal_mac_kernel<2><<<grid_for(((2LL * limbs) << log_n) / 2), kThreads, 0, s>>>(
        t, log_n, limbs, prime_base, terms, x_stride, accumulate, y, y_stride);
  else
    diagonal_mac_kernel<1><<<grid_for((2LL * limbs) << log_n), kThreads, 0, s>>>(
        t, log_n, limbs, prime_base, terms, x_stride, accumulate, y, y_stride);
  return cudaGetLastError();
}

}  // namespace fhe_b200
