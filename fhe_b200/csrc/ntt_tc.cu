// Tensor-core NTT for the transforms whose result only matters modulo q
// (tcgen05.mma kind::i8 on sm_100a; N = 2^16).
//
// ModUp's forward transform of the extended limbs and ModDown's inverse transform
// feed only value-only consumers (the key inner product reduces its sum, ModDown's
// epilogue reduces every word), so any exact evaluation of the reference's
// transform (operation/ntt.cpp:46-134 forward, 177-272 inverse) modulo q gives the
// reference's final words.  Values: the forward transform puts
//   X[p] = sum_i x_i psi^((2 br(p) + 1) i)
// at position p (br = 16-bit reversal), the inverse computes
//   x_i = sum_k X[br(k)] psi^(-(2k+1) i) (times N^-1 R^-1, the reference's
// enter-exit), with psi the prime's primitive 2N-th root.
//
// Four-step split, N = 256 x 256 (i = i1 + 256 i2, k = k2 + 256 k1):
//   forward pass 1 (per column i1): y[k2] = sum_i2 x psi^(256 (2k2+1) i2), a
//     negacyclic 256-point transform, then the twist psi^((2k2+1) i1);
//   forward pass 2 (per row k2): X[k2 + 256 k1] = sum_i1 z w^(k1 i1), w = psi^512;
//   the inverse mirrors them (pass 1 cyclic per row, twist psi^-((2k2+1) i1), pass 2
//   negacyclic per column).
// Each 256-point transform is 16 x 16: step A contracts 16 inputs (m = a + 16 b,
// over b) into 16 outputs c, a twist T(a, c) follows, step B contracts over a into
// outputs d (o = c + 16 d).  A step is one MMA for 128 rows (8 lines x 16): A holds
// the 8 little-endian bytes of each input (K = 16 x 8 bytes), B (per prime and
// matrix, built on the host) the 8 bytes of M[in][out] 2^(8 byte) R mod q (N = 16
// outputs x 8 byte columns), so the exact partial sums D_b (each below 2^23) fold into
// X == R sum_in v M (mod q), X < 2^80, and one REDC leaves the value below q + 2^18.
// The twists are Montgomery products with psi powers from a natural-order table.
// Each pass reads and writes the same 2048 words of its 8 lines, so it runs in place.
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "modarith.cuh"
#include "params.hpp"
#include "umma.cuh"

namespace fhe_b200 {

namespace {

using namespace umma;
using u128 = unsigned __int128;

constexpr int kLogN = 16;
constexpr int kN = 1 << kLogN;
constexpr int kLines = 8;                      // 256-point lines per CTA
constexpr int kTile = kLines * 256;            // words per CTA
constexpr int kMatrixBytes = kTcColumns * 128; // one byte-split 16 x 16 matrix
constexpr int kMatrices = 4;                   // per prime
enum Matrix { kNeg = 0, kCyc = 1, kCycInv = 2, kNegInvScaled = 3 };
enum Kind { kForward1 = 0, kForward2 = 1, kInverse1 = 2, kInverse2 = 3 };

__device__ __forceinline__ int reverse8(int v) { return static_cast<int>(__brev(v) >> 24); }

// psi^e * R mod q for any e (Montgomery form), from psi^e R for e < N.
__device__ __forceinline__ uint64_t psi_power(const int64_t *table, long long e, uint64_t q) {
  e &= 2 * kN - 1;
  if (e < kN) return static_cast<uint64_t>(__ldg(table + e));
  const uint64_t t = static_cast<uint64_t>(__ldg(table + (e - kN)));
  return t == 0 ? 0 : q - t;
}

// Shared memory: A of step A, A of step B, B of step A, B of step B (16 KB each), the
// step twists T(a, c) of the current prime (256 words).
constexpr size_t kSmemBytes = 4 * static_cast<size_t>(kMatrixBytes) + 256 * sizeof(int64_t);
constexpr int kPerThread = kTile / kTcThreads;  // tile words each thread loads and stores

// Where input word r (r < 8) of thread `tid` comes from: its line, its index m in the
// line's 256-point transform, and its offset in the limb.
template <int KIND>
__device__ __forceinline__ void tile_input(int tid, int r, int line0, int &line, int &m,
                                           int &addr) {
  const int idx = tid + r * kTcThreads;
  if (KIND == kForward1) {  // columns i1: x[i2 * 256 + i1], m = i2
    line = idx & 7;
    m = idx >> 3;
    addr = m * 256 + line0 + line;
  } else if (KIND == kInverse2) {  // columns i1: w[pb * 256 + i1], m = k2 = br(pb)
    line = idx & 7;
    const int pb = idx >> 3;
    m = reverse8(pb);
    addr = pb * 256 + line0 + line;
  } else {  // rows: z[P * 256 + j]; forward m = i1 = j, inverse m = k1 = br(j)
    line = idx >> 8;
    const int j = idx & 255;
    m = KIND == kInverse1 ? reverse8(j) : j;
    addr = (line0 + line) * 256 + j;
  }
}

// Each CTA transforms a run of consecutive tiles (8 lines of one limb each); the
// next tile's words are loaded into registers while the current one is on the
// tensor pipe, and the matrices and step twists are loaded once per prime.
constexpr int kCtasPerSm = 3;  // 66 KB of shared memory and at most 85 registers each

template <int KIND>
__global__ void __launch_bounds__(kTcThreads, kCtasPerSm)
    tc_ntt_kernel(TcNttTables tt, PrimeTables t, int64_t *data, long long poly_stride, int polys,
                  int limbs, int prime_base, int tiles_per_cta, TcStatus status) {
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t *sA = smem;
  uint8_t *sA2 = smem + kMatrixBytes;
  uint8_t *sBA = smem + 2 * kMatrixBytes;
  uint8_t *sBB = smem + 3 * kMatrixBytes;
  uint64_t *twist = reinterpret_cast<uint64_t *>(smem + 4 * kMatrixBytes);  // [a * 16 + c]
  int64_t *stage = reinterpret_cast<int64_t *>(sA);  // step B's results (sA is free by then)
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;

  const int total = polys * limbs * (256 / kLines);
  const int first = blockIdx.x * tiles_per_cta;
  const int last = min(total, first + tiles_per_cta);
  if (first >= last) return;  // uniform per CTA, before any barrier
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tmem_alloc(&tmem_base);
  if (tid == 0) mbar_init(&mbar);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t bar = smem_addr(&mbar);
  const int lane_base = (warp & 3) * 32;
  const int row = lane_base + lane;
  const int half = warp >> 2;
  bool ok = true;
  uint32_t phase = 0;
  int loaded_prime = -1;

  // Tile index: 32 tiles per limb, then poly, then limb (as the limbs' layout).
  auto limb_of = [&](int tile, int &line0, int &prime) -> int64_t * {
    const int pl = tile >> 5;
    const int poly = pl % polys, limb = pl / polys;
    line0 = (tile & 31) * kLines;
    prime = prime_base + limb;
    return data + poly * poly_stride + static_cast<long long>(limb) * kN;
  };
  int64_t next[kPerThread];
  {
    int line0, prime;
    const int64_t *x = limb_of(first, line0, prime);
#pragma unroll
    for (int r = 0; r < kPerThread; r++) {
      int line, m, addr;
      tile_input<KIND>(tid, r, line0, line, m, addr);
      next[r] = x[addr];
    }
  }

  for (int tile = first; tile < last; tile++) {
    int line0, prime;
    int64_t *x = limb_of(tile, line0, prime);
    const uint64_t q = t.q[prime], kq = t.k[prime];
    const int64_t *pw = tt.psi_pow + static_cast<long long>(prime) * kN;
    if (prime != loaded_prime) {  // uniform: every thread walks the same tiles
      constexpr int ma = KIND == kForward1 ? kNeg : (KIND == kForward2 ? kCyc : kCycInv);
      constexpr int mb = KIND == kForward1 ? kCyc
                                           : (KIND == kForward2 ? kCyc : (KIND == kInverse1 ? kCycInv : kNegInvScaled));
      const uint4 *src = reinterpret_cast<const uint4 *>(tt.bmat + (static_cast<size_t>(prime) * kMatrices) * kMatrixBytes);
      uint4 *da = reinterpret_cast<uint4 *>(sBA), *db = reinterpret_cast<uint4 *>(sBB);
      constexpr int chunks = kMatrixBytes / 16;
      for (int i = tid; i < chunks; i += kTcThreads) {
        da[i] = src[ma * chunks + i];
        db[i] = src[mb * chunks + i];
      }
      {
        const int a = tid >> 4, c = tid & 15;
        long long e;
        if (KIND == kForward1) e = 256LL * (2 * c + 1) * a;
        else if (KIND == kForward2) e = 512LL * c * a;
        else if (KIND == kInverse1) e = -512LL * c * a;
        else e = -256LL * (2 * a + 1) * c;
        twist[tid] = psi_power(pw, e, q);
      }
      loaded_prime = prime;
    }
    // The tile's words into A: input m = a + 16 b of line `line` goes to row
    // a * 8 + line, bytes b * 8 (a word is read unsigned; only its value mod q matters).
#pragma unroll
    for (int r = 0; r < kPerThread; r++) {
      int line, m, addr;
      tile_input<KIND>(tid, r, line0, line, m, addr);
      int64_t v = next[r];
      if (v < 0) {
        v %= static_cast<int64_t>(q);
        if (v < 0) v += static_cast<int64_t>(q);
      }
      *reinterpret_cast<uint64_t *>(sA + core_offset((m & 15) * kLines + line, (m >> 4) * 8, kTcCoeffs)) =
          static_cast<uint64_t>(v);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // Step A: D[(a, line)][(c, byte)] = sum over b and bytes.
    if (tid == 0) {
      mma_round(tmem, sA, sBA, 128);
      mma_commit(bar);
    }
    if (tile + 1 < last) {  // the next tile's words, in flight during this tile
      int nline0, nprime;
      const int64_t *nx = limb_of(tile + 1, nline0, nprime);
#pragma unroll
      for (int r = 0; r < kPerThread; r++) {
        int line, m, addr;
        tile_input<KIND>(tid, r, nline0, line, m, addr);
        next[r] = nx[addr];
      }
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, status.wait_limit)) != 0;
    if (!ok) break;
    phase ^= 1;
    tc_fence_after();
    {
      const int a = row >> 3, line = row & 7;
      for (int cp = half * 8; cp < half * 8 + 8; cp += 2) {
        uint32_t d[16];
        tmem_load16(tmem + (static_cast<uint32_t>(lane_base) << 16) + cp * 8, d);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int c = cp + h;
          uint64_t lo, hi;
          fold8(d + 8 * h, lo, hi);
          const uint64_t u = static_cast<uint64_t>(redc_wide(lo, hi, q, kq));  // < q + 2^18
          const uint64_t v = static_cast<uint64_t>(mont_mult_small(u, twist[a * 16 + c], q, kq));
          *reinterpret_cast<uint64_t *>(sA2 + core_offset(c * kLines + line, a * 8, kTcCoeffs)) = v;
        }
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // Step B: D[(c, line)][(d, byte)] = sum over a and bytes.
    if (tid == 0) {
      mma_round(tmem, sA2, sBB, 128);
      mma_commit(bar);
    }
    const int c = row >> 3, line = row & 7;
    const int L = line0 + line;
    uint64_t pass_twist[8];
    if (KIND == kForward1 || KIND == kInverse1) {  // loaded while the MMAs run
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int o = c + 16 * (half * 8 + i);
        pass_twist[i] = KIND == kForward1 ? psi_power(pw, (2LL * o + 1) * L, q)
                                          : psi_power(pw, -(2LL * reverse8(L) + 1) * o, q);
      }
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, status.wait_limit)) != 0;
    if (!ok) break;
    phase ^= 1;
    tc_fence_after();
    for (int dp = half * 8; dp < half * 8 + 8; dp += 2) {
      uint32_t dd[16];
      tmem_load16(tmem + (static_cast<uint32_t>(lane_base) << 16) + dp * 8, dd);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int o = c + 16 * (dp + h);
        uint64_t lo, hi;
        fold8(dd + 8 * h, lo, hi);
        uint64_t w = static_cast<uint64_t>(redc_wide(lo, hi, q, kq));  // < q + 2^18
        int s;
        if (KIND == kForward1) {  // y[k2] psi^((2 k2 + 1) i1) -> row br(k2), column i1
          w = static_cast<uint64_t>(mont_mult_small(w, pass_twist[dp + h - half * 8], q, kq));
          s = reverse8(o) * kLines + line;
        } else if (KIND == kForward2) {  // X[k2 + 256 k1] at P * 256 + br(k1)
          s = line * 256 + reverse8(o);
        } else if (KIND == kInverse1) {  // w[i1] psi^-((2 k2 + 1) i1), k2 = br(P)
          w = static_cast<uint64_t>(mont_mult_small(w, pass_twist[dp + h - half * 8], q, kq));
          s = line * 256 + o;
        } else {  // x[i1 + 256 i2], scaled by N^-1 R^-1 in the matrix; canonical
          w = w >= q ? w - q : w;
          s = o * kLines + line;
        }
        stage[s] = static_cast<int64_t>(w);
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // Coalesced stores of the staged results.
#pragma unroll
    for (int r = 0; r < kPerThread; r++) {
      const int idx = tid + r * kTcThreads;
      int addr;
      if (KIND == kForward1 || KIND == kInverse2) {  // [row][8 columns]
        addr = (idx >> 3) * 256 + line0 + (idx & 7);
      } else {  // [8 rows][256]
        addr = (line0 + (idx >> 8)) * 256 + (idx & 255);
      }
      x[addr] = stage[idx];
    }
    __syncthreads();  // the stage (sA) is read before the next tile's words land there
  }
  if (!ok) {
    // The MMAs of the step that timed out may still run: wait for them (bounded)
    // before the tensor memory is given back.
    if (tid == 0) atomicExch(status.error, 1);
    if (warp == 0) mbar_wait(bar, phase);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem);
}

uint64_t mul_mod(uint64_t a, uint64_t b, uint64_t m) {
  return static_cast<uint64_t>(static_cast<u128>(a) * b % m);
}

uint64_t pow_mod(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  b %= m;
  for (; e; e >>= 1, b = mul_mod(b, b, m))
    if (e & 1) r = mul_mod(r, b, m);
  return r;
}

template <int KIND>
cudaError_t launch_pass(const TcNttTables &tt, const PrimeTables &t, int polys, int limbs,
                        int prime_base, int64_t *data, long long poly_stride,
                        const TcStatus &status, cudaStream_t s) {
  static int raised = 0;
  static int ctas = 0;  // resident CTAs of the whole GPU
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  const int bit = 1 << (device & 31);
  if (!(raised & bit)) {
    e = cudaFuncSetAttribute(tc_ntt_kernel<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kSmemBytes));
    // Three CTAs of 66 KB share an SM only with the largest shared-memory carveout.
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(tc_ntt_kernel<KIND>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    ctas = sms * kCtasPerSm;
    raised |= bit;
  }
  const int total = polys * limbs * (256 / kLines);
  const int per_cta = (total + ctas - 1) / ctas;
  const int grid = (total + per_cta - 1) / per_cta;
  note_launch();
  tc_ntt_kernel<KIND><<<grid, kTcThreads, kSmemBytes, s>>>(tt, t, data, poly_stride, polys, limbs,
                                                          prime_base, per_cta, status);
  return cudaGetLastError();
}

}  // namespace

bool tc_ntt_supported(int log_n) { return log_n == kLogN; }

TcNttHost make_tc_ntt_tables(const Parameters &p) {
  TcNttHost h;
  if (!tc_ntt_supported(p.log_n)) return h;
  const int P = p.prime_count;
  const uint64_t R = uint64_t(1) << 62;
  h.psi_pow.resize(static_cast<size_t>(P) * kN);
  h.bmat.assign(static_cast<size_t>(P) * kMatrices * kMatrixBytes, 0);
  for (int i = 0; i < P; i++) {
    const uint64_t q = p.q[i];
    const uint64_t psi = static_cast<uint64_t>(p.psi[i]) % q;
    const uint64_t r = R % q;
    int64_t *pw = &h.psi_pow[static_cast<size_t>(i) * kN];
    uint64_t v = r;  // psi^e R
    for (int e = 0; e < kN; e++) {
      pw[e] = static_cast<int64_t>(v);
      v = mul_mod(v, psi, q);
    }
    const uint64_t psi_inv = pow_mod(psi, q - 2, q);
    // N^-1 R^-1: the enter-exit scaling of the inverse transform.
    const uint64_t scale = mul_mod(pow_mod(kN % q, q - 2, q), pow_mod(r, q - 2, q), q);
    for (int mtx = 0; mtx < kMatrices; mtx++) {
      uint8_t *b = &h.bmat[(static_cast<size_t>(i) * kMatrices + mtx) * kMatrixBytes];
      for (int in = 0; in < 16; in++)
        for (int out = 0; out < 16; out++) {
          uint64_t m;
          if (mtx == kNeg) m = pow_mod(psi, 4096ULL * (2 * out + 1) * in, q);
          else if (mtx == kCyc) m = pow_mod(psi, 8192ULL * in * out, q);
          else if (mtx == kCycInv) m = pow_mod(psi_inv, 8192ULL * in * out, q);
          else m = mul_mod(pow_mod(psi_inv, 4096ULL * out * (2 * in + 1), q), scale, q);
          uint64_t e = mul_mod(m, r, q);  // M 2^(8 byte) R for byte = 0, 1, ...
          for (int byte = 0; byte < 8; byte++) {
            for (int bb = 0; bb < 8; bb++)
              b[core_offset(out * 8 + bb, in * 8 + byte, kTcColumns)] = static_cast<uint8_t>(e >> (8 * bb));
            e = static_cast<uint64_t>((static_cast<u128>(e) << 8) % q);
          }
        }
    }
  }
  return h;
}

cudaError_t launch_tc_ntt(const TcNttTables &tt, const PrimeTables &t, bool inverse, int polys,
                          int limbs, int prime_base, int64_t *data, long long poly_stride,
                          const TcStatus &status, cudaStream_t s) {
  if (tt.bmat == nullptr || tt.psi_pow == nullptr || status.error == nullptr || polys < 1 ||
      limbs < 1 || t.log_n != kLogN)
    return cudaErrorInvalidValue;
  cudaError_t e;
  if (!inverse) {
    e = launch_pass<kForward1>(tt, t, polys, limbs, prime_base, data, poly_stride, status, s);
    if (e == cudaSuccess)
      e = launch_pass<kForward2>(tt, t, polys, limbs, prime_base, data, poly_stride, status, s);
  } else {
    e = launch_pass<kInverse1>(tt, t, polys, limbs, prime_base, data, poly_stride, status, s);
    if (e == cudaSuccess)
      e = launch_pass<kInverse2>(tt, t, polys, limbs, prime_base, data, poly_stride, status, s);
  }
  return e;
}

}  // namespace fhe_b200
