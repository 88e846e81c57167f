// Canonical-embedding encode and decode on the device (DESILO FHE
// ckks/core_encode.cpp:33-150, ckks/core_decode.cpp:11-124).
//
// Floating point follows the reference operation by operation: every product,
// sum and quotient is an explicitly rounded IEEE double operation (__dmul_rn,
// __dadd_rn, ...), so no fused multiply-add changes a rounding, and the cos/sin
// factors come from host tables computed with the same expressions and libm as
// the reference's.  Complex products are (a.re b.re - a.im b.im, a.re b.im +
// a.im b.re), the expansion of the reference's std::complex<double> product.
#include <cmath>
#include <cstring>

#include "engine.hpp"

namespace fhe_b200 {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxCrtWords = 48;  // CRT integers up to 3072 bits (50 limbs of 61 bits)

inline unsigned grid_for(long long work) {
  long long b = (work + kThreads - 1) / kThreads;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

__device__ __forceinline__ int bit_reverse(int i, int log_size) {
  return log_size == 0 ? 0 : static_cast<int>(__brev(static_cast<unsigned>(i)) >> (32 - log_size));
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

// pre_permute (encode.cpp:156-185) followed by bit_reversal_permute
// (fft.cpp:56-75): value `index` lands at bitrev(pre[index]) and its mirror at
// bitrev(codec - 1 - pre[index]).
__global__ void encode_scatter_kernel(const double *re, const double *im, int slot, int log_codec,
                                      const int32_t *pre, double2 *y) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= slot) return;
  const int codec = 1 << log_codec;
  const int p = pre[index];
  const double r = re[index];
  const double i = im ? im[index] : 0.0;
  y[bit_reverse(p, log_codec)] = make_double2(r, i);
  y[bit_reverse(codec - 1 - p, log_codec)] = make_double2(r, im ? -i : 0.0);
}

// One radix-2 stage of fft (fft.cpp:77-102): step 2^s, twiddle stride codec >> s.
__global__ void fft_stage_kernel(double2 *y, const double2 *twiddle, int log_codec, int s) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (1 << (log_codec - 1))) return;
  const int half = 1 << (s - 1);
  const int j = t & (half - 1);
  const int a = ((t >> (s - 1)) << s) + j;
  const int b = a + half;
  const double2 left = y[a];
  const double2 right = cmul(twiddle[j << (log_codec - s)], y[b]);
  y[a] = make_double2(__dadd_rn(left.x, right.x), __dadd_rn(left.y, right.y));
  y[b] = make_double2(__dsub_rn(left.x, right.x), __dsub_rn(left.y, right.y));
}

// normalize (fft.cpp:47-52) and apply_twister (encode.cpp:279-290), with the
// max_absolute reduction (single.cpp:567-575) of the result.
__global__ void encode_twist_kernel(const double2 *y, int codec, const double2 *twist, double scale,
                                    double *v, unsigned long long *max_bits) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= codec) return;
  const double size = static_cast<double>(codec);
  const double re = __ddiv_rn(y[i].x, size);
  const double im = __ddiv_rn(y[i].y, size);
  const double2 c = twist[i];
  const double value = __dmul_rn(__dsub_rn(__dmul_rn(re, c.x), __dmul_rn(im, c.y)), scale);
  v[i] = value;
  atomicMax(max_bits, static_cast<unsigned long long>(__double_as_longlong(fabs(value))));
}

__device__ __forceinline__ int64_t positive_mod(int64_t x, int64_t m) { return (m + x % m) % m; }

// round_ + tile_unsigned_reduce_2q_to_q (single.cpp:555-565, 315-326), or
// double_to_rns (arithmetic.cpp:242-270) when some |coefficient| exceeds 2^59,
// then mont_enter by r_mult_scale_after_tile.  Coefficient i of the codec lands
// at i * jump (decompress_polynomial).
__global__ void encode_tile_kernel(const double *v, const unsigned long long *max_bits, PrimeTables t,
                                   int first_prime, int limbs, const int64_t *multiplier,
                                   int limb_offset, int jump, int codec, int log_n, int64_t *out) {
  const long long w = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (w >= static_cast<long long>(limbs) * codec) return;
  const int j = static_cast<int>(w / codec);
  const int i = static_cast<int>(w - static_cast<long long>(j) * codec);
  const int prime = first_prime + j;
  const int64_t q = static_cast<int64_t>(t.q[prime]);
  const double x = v[i];
  const double max_abs = __longlong_as_double(static_cast<long long>(*max_bits));
  int64_t y;
  if (max_abs > 576460752303423488.0) {       // 2^59
    if (fabs(x) < 4611686018427387904.0) {    // 2^62
      const int64_t rounded = static_cast<int64_t>(__dadd_rn(x, 0.5));
      y = positive_mod(rounded, q);
    } else {
      int exponent = 0;
      const double mantissa = frexp(__dadd_rn(x, 0.5), &exponent);
      const int64_t int_mantissa = static_cast<int64_t>(__dmul_rn(mantissa, 4503599627370496.0));
      y = positive_mod(int_mantissa, q);
      for (int e = 52; e < exponent; e++) {
        y <<= 1;
        y %= q;
      }
    }
  } else {
    // std::llround: to nearest, halves away from zero (exact for |x| <= 2^59).
    double r = trunc(x);
    if (fabs(__dsub_rn(x, r)) >= 0.5) r = __dadd_rn(r, x < 0 ? -1.0 : 1.0);
    const int64_t rounded = static_cast<int64_t>(r);
    y = rounded < 0 ? rounded + q : guard(rounded, q);
  }
  y = mont_mult(y, multiplier[j], t.q[prime], t.k[prime]);
  out[(static_cast<long long>(limb_offset + j) << log_n) + static_cast<long long>(i) * jump] = y;
}

// Constants of the CRT reconstruction (DecodeParameters, parameter/decode.cpp):
// for limb j, inverse_r[j] = (Q/q_j)^-1 * R mod q_j and Q/q_j as `words` 64-bit
// words; Q and floor(Q/2) likewise.
struct CrtConstants {
  int limbs = 0;
  int words = 0;
  const int64_t *inverse_r = nullptr;  // [limbs]
  const uint64_t *cofactor = nullptr;  // [limbs][words]
  const uint64_t *modulus = nullptr;   // [words]
  const uint64_t *half = nullptr;      // [words]
};

__device__ __forceinline__ bool words_ge(const uint64_t *a, const uint64_t *b, int words) {
  for (int w = words - 1; w >= 0; w--) {
    if (a[w] != b[w]) return a[w] > b[w];
  }
  return true;
}

// BigInt::get_double (big_int.cpp:219-225): sum of double(word) * 2^(64 w) in
// word order over the trimmed words (2^(64 w) overflows to infinity past w = 15).
__device__ __forceinline__ double words_to_double(const uint64_t *a, int words) {
  int top = words - 1;
  while (top > 0 && a[top] == 0) top--;
  double y = 0.0;
  for (int w = 0; w <= top; w++) {
    const double scale = w < 16 ? ldexp(1.0, 64 * w) : __longlong_as_double(0x7ff0000000000000LL);
    y = __dadd_rn(y, __dmul_rn(__ull2double_rn(a[w]), scale));
  }
  return y;
}

// convert_plaintext_to_double after the rescale loop (core_decode.cpp:77-98):
// make_unsigned, then the centred CRT integer as a double (rns_to_double,
// arithmetic.cpp:169-197, whose Montgomery BigInt reduction yields the canonical
// residue mod Q); one limb: make_signed (unit.cpp:36-42, unsigned comparison).
__global__ void decode_crt_kernel(const int64_t *x, PrimeTables t, int first_prime, int jump,
                                  int codec, int log_n, CrtConstants c, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= codec) return;
  const long long pos = static_cast<long long>(i) * jump;
  if (c.limbs == 1) {
    const int64_t v = x[pos];
    const uint64_t q = t.q[first_prime];
    out[i] = static_cast<double>(static_cast<uint64_t>(v) <= (q >> 1) ? v : v - static_cast<int64_t>(q));
    return;
  }
  uint64_t acc[kMaxCrtWords + 1];
  for (int w = 0; w <= c.words; w++) acc[w] = 0;
  for (int j = 0; j < c.limbs; j++) {
    const int prime = first_prime + j;
    const uint64_t qu = t.q[prime];
    const int64_t q = static_cast<int64_t>(qu);
    int64_t v = x[(static_cast<long long>(j) << log_n) + pos];
    v = v < 0 ? v + q : guard(v, q);  // make_unsigned_reduce_2q_to_q
    int64_t d = mont_mult(v, c.inverse_r[j], qu, t.k[prime]);
    if (d < 0) d += q;
    if (d >= q) d -= q;
    // acc += d * (Q / q_j)
    const uint64_t *cof = c.cofactor + static_cast<long long>(j) * c.words;
    unsigned long long carry = 0;
    for (int w = 0; w < c.words; w++) {
      const unsigned long long lo = static_cast<unsigned long long>(d) * cof[w];
      const unsigned long long hi = __umul64hi(static_cast<unsigned long long>(d), cof[w]);
      const unsigned long long s = acc[w] + lo;
      unsigned long long c1 = s < lo ? 1 : 0;
      const unsigned long long s2 = s + carry;
      c1 += s2 < s ? 1 : 0;
      acc[w] = s2;
      carry = hi + c1;
    }
    acc[c.words] += carry;
  }
  // Reduce modulo Q: the sum is below limbs * Q.
  for (int iter = 0; iter < 4 * kMaxCrtWords; iter++) {
    bool ge = acc[c.words] != 0;
    if (!ge) ge = words_ge(acc, c.modulus, c.words);
    if (!ge) break;
    unsigned long long borrow = 0;
    for (int w = 0; w < c.words; w++) {
      const unsigned long long bw = c.modulus[w];
      const unsigned long long d = acc[w] - bw - borrow;
      borrow = (acc[w] < bw || (acc[w] == bw && borrow)) ? 1 : 0;
      acc[w] = d;
    }
    acc[c.words] -= borrow;
  }
  double value;
  if (words_ge(acc, c.half, c.words)) {
    // Q - X
    unsigned long long borrow = 0;
    for (int w = 0; w < c.words; w++) {
      const unsigned long long aw = c.modulus[w], bw = acc[w];
      const unsigned long long d = aw - bw - borrow;
      borrow = (aw < bw || (aw == bw && borrow)) ? 1 : 0;
      acc[w] = d;
    }
    value = -words_to_double(acc, c.words);
  } else {
    value = words_to_double(acc, c.words);
  }
  out[i] = value;
}

// apply_skewer (encode.cpp:292-301) and bit_reversal_permute.
__global__ void decode_skew_kernel(const double *x, int log_codec, const double2 *skew, double2 *y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (1 << log_codec)) return;
  const double v = x[i];
  y[bit_reverse(i, log_codec)] = make_double2(__dmul_rn(v, skew[i].x), __dmul_rn(v, skew[i].y));
}

// permute_after_ifft (encode.cpp:481-503).
__global__ void decode_permute_kernel(const double2 *z, int codec, int slot, const int32_t *post,
                                      double scale_inverse, double *re, double *im) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= codec) return;
  const int p = post[index];
  if (p < slot) {
    re[p] = __dmul_rn(z[index].x, scale_inverse);
    if (im) im[p] = __dmul_rn(z[index].y, scale_inverse);
  }
}

inline size_t even(size_t words) { return (words + 1) & ~static_cast<size_t>(1); }

}  // namespace

// --------------------------------------------------------------- host side --

const Engine::DeviceCodec &Engine::codec() {
  if (codec_.codec) return codec_;
  const CodecTables h = params.codec_tables();
  const int c = h.codec;
  auto pairs = [&](const std::vector<double> &a, const std::vector<double> &b) {
    std::vector<double> v(2 * static_cast<size_t>(c));
    for (int i = 0; i < c; i++) {
      v[2 * i] = a[i];
      v[2 * i + 1] = b[i];
    }
    return reinterpret_cast<const double2 *>(upload_table(v));
  };
  DeviceCodec d;
  d.pre = upload_table(h.pre);
  d.post = upload_table(h.post);
  d.fft = pairs(h.fft_cos, h.fft_sin);
  d.ifft = pairs(h.ifft_cos, h.ifft_sin);
  d.twist = pairs(h.twist_cos, h.twist_sin);
  d.skew = pairs(h.skew_cos, h.skew_sin);
  while ((1 << d.log_codec) < c) d.log_codec++;
  d.codec = c;
  codec_ = d;
  return codec_;
}

void Engine::fft_on_device(double2 *y, const double2 *twiddle, int log_codec) {
  for (int s = 1; s <= log_codec; s++) {
    note_launch();
    fft_stage_kernel<<<grid_for(1LL << (log_codec - 1)), kThreads, 0, stream_>>>(y, twiddle,
                                                                                 log_codec, s);
  }
  check(cudaGetLastError(), "fft");
}

std::unique_ptr<Data> Engine::encode(const double *re, const double *im, int count, int level,
                                     bool include_special) {
  const std::string fn = im ? "Encode Complex Double Vector To Unit Plaintext"
                            : "Encode Double Vector To Unit Plaintext";
  if (level < 0 || level > params.max_level())
    throw std::runtime_error(fn + ": the target level cannot be reached with the current engine "
                                  "parameters.");
  if (count < 0 || (count > 0 && re == nullptr))
    throw std::invalid_argument(fn + ": the input values are missing.");
  const DeviceCodec &dc = codec();
  const int slot = params.slot_count;
  const int codec_n = dc.codec;
  const EncodeLevel el = params.encode_level(level);
  const int mid = params.moduli_id(level);
  int limbs = params.chains(mid, include_special);
  int limb_offset = 0;
  if (el.max_level_in_one_more_level) {
    limb_offset = 1;
    limbs -= 1;
  }
  const int flag = (im ? kFlagComplex : 0) | (include_special ? kFlagSpecial : 0);
  auto pt = make_data(kUnitPlaintext, flag, mid, 1, el.ckks_scale);

  // The slot values padded with zeros (CKKSCore::pad); surplus values are ignored.
  const int used = count < slot ? count : slot;
  std::vector<double> host(static_cast<size_t>(slot) * (im ? 2 : 1), 0.0);
  if (used > 0) {
    std::memcpy(host.data(), re, sizeof(double) * used);
    if (im) std::memcpy(host.data() + slot, im, sizeof(double) * used);
  }
  const size_t in_words = even(host.size());
  const size_t scratch_words = in_words + 2 * static_cast<size_t>(codec_n) + codec_n + 2 +
                               el.r_mult_scale_after_tile.size();
  int64_t *scratch = alloc_words(scratch_words);
  double *d_in = reinterpret_cast<double *>(scratch);
  double2 *y = reinterpret_cast<double2 *>(scratch + in_words);
  double *v = reinterpret_cast<double *>(y + codec_n);
  unsigned long long *max_bits = reinterpret_cast<unsigned long long *>(v + codec_n);
  int64_t *multiplier = reinterpret_cast<int64_t *>(max_bits + 2);
  // Pageable host sources: the copies have read them when the calls return.
  cudaError_t e = cudaMemcpyAsync(d_in, host.data(), host.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(multiplier, el.r_mult_scale_after_tile.data(),
                        el.r_mult_scale_after_tile.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                        stream_);
  if (e == cudaSuccess) e = cudaMemsetAsync(y, 0, sizeof(double2) * codec_n, stream_);
  if (e == cudaSuccess) e = cudaMemsetAsync(max_bits, 0, sizeof(unsigned long long), stream_);
  if (e == cudaSuccess) e = cudaMemsetAsync(pt->d, 0, pt->words() * sizeof(int64_t), stream_);
  if (e == cudaSuccess)
    e = timed("encode", [&] {
      note_launch();
      encode_scatter_kernel<<<grid_for(slot), kThreads, 0, stream_>>>(
          d_in, im ? d_in + slot : nullptr, slot, dc.log_codec, dc.pre, y);
      fft_on_device(y, dc.fft, dc.log_codec);
      note_launch();
      encode_twist_kernel<<<grid_for(codec_n), kThreads, 0, stream_>>>(
          y, codec_n, dc.twist, el.scale_before_tile, v, max_bits);
      note_launch();
      encode_tile_kernel<<<grid_for(static_cast<long long>(limbs) * codec_n), kThreads, 0,
                           stream_>>>(v, max_bits, tables_, el.first_moduli_id, limbs, multiplier,
                                      limb_offset, params.n / codec_n, codec_n, params.log_n,
                                      pt->d);
      return cudaGetLastError();
    });
  free_words(scratch);
  check(e, "encode");
  return pt;
}

void Engine::decode(const Data &pt, double *re, double *im) {
  const std::string fn = im ? "Decode Unit Plaintext To Complex Vector"
                            : "Decode Unit Plaintext To Double Vector";
  if (pt.is_rescaled())
    throw std::runtime_error(fn + ": the input " + std::string(pt.type_name()) +
                             " should not be rescaled.");
  if (re == nullptr) throw std::invalid_argument(fn + ": the output buffer is null.");
  if (pt.chains == 1)
    throw std::runtime_error("A plaintext needs at least two chains to be decoded.");
  const bool include_special = (pt.flag & kFlagSpecial) != 0;
  {
    long double modulus = 1;
    for (int j = 0; j < pt.chains; j++) modulus *= static_cast<long double>(params.q[pt.moduli_id + j]);
    if (pt.scale > modulus)
      throw std::invalid_argument(
          "Overflow due to large ckks_scale and small unit plaintext modulus.");
  }
  // The rescale loop of convert_plaintext_to_double (core_decode.cpp:36-54): the
  // limbs are read as coefficient form, as the reference does.
  std::unique_ptr<Data> hold;
  const Data *x = &pt;
  if (!include_special) {
    while (x->moduli_id <= params.chain_count - 2) {
      if (params.rescaled_scale(x->scale, x->moduli_id) <= params.scale) break;
      auto r = core_rescale(*x);
      hold = std::move(r);
      x = hold.get();
    }
  }
  const long double output_scale = x->scale;
  const DeviceCodec &dc = codec();
  const int codec_n = dc.codec;
  const int slot = params.slot_count;
  const int limbs = x->chains;
  const int mid = x->moduli_id;
  const int words = limbs > 1 ? (limbs * 61 + 63) / 64 + 1 : 1;
  if (words > kMaxCrtWords) throw std::invalid_argument(fn + ": too many limbs to decode.");

  // CRT constants (DecodeParameters, parameter/decode.cpp:5-60) as exact words.
  std::vector<uint64_t> modulus(words, 0), half(words, 0), cof(static_cast<size_t>(limbs) * words, 0);
  std::vector<int64_t> inverse_r(limbs, 0);
  auto mul_small = [&](uint64_t *a, uint64_t m) {
    unsigned __int128 carry = 0;
    for (int w = 0; w < words; w++) {
      const unsigned __int128 p = static_cast<unsigned __int128>(a[w]) * m + carry;
      a[w] = static_cast<uint64_t>(p);
      carry = p >> 64;
    }
  };
  if (limbs > 1) {
    modulus[0] = 1;
    for (int j = 0; j < limbs; j++) mul_small(modulus.data(), params.q[mid + j]);
    for (int w = 0; w < words; w++)
      half[w] = (modulus[w] >> 1) | (w + 1 < words ? (modulus[w + 1] << 63) : 0);
    for (int j = 0; j < limbs; j++) {
      uint64_t *c = &cof[static_cast<size_t>(j) * words];
      c[0] = 1;
      const int64_t qj = static_cast<int64_t>(params.q[mid + j]);
      int64_t inv = 1;
      for (int i = 0; i < limbs; i++) {
        if (i == j) continue;
        mul_small(c, params.q[mid + i]);
        inv = mod_mul(inv, mod_invert(static_cast<int64_t>(params.q[mid + i] % qj), qj), qj);
      }
      inverse_r[j] = mod_mul(inv, (INT64_C(1) << 62) % qj, qj);
    }
  }
  const size_t o_cof = even(limbs);
  const size_t o_mod = o_cof + cof.size();
  const size_t o_half = o_mod + words;
  const size_t o_plain = even(o_half + words);
  const size_t o_z = o_plain + codec_n;  // codec_n is even
  const size_t o_re = o_z + 2 * static_cast<size_t>(codec_n);
  int64_t *scratch = alloc_words(o_re + 2 * static_cast<size_t>(slot));
  int64_t *d_inv = scratch;
  uint64_t *d_cof = reinterpret_cast<uint64_t *>(scratch + o_cof);
  uint64_t *d_mod = reinterpret_cast<uint64_t *>(scratch + o_mod);
  uint64_t *d_half = reinterpret_cast<uint64_t *>(scratch + o_half);
  double *plain = reinterpret_cast<double *>(scratch + o_plain);
  double2 *z = reinterpret_cast<double2 *>(scratch + o_z);
  double *d_re = reinterpret_cast<double *>(scratch + o_re);
  double *d_im = d_re + slot;
  cudaError_t e = cudaMemcpyAsync(d_inv, inverse_r.data(), limbs * sizeof(int64_t),
                                  cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess && limbs > 1)
    e = cudaMemcpyAsync(d_cof, cof.data(), cof.size() * sizeof(uint64_t), cudaMemcpyHostToDevice,
                        stream_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_mod, modulus.data(), words * sizeof(uint64_t), cudaMemcpyHostToDevice,
                        stream_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_half, half.data(), words * sizeof(uint64_t), cudaMemcpyHostToDevice,
                        stream_);
  if (e == cudaSuccess)
    e = timed("decode", [&] {
      CrtConstants c;
      c.limbs = limbs;
      c.words = words;
      c.inverse_r = d_inv;
      c.cofactor = d_cof;
      c.modulus = d_mod;
      c.half = d_half;
      note_launch();
      decode_crt_kernel<<<grid_for(codec_n), kThreads, 0, stream_>>>(
          x->d, tables_, mid, params.n / codec_n, codec_n, params.log_n, c, plain);
      note_launch();
      decode_skew_kernel<<<grid_for(codec_n), kThreads, 0, stream_>>>(plain, dc.log_codec, dc.skew,
                                                                       z);
      fft_on_device(z, dc.ifft, dc.log_codec);
      const double scale_inverse = static_cast<double>(1.0 / output_scale);
      note_launch();
      decode_permute_kernel<<<grid_for(codec_n), kThreads, 0, stream_>>>(
          z, codec_n, slot, dc.post, scale_inverse, d_re, im ? d_im : nullptr);
      return cudaGetLastError();
    });
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(re, d_re, slot * sizeof(double), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess && im)
    e = cudaMemcpyAsync(im, d_im, slot * sizeof(double), cudaMemcpyDeviceToHost, stream_);
  free_words(scratch);
  check(e, "decode");
  synchronize();
}

}  // namespace fhe_b200
