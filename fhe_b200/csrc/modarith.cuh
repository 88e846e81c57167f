// Modular arithmetic of the B200 CKKS engine (device code; also compiles as host
// C++ so the exact word semantics can be checked on the CPU).
//
// Words are int64 holding residues.  As in the reference (DESILO FHE
// montgomery/unit.h:10-31, montgomery/compound.cpp) every comparison is signed and
// the REDC product is formed from sign-extended operands, so out-of-range
// intermediates evaluate to the same words as on the CPU.  R = 2^62.
//
// The 64x64 -> 128-bit products are four 32x32 -> 64-bit multiply-adds: on the
// device they are PTX chains of 32-bit multiply-adds through the carry flag (no
// 64-bit register pair per partial product, no carry recomputed by compares); the
// host form of each function computes the same integers in C++.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define FHE_HD __host__ __device__ __forceinline__
#else
#define FHE_HD inline
#endif

namespace fhe_b200 {

constexpr int kMontBits = 62;
constexpr uint64_t kMontMask = (uint64_t(1) << kMontBits) - 1;

// (x < q) ? x : x - q  (unit.h:13)
FHE_HD int64_t guard(int64_t x, int64_t q) { return x < q ? x : x - q; }

FHE_HD uint64_t mad32(uint32_t a, uint32_t b, uint64_t c) {
  return static_cast<uint64_t>(a) * b + c;
}

// Full unsigned product a * b = hi * 2^64 + lo.
FHE_HD void mul_wide(uint64_t a, uint64_t b, uint64_t &lo, uint64_t &hi) {
#ifdef __CUDA_ARCH__
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, z0, z1, z2, z3;\n\t"
      "mov.b64 {a0, a1}, %2;\n\t"
      "mov.b64 {b0, b1}, %3;\n\t"
      "mul.lo.u32 z0, a0, b0;\n\t"
      "mul.hi.u32 z1, a0, b0;\n\t"
      "mad.lo.cc.u32 z1, a0, b1, z1;\n\t"
      "madc.hi.u32 z2, a0, b1, 0;\n\t"
      "mad.lo.cc.u32 z1, a1, b0, z1;\n\t"
      "madc.hi.cc.u32 z2, a1, b0, z2;\n\t"
      "addc.u32 z3, 0, 0;\n\t"
      "mad.lo.cc.u32 z2, a1, b1, z2;\n\t"
      "madc.hi.u32 z3, a1, b1, z3;\n\t"
      "mov.b64 %0, {z0, z1};\n\t"
      "mov.b64 %1, {z2, z3};\n\t"
      "}"
      : "=l"(lo), "=l"(hi)
      : "l"(a), "l"(b));
#else
  const uint32_t a0 = static_cast<uint32_t>(a), a1 = static_cast<uint32_t>(a >> 32);
  const uint32_t b0 = static_cast<uint32_t>(b), b1 = static_cast<uint32_t>(b >> 32);
  const uint64_t t = mad32(a0, b0, 0);
  const uint64_t m = mad32(a0, b1, t >> 32);                       // < 2^64
  const uint64_t m2 = mad32(a1, b0, static_cast<uint32_t>(m));    // < 2^64
  const uint64_t h = mad32(a1, b1, m >> 32);
  hi = h + (m2 >> 32);                                             // no overflow
  lo = static_cast<uint32_t>(t) | (m2 << 32);
#endif
}

// Bits [62, 126) of X + s*q with s = (X mod 2^64) * k mod 2^62, X = hi*2^64 + lo
// (every sum modulo 2^128).
FHE_HD int64_t redc_wide(uint64_t lo, uint64_t hi, uint64_t q, uint64_t k) {
#ifdef __CUDA_ARCH__
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 z0, z1, z2, z3, q0, q1, k0, k1, s0, s1;\n\t"
      "mov.b64 {z0, z1}, %1;\n\t"
      "mov.b64 {z2, z3}, %2;\n\t"
      "mov.b64 {q0, q1}, %3;\n\t"
      "mov.b64 {k0, k1}, %4;\n\t"
      "mul.lo.u32 s0, z0, k0;\n\t"          // s = (X mod 2^64) k mod 2^62
      "mul.hi.u32 s1, z0, k0;\n\t"
      "mad.lo.u32 s1, z0, k1, s1;\n\t"
      "mad.lo.u32 s1, z1, k0, s1;\n\t"
      "and.b32 s1, s1, 0x3fffffff;\n\t"
      "mad.lo.cc.u32 z0, s0, q0, z0;\n\t"   // X += s q
      "madc.hi.cc.u32 z1, s0, q0, z1;\n\t"
      "madc.lo.cc.u32 z2, s1, q1, z2;\n\t"
      "madc.hi.u32 z3, s1, q1, z3;\n\t"
      "mad.lo.cc.u32 z1, s0, q1, z1;\n\t"
      "madc.hi.cc.u32 z2, s0, q1, z2;\n\t"
      "addc.u32 z3, z3, 0;\n\t"
      "mad.lo.cc.u32 z1, s1, q0, z1;\n\t"
      "madc.hi.cc.u32 z2, s1, q0, z2;\n\t"
      "addc.u32 z3, z3, 0;\n\t"
      "shf.r.clamp.b32 z0, z1, z2, 30;\n\t"  // bits [62, 126)
      "shf.r.clamp.b32 z1, z2, z3, 30;\n\t"
      "mov.b64 %0, {z0, z1};\n\t"
      "}"
      : "=l"(r)
      : "l"(lo), "l"(hi), "l"(q), "l"(k));
  return static_cast<int64_t>(r);
#else
  const uint64_t s = (lo * k) & kMontMask;
  uint64_t sl, sh;
  mul_wide(s, q, sl, sh);
  const uint64_t zl = lo + sl;
  const uint64_t zh = hi + sh + (zl < lo ? 1 : 0);
  return static_cast<int64_t>((zh << 2) | (zl >> kMontBits));
#endif
}

// REDC(a * b) with R = 2^62 on sign-extended operands (unit.h:15-23).  The signed
// high product is the unsigned one minus b when a < 0 and minus a when b < 0.  On
// the device the 128-bit product, its sign correction, s q and the sum run as one
// chain of 32-bit multiply-adds through the carry flag.
FHE_HD int64_t mont_mult(int64_t a, int64_t b, uint64_t q, uint64_t k) {
#ifdef __CUDA_ARCH__
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 a0, a1, b0, b1, q0, q1, k0, k1, z0, z1, z2, z3, s0, s1, c0, c1;\n\t"
      ".reg .pred na, nb;\n\t"
      "mov.b64 {a0, a1}, %1;\n\t"
      "mov.b64 {b0, b1}, %2;\n\t"
      "mov.b64 {q0, q1}, %3;\n\t"
      "mov.b64 {k0, k1}, %4;\n\t"
      "mul.lo.u32 z0, a0, b0;\n\t"          // z = a b, unsigned, 128 bits
      "mul.hi.u32 z1, a0, b0;\n\t"
      "mad.lo.cc.u32 z1, a0, b1, z1;\n\t"
      "madc.hi.u32 z2, a0, b1, 0;\n\t"
      "mad.lo.cc.u32 z1, a1, b0, z1;\n\t"
      "madc.hi.cc.u32 z2, a1, b0, z2;\n\t"
      "addc.u32 z3, 0, 0;\n\t"
      "mad.lo.cc.u32 z2, a1, b1, z2;\n\t"
      "madc.hi.u32 z3, a1, b1, z3;\n\t"
      "setp.lt.s32 na, a1, 0;\n\t"          // signed high half
      "setp.lt.s32 nb, b1, 0;\n\t"
      "selp.b32 c0, b0, 0, na;\n\t"
      "selp.b32 c1, b1, 0, na;\n\t"
      "sub.cc.u32 z2, z2, c0;\n\t"
      "subc.u32 z3, z3, c1;\n\t"
      "selp.b32 c0, a0, 0, nb;\n\t"
      "selp.b32 c1, a1, 0, nb;\n\t"
      "sub.cc.u32 z2, z2, c0;\n\t"
      "subc.u32 z3, z3, c1;\n\t"
      "mul.lo.u32 s0, z0, k0;\n\t"          // s = (z mod 2^64) k mod 2^62
      "mul.hi.u32 s1, z0, k0;\n\t"
      "mad.lo.u32 s1, z0, k1, s1;\n\t"
      "mad.lo.u32 s1, z1, k0, s1;\n\t"
      "and.b32 s1, s1, 0x3fffffff;\n\t"
      "mad.lo.cc.u32 z0, s0, q0, z0;\n\t"   // z += s q
      "madc.hi.cc.u32 z1, s0, q0, z1;\n\t"
      "madc.lo.cc.u32 z2, s1, q1, z2;\n\t"
      "madc.hi.u32 z3, s1, q1, z3;\n\t"
      "mad.lo.cc.u32 z1, s0, q1, z1;\n\t"
      "madc.hi.cc.u32 z2, s0, q1, z2;\n\t"
      "addc.u32 z3, z3, 0;\n\t"
      "mad.lo.cc.u32 z1, s1, q0, z1;\n\t"
      "madc.hi.cc.u32 z2, s1, q0, z2;\n\t"
      "addc.u32 z3, z3, 0;\n\t"
      "shf.r.clamp.b32 z0, z1, z2, 30;\n\t"  // bits [62, 126)
      "shf.r.clamp.b32 z1, z2, z3, 30;\n\t"
      "mov.b64 %0, {z0, z1};\n\t"
      "}"
      : "=l"(r)
      : "l"(a), "l"(b), "l"(q), "l"(k));
  return static_cast<int64_t>(r);
#else
  const uint64_t ua = static_cast<uint64_t>(a), ub = static_cast<uint64_t>(b);
  uint64_t lo, hi;
  mul_wide(ua, ub, lo, hi);
  hi -= (a < 0 ? ub : 0) + (b < 0 ? ua : 0);
  return redc_wide(lo, hi, q, k);
#endif
}

// mont_mult when `a` is known to be non-negative (a twiddle or table constant).
FHE_HD int64_t mont_mult_const(int64_t a, int64_t b, uint64_t q, uint64_t k) {
#ifdef __CUDA_ARCH__
  return mont_mult(a, b, q, k);  // the same word; the device form has no cheaper variant
#else
  const uint64_t ua = static_cast<uint64_t>(a), ub = static_cast<uint64_t>(b);
  uint64_t lo, hi;
  mul_wide(ua, ub, lo, hi);
  hi -= (b < 0 ? ua : 0);
  return redc_wide(lo, hi, q, k);
#endif
}

// mont_mult_const for operands known to lie in range: 0 <= w, b < 2^62 and odd
// q < 2^61, with k = -q^-1 mod 2^62.  Same word, fewer carries: with 32-bit
// halves, Z = w b + s q = c0 + c1 2^32 + c2 2^64 where
//   c0 = w0 b0 + s0 q0,  c1 = w0 b1 + w1 b0 + s0 q1 + s1 q0,  c2 = w1 b1 + s1 q1.
// Z is a multiple of 2^62, so the low words of w0 b0 and s0 q0 sum to 0 or 2^32 and
// c0 / 2^32 = hi(w0 b0) + hi(s0 q0 + lo(w0 b0)); Y = c1 + c0 / 2^32 is below 2^64
// and a multiple of 2^30, and Z / 2^62 = Y / 2^30 + 4 c2.  Every partial sum below
// stays under 2^64 for these bounds (w1, b1, s1 < 2^30; q1 < 2^29).
// On the device the same sums run as 32-bit multiply-adds chained through the
// carry flag, so no partial product needs a 64-bit register pair of its own.
FHE_HD int64_t mont_mult_small(uint64_t w, uint64_t b, uint64_t q, uint64_t k) {
#ifdef __CUDA_ARCH__
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 w0, w1, b0, b1, q0, q1, k0, k1, pl, ph, yl, yh, s0, s1, ul, uh, tl, th, wx, sx, rl, rh;\n\t"
      "mov.b64 {w0, w1}, %1;\n\t"
      "mov.b64 {b0, b1}, %2;\n\t"
      "mov.b64 {q0, q1}, %3;\n\t"
      "mov.b64 {k0, k1}, %4;\n\t"
      "mul.lo.u32 pl, w0, b0;\n\t"           // p = w0 b0
      "mul.hi.u32 ph, w0, b0;\n\t"
      "mad.lo.cc.u32 yl, w0, b1, ph;\n\t"    // y = w0 b1 + w1 b0 + p / 2^32
      "madc.hi.u32 yh, w0, b1, 0;\n\t"
      "mad.lo.cc.u32 yl, w1, b0, yl;\n\t"
      "madc.hi.u32 yh, w1, b0, yh;\n\t"
      "mul.lo.u32 s0, pl, k0;\n\t"           // s = ((yl, pl) k) mod 2^62
      "mul.hi.u32 s1, pl, k0;\n\t"
      "mad.lo.u32 s1, pl, k1, s1;\n\t"
      "mad.lo.u32 s1, yl, k0, s1;\n\t"
      "and.b32 s1, s1, 0x3fffffff;\n\t"
      "mad.lo.cc.u32 ul, s0, q0, pl;\n\t"    // u = s0 q0 + p mod 2^32
      "madc.hi.u32 uh, s0, q0, 0;\n\t"
      "mad.lo.cc.u32 yl, s1, q0, yl;\n\t"    // y += s1 q0 + s0 q1 + u / 2^32
      "madc.hi.u32 yh, s1, q0, yh;\n\t"
      "mad.lo.cc.u32 yl, s0, q1, yl;\n\t"
      "madc.hi.u32 yh, s0, q1, yh;\n\t"
      "add.cc.u32 yl, yl, uh;\n\t"
      "addc.u32 yh, yh, 0;\n\t"
      "shf.r.clamp.b32 tl, yl, yh, 30;\n\t"  // y / 2^30
      "shr.b32 th, yh, 30;\n\t"
      "shl.b32 wx, w1, 2;\n\t"
      "shl.b32 sx, s1, 2;\n\t"
      "mad.lo.cc.u32 rl, wx, b1, tl;\n\t"    // + 4 w1 b1 + 4 s1 q1
      "madc.hi.u32 rh, wx, b1, th;\n\t"
      "mad.lo.cc.u32 rl, sx, q1, rl;\n\t"
      "madc.hi.u32 rh, sx, q1, rh;\n\t"
      "mov.b64 %0, {rl, rh};\n\t"
      "}"
      : "=l"(r)
      : "l"(w), "l"(b), "l"(q), "l"(k));
  return static_cast<int64_t>(r);
#else
  const uint32_t w0 = static_cast<uint32_t>(w), w1 = static_cast<uint32_t>(w >> 32);
  const uint32_t b0 = static_cast<uint32_t>(b), b1 = static_cast<uint32_t>(b >> 32);
  const uint32_t q0 = static_cast<uint32_t>(q), q1 = static_cast<uint32_t>(q >> 32);
  const uint64_t p = mad32(w0, b0, 0);
  uint64_t y = mad32(w1, b0, mad32(w0, b1, p >> 32));
  const uint64_t lo = static_cast<uint32_t>(p) | (y << 32);  // w b mod 2^64
  const uint64_t s = (lo * k) & kMontMask;
  const uint32_t s0 = static_cast<uint32_t>(s), s1 = static_cast<uint32_t>(s >> 32);
  const uint64_t u = mad32(s0, q0, static_cast<uint32_t>(p));
  y = mad32(s1, q0, mad32(s0, q1, y)) + (u >> 32);
  return static_cast<int64_t>(mad32(s1 << 2, q1, mad32(w1 << 2, b1, y >> 30)));
#endif
}

// Shoup's product for words whose value only matters modulo q: W b mod q in
// [0, 2q), with W < q a plain (not Montgomery) constant and W' = floor(W 2^64 / q),
// for any b < 2^64.  qt = floor(W' b / 2^64) undershoots W b / q by less than 2, so
// W b - qt q, computed modulo 2^64, is the product up to one q.
FHE_HD uint64_t shoup_mult(uint64_t w, uint64_t wp, uint64_t b, uint64_t q) {
#ifdef __CUDA_ARCH__
  uint64_t r;
  asm("{\n\t"
      ".reg .u32 w0, w1, p0, p1, b0, b1, q0, q1, t0, t1, t2, r0, r1, s0, s1;\n\t"
      "mov.b64 {w0, w1}, %1;\n\t"
      "mov.b64 {p0, p1}, %2;\n\t"
      "mov.b64 {b0, b1}, %3;\n\t"
      "mov.b64 {q0, q1}, %4;\n\t"
      "mul.hi.u32 t0, p0, b0;\n\t"          // (t2, t1) = high 64 bits of W' b
      "mad.lo.cc.u32 t0, p0, b1, t0;\n\t"
      "madc.hi.u32 t1, p0, b1, 0;\n\t"
      "mad.lo.cc.u32 t0, p1, b0, t0;\n\t"
      "madc.hi.cc.u32 t1, p1, b0, t1;\n\t"
      "addc.u32 t2, 0, 0;\n\t"
      "mad.lo.cc.u32 t1, p1, b1, t1;\n\t"
      "madc.hi.u32 t2, p1, b1, t2;\n\t"
      "mul.lo.u32 r0, w0, b0;\n\t"          // W b mod 2^64
      "mul.hi.u32 r1, w0, b0;\n\t"
      "mad.lo.u32 r1, w0, b1, r1;\n\t"
      "mad.lo.u32 r1, w1, b0, r1;\n\t"
      "mul.lo.u32 s0, t1, q0;\n\t"          // qt q mod 2^64
      "mul.hi.u32 s1, t1, q0;\n\t"
      "mad.lo.u32 s1, t1, q1, s1;\n\t"
      "mad.lo.u32 s1, t2, q0, s1;\n\t"
      "sub.cc.u32 r0, r0, s0;\n\t"
      "subc.u32 r1, r1, s1;\n\t"
      "mov.b64 %0, {r0, r1};\n\t"
      "}"
      : "=l"(r)
      : "l"(w), "l"(wp), "l"(b), "l"(q));
  return r;
#else
  const uint64_t qt = static_cast<uint64_t>((static_cast<unsigned __int128>(wp) * b) >> 64);
  return w * b - qt * q;
#endif
}

// mont_mult taking the short form when both words are below 2^62 (lazy [0, 2q)
// words and table constants are); every engine prime is below 2^61.  The same word
// as mont_mult for every input.  Used in the element-wise kernels and the NTT's
// loaders and storers; in the serial triangles of the Garner digits and the ModDown
// divisors the branch measured slower.
FHE_HD int64_t mont_mult_lazy(int64_t a, int64_t b, uint64_t q, uint64_t k) {
  const uint64_t ua = static_cast<uint64_t>(a), ub = static_cast<uint64_t>(b);
  if (((ua | ub) >> kMontBits) == 0) return mont_mult_small(ua, ub, q, k);
  return mont_mult(a, b, q, k);
}

// Montgomery exit (unit.h:25-31): REDC of a single (sign-extended) word.
FHE_HD int64_t mont_exit(int64_t x, uint64_t q, uint64_t k) {
  return redc_wide(static_cast<uint64_t>(x), x < 0 ? ~uint64_t(0) : 0, q, k);
}

// Lazy sums of REDC terms.
//
// For operands a_i, b_i in [0, 2^61) and q < 2^61 every t_i = REDC(a_i b_i) lies in
// [0, 2q), and a chain acc = guard(acc + t_i, 2q) started from t_0 equals
// (sum t_i) mod 2q.  Since a_i b_i + s_i q = t_i 2^62 exactly (s_i = a_i b_i k mod
// 2^62), sum t_i = (sum a_i b_i + q sum s_i) / 2^62: the products and the s_i are
// accumulated in 128 bits and reduced once.  Used for the ModUp contraction and
// the key inner product, whose reference form is such a chain.
struct RedcSum {
  uint64_t p_lo = 0, p_hi = 0;  // sum of a_i b_i
  uint64_t s_lo = 0, s_hi = 0;  // sum of s_i
  FHE_HD void add(uint64_t a, uint64_t b, uint64_t k) {
    uint64_t lo, hi;
    mul_wide(a, b, lo, hi);
    const uint64_t nl = p_lo + lo;
    p_hi += hi + (nl < p_lo ? 1 : 0);
    p_lo = nl;
    const uint64_t s = (lo * k) & kMontMask;
    const uint64_t ns = s_lo + s;
    s_hi += ns < s_lo ? 1 : 0;
    s_lo = ns;
  }
  // (sum t_i) mod m for m = q or 2q, given the sum is below 64 m; inv_m ~ 1/m.
  FHE_HD int64_t reduce(uint64_t q, uint64_t m, double inv_m) const {
    uint64_t ql, qh;
    mul_wide(s_lo, q, ql, qh);
    qh += s_hi * q;
    const uint64_t zl = p_lo + ql;
    const uint64_t zh = p_hi + qh + (zl < p_lo ? 1 : 0);
    const uint64_t t_lo = (zh << 2) | (zl >> kMontBits);  // T = Z >> 62 < 2^66
    const uint64_t t_hi = zh >> kMontBits;
    const double td = static_cast<double>(t_hi) * 18446744073709551616.0 + static_cast<double>(t_lo);
    const uint64_t est = static_cast<uint64_t>(td * inv_m);
    int64_t r = static_cast<int64_t>(t_lo - est * m);  // |T - est m| < 2m
    const int64_t ms = static_cast<int64_t>(m);
    if (r < 0) r += ms;
    if (r >= ms) r -= ms;
    return r;
  }
};

// sum_i a_i b_i accumulated exactly in 128 bits and reduced by one REDC of the whole
// sum: the value is that of the chain of REDC(a_i b_i) terms modulo q, but not its
// representative.  For sums whose consumers only use the value modulo q (ModUp's
// extended limbs feed value-only transforms).  Valid for a_i, b_i < 2^61 and at most
// 16 terms: the sum is below 2^126 and its REDC below (terms / 2 + 1) q.
struct WideSum {
  uint64_t lo = 0, hi = 0;
  // sum += a b (the caller keeps the sum below 2^128).  On the device the four
  // 32 x 32 partial products go straight into the 128-bit sum through the carry
  // flag, column by column.
  FHE_HD void add(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    asm("{\n\t"
        ".reg .u32 a0, a1, b0, b1, s0, s1, s2, s3;\n\t"
        "mov.b64 {a0, a1}, %2;\n\t"
        "mov.b64 {b0, b1}, %3;\n\t"
        "mov.b64 {s0, s1}, %0;\n\t"
        "mov.b64 {s2, s3}, %1;\n\t"
        "mad.lo.cc.u32 s0, a0, b0, s0;\n\t"
        "madc.hi.cc.u32 s1, a0, b0, s1;\n\t"
        "madc.lo.cc.u32 s2, a1, b1, s2;\n\t"
        "madc.hi.u32 s3, a1, b1, s3;\n\t"
        "mad.lo.cc.u32 s1, a0, b1, s1;\n\t"
        "madc.hi.cc.u32 s2, a0, b1, s2;\n\t"
        "addc.u32 s3, s3, 0;\n\t"
        "mad.lo.cc.u32 s1, a1, b0, s1;\n\t"
        "madc.hi.cc.u32 s2, a1, b0, s2;\n\t"
        "addc.u32 s3, s3, 0;\n\t"
        "mov.b64 %0, {s0, s1};\n\t"
        "mov.b64 %1, {s2, s3};\n\t"
        "}"
        : "+l"(lo), "+l"(hi)
        : "l"(a), "l"(b));
#else
    uint64_t l, h;
    mul_wide(a, b, l, h);
    const uint64_t nl = lo + l;
    hi += h + (nl < lo ? 1 : 0);
    lo = nl;
#endif
  }
  // REDC(sum) reduced modulo m (q or 2q); inv_m ~ 1/m.
  FHE_HD int64_t reduce(uint64_t q, uint64_t k, uint64_t m, double inv_m) const {
    RedcSum r;
    r.p_lo = lo;
    r.p_hi = hi;
    r.s_lo = (lo * k) & kMontMask;
    return r.reduce(q, m, inv_m);
  }
};

// One word of rescale_once_ (core_rescale.cpp:5-25): (x_j - x_0) reduced, times
// q_0^-1 R, plus the rounder of x_0, reduced to [0, q).
template <bool LAZY = false>
FHE_HD int64_t rescale_word(int64_t xj, int64_t x0, int64_t rounder, uint64_t q, uint64_t k,
                            int64_t constant) {
  const int64_t qs = static_cast<int64_t>(q), q2 = qs << 1;
  int64_t v = xj - x0;  // mont_subtract (unit.cpp:58-64)
  v = v >= 0 ? v : v + q2;
  v = guard(v, qs);
  v = LAZY ? mont_mult_lazy(v, constant, q, k) : mont_mult(v, constant, q, k);
  v = guard(v + rounder, q2);  // add_tiled
  return guard(v, qs);
}

// rescale_word with the product by q_0^-1 taken as Shoup's when the reduced
// difference is below 2^62: both products lie in [0, 2q) and have the same value,
// and the two guards after them leave the canonical residue, so the word is the
// same.  shoup = (C, C') of the constant (KeySwitchTables::rescale_shoup).
FHE_HD int64_t rescale_word_shoup(int64_t xj, int64_t x0, int64_t rounder, uint64_t q, uint64_t k,
                                  int64_t constant, const int64_t *shoup) {
  const int64_t qs = static_cast<int64_t>(q), q2 = qs << 1;
  int64_t v = xj - x0;  // mont_subtract (unit.cpp:58-64)
  v = v >= 0 ? v : v + q2;
  v = guard(v, qs);
  if ((static_cast<uint64_t>(v) >> kMontBits) == 0)
    v = static_cast<int64_t>(shoup_mult(static_cast<uint64_t>(shoup[0]), static_cast<uint64_t>(shoup[1]),
                                        static_cast<uint64_t>(v), q));
  else
    v = mont_mult(v, constant, q, k);
  v = guard(v + rounder, q2);  // add_tiled
  return guard(v, qs);
}

FHE_HD bool redc_operand_ok(int64_t x) {
  return static_cast<uint64_t>(x) < (uint64_t(1) << 61);
}

// Per-prime constants as the kernels read them.
struct PrimeTables {
  const uint64_t *q;
  const uint64_t *k;
  const int64_t *r_squared;
  const int64_t *n_inverse;
  const int64_t *root;          // [prime][N-1]
  const int64_t *root_inverse;  // [prime][N-1]
  const int64_t *root_reduced;          // root, each word reduced to [0, q)
  const int64_t *root_inverse_reduced;  // root_inverse, each word reduced to [0, q)
  // The same twiddles as (W, W') pairs for shoup_mult: W = root R^-1 mod q, the
  // plain twiddle, and W' = floor(W 2^64 / q); [prime][N-1][2].
  const int64_t *root_shoup;
  const int64_t *root_inverse_shoup;
  // (C, C') per prime for the reduced exit of a value-only inverse transform:
  // C = N^-1 R^-1 mod q, the value mont_exit(mont_mult(v, n_inverse)) multiplies by,
  // and C' = floor(C 2^64 / q).
  const int64_t *exit_shoup;
  const double *inv_q;          // 1 / q
  const double *inv_2q;         // 1 / (2q)
  int log_n;
};

}  // namespace fhe_b200
