// Exact arithmetic modulo the Goldilocks prime p = 2^64 - 2^32 + 1.
//
// Replaces the reference's common/arithmetics.cuh:26-312 (add_Mod, sub_Mod,
// mul_Mod, pow_Mod, inv_Mod and the shift24/48/72 family).  Written from the
// two identities 2^64 == 2^32 - 1 and 2^96 == -1 (mod p); every function keeps
// its result canonical in [0, p).  The functions are __host__ __device__ so the
// CPU test suite checks them bit-for-bit against the oracle.
#pragma once
#include <stdint.h>

// LNT_GL_SHORT = 1 (default): carry chains one or two instructions shorter per
// operation (557 vs 561 us per squaring at n = 2^23 with the radix-8 kernels;
// with spilling radix-16 kernels they were slower).  0: the longer chains.
#ifndef LNT_GL_SHORT
#define LNT_GL_SHORT 1
#endif
// LNT_GL_SUBMAD = 1: the borrow correction of sub_chain on the multiplier pipe.
#ifndef LNT_GL_SUBMAD
#define LNT_GL_SUBMAD 1
#endif

#if defined(__CUDACC__)
#define GL_HD __host__ __device__ __forceinline__
#else
#define GL_HD static inline
#endif

namespace gl {

constexpr uint64_t P = 0xFFFFFFFF00000001ull;
constexpr uint64_t EPS = 0x00000000FFFFFFFFull;  // 2^64 mod p
constexpr uint64_t HALF = P >> 1;                // values above this are negative

GL_HD uint64_t mulhi(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

#if defined(__CUDA_ARCH__)
// a - b with the 32-bit carry chain: the borrow of the subtraction itself
// selects the correction (+p: low word + 1, high word + 2^32 - 1), no compare.
__device__ __forceinline__ uint64_t sub_chain(uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1) {
  uint32_t d0, d1;
#if LNT_GL_SUBMAD
  // the wrapped difference plus p times the borrow b, with the borrow mask
  // m = -b: its low word gains m * m = b (mod 2^32) on the multiplier pipe (m is
  // not a constant, so the multiply stays a multiply), its high word m plus the
  // carry.  Same result and instruction count as the two subtractions below,
  // one of them moved off the integer ALU pipe.
  asm("{\n\t"
      ".reg .u32 m;\n\t"
      "sub.cc.u32    %0, %2, %4;\n\t"
      "subc.cc.u32   %1, %3, %5;\n\t"
      "subc.u32      m, 0, 0;\n\t"
      "mad.lo.cc.u32 %0, m, m, %0;\n\t"
      "addc.u32      %1, %1, m;\n\t"
      "}"
      : "=r"(d0), "=r"(d1)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
#elif LNT_GL_SHORT
  // the wrapped difference minus 2^64 - p = 2^32 - 1, which is the borrow mask
  asm("{\n\t"
      ".reg .u32 m;\n\t"
      "sub.cc.u32  %0, %2, %4;\n\t"
      "subc.cc.u32 %1, %3, %5;\n\t"
      "subc.u32    m, 0, 0;\n\t"
      "sub.cc.u32  %0, %0, m;\n\t"
      "subc.u32    %1, %1, 0;\n\t"
      "}"
      : "=r"(d0), "=r"(d1)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
#else
  uint32_t m;
  asm("{\n\t"
      "sub.cc.u32  %0, %3, %5;\n\t"
      "subc.cc.u32 %1, %4, %6;\n\t"
      "subc.u32    %2, 0, 0;\n\t"
      "}"
      : "=r"(d0), "=r"(d1), "=r"(m)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
  asm("{\n\t"
      "add.cc.u32 %0, %0, %2;\n\t"
      "addc.u32   %1, %1, %3;\n\t"
      "}"
      : "+r"(d0), "+r"(d1)
      : "r"(m & 1u), "r"(m));
#endif
  return ((uint64_t)d1 << 32) | d0;
}
#endif

GL_HD uint64_t sub(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return sub_chain((uint32_t)a, (uint32_t)(a >> 32), (uint32_t)b, (uint32_t)(b >> 32));
#else
  uint64_t d = a - b;
  return (a < b) ? d + P : d;
#endif
}

GL_HD uint64_t add(uint64_t a, uint64_t b) {
  // a + b - p = a - (p - b): one subtraction and one conditional correction
#if defined(__CUDA_ARCH__)
  uint32_t t0, t1;
  asm("{\n\t"
      "sub.cc.u32 %0, 1, %2;\n\t"
      "subc.u32   %1, 0xFFFFFFFF, %3;\n\t"
      "}"
      : "=r"(t0), "=r"(t1)
      : "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
  return sub_chain((uint32_t)a, (uint32_t)(a >> 32), t0, t1);
#else
  const uint64_t t = P - b;
  const uint64_t d = a - t;
  return (a < t) ? d + P : d;
#endif
}

GL_HD uint64_t neg(uint64_t a) { return a ? P - a : 0; }

// LNT_GL_MUL selects the device reductions: 1 (default) reduce_words below,
// with the product r2 (2^32 - 1) on the multiplier pipe, which the
// integer-bound kernels leave mostly idle; 0 the add/sub chains of mul
// (r2 (2^32 - 1) from two subtractions).  At n = 2^23: 462.5 us per squaring
// with 1, 519.4 with 0; 1 with the 128-bit product from four 32 x 32 -> 64
// multiply-adds instead of the mad chain of mul: 471.6.
#ifndef LNT_GL_MUL
#define LNT_GL_MUL 1
#endif

#if defined(__CUDA_ARCH__)
// (t1:t0) in [0, 2^64) to [0, p): a value >= p has the high word 2^32 - 1 and
// a non-zero low word, and minus p it is the low word minus one.
__device__ __forceinline__ uint64_t canon_words(uint32_t t0, uint32_t t1) {
  if (t1 == 0xFFFFFFFFu && t0 != 0u) {
    t0 -= 1u;
    t1 = 0u;
  }
  return ((uint64_t)t1 << 32) | t0;
}

// r0 + r1 2^32 + r2 2^64 + r3 2^96 mod p for any 32-bit words, canonical:
// (r1:r0) + r2 (2^32 - 1) - r3 (2^64 = 2^32 - 1, 2^96 = -1).  The first sum
// runs on the multiplier (mad with carry); with c its carry and b the borrow
// of the subtraction the value is the 64-bit word plus (c - b)(2^32 - 1).
// That correction cannot overflow (c = 1 leaves at most 2^64 - 2^33) nor
// underflow (b = 1 leaves at least p), and its result is below p, so only
// c = b can leave a word >= p for canon_words.
__device__ __forceinline__ uint64_t reduce_words(uint32_t r0, uint32_t r1, uint32_t r2,
                                                 uint32_t r3) {
  uint32_t t0, t1;
  asm("{\n\t"
      ".reg .u32 cm, b, lo, hi;\n\t"
      "mad.lo.cc.u32  %0, %4, 0xFFFFFFFF, %2;\n\t"
      "madc.hi.cc.u32 %1, %4, 0xFFFFFFFF, %3;\n\t"
      "addc.u32       cm, 0xFFFFFFFF, 0;\n\t"  // c - 1
      "sub.cc.u32     %0, %0, %5;\n\t"
      "subc.cc.u32    %1, %1, 0;\n\t"
      "subc.u32       b, 0, 0;\n\t"            // -b
      "sub.u32        lo, 0xFFFFFFFF, cm;\n\t"
      "sub.u32        lo, lo, b;\n\t"          // low word of (c - b)(2^32 - 1): b - c
      "and.b32        hi, b, cm;\n\t"          // high word: all ones iff c - b = -1
      "add.cc.u32     %0, %0, lo;\n\t"
      "addc.u32       %1, %1, hi;\n\t"
      "}"
      : "=r"(t0), "=r"(t1)
      : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
  return canon_words(t0, t1);
}

// r0 + r1 2^32 + r2 2^64 mod p: (r1:r0) + r2 (2^32 - 1) on the multiplier,
// its carry c folded back as c 2^32 - c (c = 1 leaves at most (2^32 - 1)^2 - 1,
// so neither step wraps and the result is below p).
__device__ __forceinline__ uint64_t reduce_words3(uint32_t r0, uint32_t r1, uint32_t r2) {
  uint32_t t0, t1;
  asm("{\n\t"
      ".reg .u32 c;\n\t"
      "mad.lo.cc.u32  %0, %4, 0xFFFFFFFF, %2;\n\t"
      "madc.hi.cc.u32 %1, %4, 0xFFFFFFFF, %3;\n\t"
      "addc.u32       c, 0, 0;\n\t"
      "add.u32        %1, %1, c;\n\t"
      "sub.cc.u32     %0, %0, c;\n\t"
      "subc.u32       %1, %1, 0;\n\t"
      "}"
      : "=r"(t0), "=r"(t1)
      : "r"(r0), "r"(r1), "r"(r2));
  return canon_words(t0, t1);
}
#endif

// lo + 2^64 * hi, with hi = h1 * 2^32 + h0, is lo + h0 * (2^32 - 1) - h1.
GL_HD uint64_t reduce128(uint64_t lo, uint64_t hi) {
  uint64_t h1 = hi >> 32, h0 = hi & 0xFFFFFFFFull;
  uint64_t t = lo - h1;
  if (lo < h1) t -= EPS;  // borrow: t - 2^64 == t - EPS (mod p)
  uint64_t m = (h0 << 32) - h0;
  uint64_t r = t + m;
  if (r < m) r += EPS;    // carry: r + 2^64 == r + EPS (mod p)
  return r >= P ? r - P : r;
}

GL_HD uint64_t mul(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  // 128-bit product from 32-bit limbs (multiplier pipe), then the reduction
  // lo + r2 (2^32 - 1) - r3.
  uint32_t r0, r1, r2, r3;
  asm("{\n\t"
      "mul.lo.u32     %0, %4, %6;\n\t"
      "mul.hi.u32     %1, %4, %6;\n\t"
      "mad.lo.cc.u32  %1, %4, %7, %1;\n\t"
      "madc.hi.u32    %2, %4, %7, 0;\n\t"
      "mad.lo.cc.u32  %1, %5, %6, %1;\n\t"
      "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
      "madc.hi.u32    %3, %5, %7, 0;\n\t"
      "mad.lo.cc.u32  %2, %5, %7, %2;\n\t"
      "addc.u32       %3, %3, 0;\n\t"
      "}"
      : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
      : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
#if LNT_GL_MUL == 1
  return reduce_words(r0, r1, r2, r3);
#else
#if LNT_GL_SHORT
  // t = (r1:r0) - r3 (borrow: minus the mask 2^32 - 1, as sub_chain), then
  // t + r2 (2^32 - 1) with its carry read by addc and folded back as 2^32 - 1.
  // An add chain's carry is never read with subc: a subtraction reads the
  // flag with the opposite sense (measured on sm_100a).
  uint32_t t0, t1;
  asm("{\n\t"
      ".reg .u32 m, u0, u1, c;\n\t"
      "sub.cc.u32  %0, %2, %4;\n\t"
      "subc.cc.u32 %1, %3, 0;\n\t"
      "subc.u32    m, 0, 0;\n\t"
      "sub.cc.u32  %0, %0, m;\n\t"
      "subc.u32    %1, %1, 0;\n\t"
      "sub.cc.u32  u0, 0, %5;\n\t"
      "subc.u32    u1, %5, 0;\n\t"
      "add.cc.u32  %0, %0, u0;\n\t"
      "addc.cc.u32 %1, %1, u1;\n\t"
      "addc.u32    c, 0, 0;\n\t"
      "neg.s32     m, c;\n\t"
      "add.cc.u32  %0, %0, m;\n\t"
      "addc.u32    %1, %1, 0;\n\t"
      "}"
      : "=r"(t0), "=r"(t1)
      : "r"(r0), "r"(r1), "r"(r3), "r"(r2));
#else
  uint32_t t0, t1, m;
  asm("{\n\tsub.cc.u32 %0, %3, %5;\n\tsubc.cc.u32 %1, %4, 0;\n\tsubc.u32 %2, 0, 0;\n\t}"
      : "=r"(t0), "=r"(t1), "=r"(m)
      : "r"(r0), "r"(r1), "r"(r3));
  asm("{\n\tadd.cc.u32 %0, %0, %2;\n\taddc.u32 %1, %1, %3;\n\t}"
      : "+r"(t0), "+r"(t1)
      : "r"(m & 1u), "r"(m));
  uint32_t u0, u1, c;
  asm("{\n\tsub.cc.u32 %0, 0, %2;\n\tsubc.u32 %1, %2, 0;\n\t}" : "=r"(u0), "=r"(u1) : "r"(r2));
  asm("{\n\tadd.cc.u32 %0, %0, %3;\n\taddc.cc.u32 %1, %1, %4;\n\taddc.u32 %2, 0, 0;\n\t}"
      : "+r"(t0), "+r"(t1), "=r"(c)
      : "r"(u0), "r"(u1));
  asm("{\n\tadd.cc.u32 %0, %0, %2;\n\taddc.u32 %1, %1, 0;\n\t}" : "+r"(t0), "+r"(t1) : "r"(0u - c));
#endif
  const uint64_t r = ((uint64_t)t1 << 32) | t0;
  return r >= P ? r - P : r;
#endif
#else
  return reduce128(a * b, mulhi(a, b));
#endif
}

GL_HD uint64_t sqr(uint64_t a) { return mul(a, a); }

GL_HD uint64_t pow(uint64_t a, uint64_t e) {
  uint64_t r = 1;
  while (e) {
    if (e & 1) r = mul(r, a);
    a = mul(a, a);
    e >>= 1;
  }
  return r;
}

GL_HD uint64_t inv(uint64_t a) { return pow(a, P - 2); }

// x * 2^s for 0 <= s < 192 (2 has multiplicative order 192 modulo p).
// Only shifts and adds: no multiplier.
GL_HD uint64_t mul_pow2(uint64_t x, unsigned s) {
  bool negate = false;
  if (s >= 96) { s -= 96; negate = true; }  // 2^96 == -1
  uint64_t r;
  if (s == 0) {
    r = x;
  } else if (s < 64) {
    r = reduce128(x << s, x >> (64 - s));
  } else {
    // x 2^s = (hi 2^64 + lo) 2^64 with (hi, lo) = x 2^k, k = s - 64 < 32;
    // 2^128 == -2^32, so this is reduce(lo 2^64) - hi 2^32 with hi 2^32 < p.
    unsigned k = s - 64;
    uint64_t lo = x << k, hi = k ? (x >> (64 - k)) : 0;
    r = sub(reduce128(0, lo), hi << 32);
  }
  return negate ? neg(r) : r;
}

// d * w for a digit |d| < 2^32 (a balanced or non-negative residue word) and a
// field element w: a 32 x 64-bit product (96 bits, so the reduction has no
// 2^96 term), then the sign.  Equals mul(from_signed(d), w).
GL_HD uint64_t mul_digit(int64_t d, uint64_t w) {
  const bool negative = d < 0;
  const uint32_t a = (uint32_t)(negative ? -d : d);
#if defined(__CUDA_ARCH__) && LNT_GL_MUL >= 1
  uint32_t r0, r1, r2;
  asm("{\n\t"
      "mul.lo.u32     %0, %3, %4;\n\t"
      "mul.hi.u32     %1, %3, %4;\n\t"
      "mad.lo.cc.u32  %1, %3, %5, %1;\n\t"
      "madc.hi.u32    %2, %3, %5, 0;\n\t"
      "}"
      : "=r"(r0), "=r"(r1), "=r"(r2)
      : "r"(a), "r"((uint32_t)w), "r"((uint32_t)(w >> 32)));
  const uint64_t r = reduce_words3(r0, r1, r2);
#elif defined(__CUDA_ARCH__)
  uint32_t t0, t1;
  asm("{\n\t"
      ".reg .u32 r2, u0, u1, c, m;\n\t"
      "mul.lo.u32     %0, %2, %3;\n\t"
      "mul.hi.u32     %1, %2, %3;\n\t"
      "mad.lo.cc.u32  %1, %2, %4, %1;\n\t"
      "madc.hi.u32    r2, %2, %4, 0;\n\t"
      // (t1:t0) + r2 (2^32 - 1): plus (r2 - [r2 != 0]) : (0 - r2)
      "sub.cc.u32     u0, 0, r2;\n\t"
      "subc.u32       u1, r2, 0;\n\t"
      "add.cc.u32     %0, %0, u0;\n\t"
      "addc.cc.u32    %1, %1, u1;\n\t"
      "addc.u32       c, 0, 0;\n\t"
      "neg.s32        m, c;\n\t"
      "add.cc.u32     %0, %0, m;\n\t"
      "addc.u32       %1, %1, 0;\n\t"
      "}"
      : "=r"(t0), "=r"(t1)
      : "r"(a), "r"((uint32_t)w), "r"((uint32_t)(w >> 32)));
  uint64_t r = ((uint64_t)t1 << 32) | t0;
  r = r >= P ? r - P : r;
#else
  const uint64_t r = reduce128((uint64_t)a * w, mulhi((uint64_t)a, w));
#endif
  return negative ? neg(r) : r;
}

// Balanced digit d (|d| < 2^62) as a field element.
GL_HD uint64_t from_signed(int64_t d) { return d >= 0 ? (uint64_t)d : (uint64_t)d + P; }

// Field element as a signed integer in (-p/2, p/2].
GL_HD int64_t to_signed(uint64_t c) { return c > HALF ? (int64_t)(c - P) : (int64_t)c; }

}  // namespace gl
