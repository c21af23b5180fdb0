// Register-resident NTTs of up to 64 points with power-of-two roots.
//
// In F_p, 2 has order 192 and 554^((p-1)/64) = 2^3, so the R-point root used by
// every sub-transform of the reference's roots (pre_calculation.cu:61-66) with
// R | 64 is omega_R = 2^(192/R): each butterfly twiddle is a multiplication by
// a power of two, done with shifts and adds (shl_c), never the multiplier.  The
// reference reaches this only for its radix-4/8 inner roots and its 32x32 row
// kernel (kernels/fftr_sqr_ifftr__r2_32x32_1024.cu); here every transform of
// length L = 64 * R is split into register passes of 64 and R points with one
// table-twiddle level between them.
//
// dif<R>: natural order in, bit-reversed order out (decimation in frequency).
// dit_inv<R>: bit-reversed in, natural out, inverse roots, unscaled.
// Shift amounts are template arguments, so every butterfly compiles to a fixed
// shift/add sequence.
#pragma once
#include <stdint.h>
#include <utility>
#include "goldilocks.cuh"

namespace lnt {

// x * 2^S mod p, 0 <= S < 192, S a compile-time constant.
template <unsigned S>
GL_HD uint64_t shl_c(uint64_t x) {
  if constexpr (S == 0) {
    return x;
  } else if constexpr (S >= 96) {
    return gl::neg(shl_c<S - 96>(x));  // 2^96 = -1
#if defined(__CUDA_ARCH__) && LNT_GL_MUL >= 1
    // device: the shifted words, reduced by gl::reduce_words(3)
  } else if constexpr (S < 32) {
    const uint64_t lo = x << S;  // + 2^64 (x >> (64 - S)), below 2^32
    return gl::reduce_words3((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)(x >> (64 - S)));
  } else if constexpr (S == 32) {
    return gl::reduce_words3(0u, (uint32_t)x, (uint32_t)(x >> 32));
  } else if constexpr (S < 64) {
    const uint64_t hi = x >> (64 - S);  // x 2^S = (x0 << (S - 32)) 2^32 + hi 2^64
    return gl::reduce_words(0u, (uint32_t)x << (S - 32), (uint32_t)hi, (uint32_t)(hi >> 32));
  } else {
    // x 2^S = y 2^64 + z 2^128 with y = x << k (64 bits), z = x >> (64 - k) < 2^32
    // (k = S - 64); 2^128 = -2^32 and p - z 2^32 = (2^32 - 1 - z) 2^32 + 1
    constexpr unsigned k = S - 64;
    const uint64_t y = x << k;
    const uint32_t z = k ? (uint32_t)(x >> ((64 - k) & 63)) : 0u;
    return gl::reduce_words(1u, ~z, (uint32_t)y, (uint32_t)(y >> 32));
  }
#else
  } else if constexpr (S <= 32) {
    // x 2^S = lo + 2^64 hi with hi < 2^32: lo + hi (2^32 - 1)
    const uint64_t lo = x << S, hi = x >> (64 - S);
    const uint64_t m = (hi << 32) - hi;
    uint64_t r = lo + m;
    if (r < m) r += gl::EPS;
    return r >= gl::P ? r - gl::P : r;
  } else if constexpr (S < 64) {
    return gl::reduce128(x << S, x >> (64 - S));
  } else {
    // x 2^S = (hi 2^64 + lo) 2^64 with (hi, lo) = x 2^k; 2^128 = -2^32
    constexpr unsigned k = S - 64;
    const uint64_t lo = x << k, hi = k ? (x >> ((64 - k) & 63)) : 0;
    return gl::sub(gl::reduce128(0, lo), hi << 32);
  }
#endif
}

// a*w, b -> (a + b, (a - b) * 2^S): the DIF butterfly with a power-of-two twiddle.
template <unsigned S>
GL_HD void bfly_dif(uint64_t& a, uint64_t& b) {
  const uint64_t s = gl::add(a, b);
  if constexpr (S >= 96)
    b = shl_c<S - 96>(gl::sub(b, a));
  else
    b = shl_c<S>(gl::sub(a, b));
  a = s;
}

// (a, b) -> (a + b 2^S, a - b 2^S): the DIT butterfly.
template <unsigned S>
GL_HD void bfly_dit(uint64_t& a, uint64_t& b) {
  const uint64_t t = shl_c<S % 96>(b);
  if constexpr (S >= 96) {
    const uint64_t s = gl::sub(a, t);
    b = gl::add(a, t);
    a = s;
  } else {
    const uint64_t s = gl::add(a, t);
    b = gl::sub(a, t);
    a = s;
  }
}

namespace detail {

// one DIF stage of half-size H over R registers: I enumerates the R/2 butterflies
template <int R, int H, int... I>
GL_HD void dif_stage(uint64_t* x, std::integer_sequence<int, I...>) {
  (bfly_dif<(unsigned)((192 / (2 * H)) * (I % H))>(x[(I / H) * 2 * H + I % H],
                                                     x[(I / H) * 2 * H + I % H + H]),
   ...);
}

template <int R, int H>
GL_HD void dif_stages(uint64_t* x) {
  dif_stage<R, H>(x, std::make_integer_sequence<int, R / 2>{});
  if constexpr (H > 1) dif_stages<R, H / 2>(x);
}

// inverse twiddle of omega_2H^i is 2^(192 - 192 i / 2H) (i > 0)
template <int R, int H, int... I>
GL_HD void dit_stage(uint64_t* x, std::integer_sequence<int, I...>) {
  (bfly_dit<(unsigned)((192 - (192 / (2 * H)) * (I % H)) % 192)>(
       x[(I / H) * 2 * H + I % H], x[(I / H) * 2 * H + I % H + H]),
   ...);
}

template <int R, int H>
GL_HD void dit_stages(uint64_t* x) {
  dit_stage<R, H>(x, std::make_integer_sequence<int, R / 2>{});
  if constexpr (2 * H < R) dit_stages<R, 2 * H>(x);
}

}  // namespace detail

template <int R>
GL_HD void dif(uint64_t (&x)[R]) {
  static_assert(R >= 1 && R <= 64 && (R & (R - 1)) == 0, "register NTT size");
  if constexpr (R > 1) detail::dif_stages<R, R / 2>(x);
}

template <int R>
GL_HD void dit_inv(uint64_t (&x)[R]) {
  static_assert(R >= 1 && R <= 64 && (R & (R - 1)) == 0, "register NTT size");
  if constexpr (R > 1) detail::dit_stages<R, 1>(x);
}

// bit reversal of i over log2(R) bits, at compile time
template <int R>
GL_HD constexpr int brev_c(int i) {
  int r = 0;
  for (int b = 1; b < R; b <<= 1) {
    r <<= 1;
    if (i & b) r |= 1;
  }
  return r;
}

}  // namespace lnt
