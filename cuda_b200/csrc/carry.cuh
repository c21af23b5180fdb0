// Digit-carry helpers shared by the squaring kernels.
//
// The reference normalises every word to a non-negative digit of its width
// with a cyclic ripple of CAS loops (kernels/r2b.cu:25-50, core/atomic.cuh:23-32)
// and subtracts 2 with a serial borrow (kernels/m2.cu:23-41).  Here the words
// between squarings are BALANCED digits, |d| <= 2^(w-1) (plus a small excess
// at the end of a carry run), which keeps every convolution output below p/4 in
// magnitude so it can be read back as a signed integer.  Carries are resolved
// per run of consecutive words; a run hands its outgoing carry to the next run,
// which ripples it over its first words and absorbs what is left in its last
// word.  The canonical non-negative digits of the reference are produced only
// when a residue is read out (lnt_canon.cu).
#pragma once
#include <stdint.h>
#include "goldilocks.cuh"

namespace lnt {

// Largest carry a run may absorb into its last word.  The run lengths used are
// long enough that the carry has decayed to +-1 before the last word; anything
// above this bound means the exactness headroom is no longer guaranteed.
constexpr int64_t kAbsorbLimit = 2;

// Split a convolution output c into (hi, lo) with c = hi * 2^w + lo, 0 <= lo < 2^w.
// `unsigned_mode` reads c as a non-negative integer in [0, p); this is the case
// for the first squaring of non-negative digits, where the reference's length
// bound 2 n m^2 < p allows outputs above p/2.  Otherwise c is read as signed.
GL_HD void split_output(uint64_t c, bool unsigned_mode, unsigned w, int64_t& hi, int64_t& lo) {
  w &= 31u;  // widths are at most 30 bits (lnt_create): shifts by less than 32 are cheaper
  const uint64_t mask = (1ull << w) - 1;
  if (unsigned_mode) {
    hi = (int64_t)(c >> w);
    lo = (int64_t)(c & mask);
  } else {
    int64_t s = gl::to_signed(c);
    hi = s >> w;  // arithmetic shift: floor division
    lo = s & (int64_t)mask;
  }
}

// Balanced split of t: returns the digit in [-2^(w-1), 2^(w-1)) and sets k so
// that t = k 2^w + digit.
GL_HD int64_t balance(int64_t t, unsigned w, int64_t& k) {
  w &= 31u;  // as in split_output
  k = (t + (int64_t(1) << (w - 1))) >> w;
  return t - (k << w);
}

// A convolution output c plus the incoming carry, as one balanced digit (the
// return value) and the outgoing carry (*out).  The same pair as split_output
// followed by balance(lo + carry), with one balance of c + carry instead: with
// c = hi 2^w + lo, floor((c + carry + 2^(w-1)) / 2^w) = hi + floor((lo + carry +
// 2^(w-1)) / 2^w).  Signed outputs stay below p/4 in magnitude (the length
// policy's bound), so c + carry cannot overflow; the unsigned reading of the
// first squaring, up to p, keeps the split.
GL_HD int64_t carry_digit(uint64_t c, bool unsigned_mode, int64_t carry, unsigned w, int64_t& out) {
  int64_t q;
  if (unsigned_mode) {
    int64_t hi, lo;
    split_output(c, true, w, hi, lo);
    const int64_t d = balance(lo + carry, w, q);
    out = hi + q;
    return d;
  }
  const int64_t d = balance(gl::to_signed(c) + carry, w, q);
  out = q;
  return d;
}

}  // namespace lnt
