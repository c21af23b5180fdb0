// Per-block logic of the canonical readout (lnt_canon.cu), shared by the CUDA
// kernels and the CPU test harness (tests/native/canon_selftest.cpp).
//
// The reference keeps its words normalised after every squaring (kernels/r2b.cu
// cyclic carry to 0 <= d_j < 2^w_j, kernels/m2.cu borrow) and dumps them as they
// are (lucas_prp.cu:254-263).  Those digits are the unique base-(2^w_j)
// representation of the residue value in [0, M]; these steps rebuild that
// vector from the balanced form:
//   1. canon_local_block : a block of consecutive words normalises itself
//                          with carry-in 0 (pending run carries added in);
//   2. canon_hop_block   : the block adds its predecessor's outgoing carry and
//                          re-normalises; what leaves it is then in {-1, 0, 1},
//                          and its carry transfer function is recorded
//                          (a +1 crosses a block of maximal digits, a -1 a
//                          block of zeros);
//   3. canon_scan_*      : the transfer functions are composed in order and
//                          the cyclic wrap (2^q == 1 mod M) is resolved as the
//                          fixed point reached from carry 0;
//   4. canon_apply_block : each block adds its resolved carry-in.
#pragma once
#include <stdint.h>
#include "goldilocks.cuh"
#include "lnt_internal.h"

namespace lnt {

GL_HD int64_t canon_pending_carry(const CanonDesc& D, uint32_t j) {
  if (D.carry == nullptr) return 0;
  const uint32_t j1 = j % D.n1;
  if (j1 % D.tile) return 0;
  const uint32_t t = j1 / D.tile, r = j / D.n1;
  const size_t pi = t > 0 ? (size_t)(t - 1) * D.n2 + r
                          : (size_t)(D.ntiles - 1) * D.n2 + (r ? r - 1 : D.n2 - 1);
  return D.carry[pi];
}

GL_HD void canon_local_block(const CanonDesc& D, uint32_t b) {
  int64_t carry = 0;
  for (uint32_t k = 0; k < D.block; ++k) {
    const uint32_t j = b * D.block + k;
    const unsigned w = D.widths[j];
    const int64_t v = D.x[j] + carry + canon_pending_carry(D, j);
    D.out[j] = (uint64_t)(v & ((int64_t(1) << w) - 1));
    carry = v >> w;
  }
  D.blk_carry[b] = carry;
}

// A carry transfer function maps a carry in {-1, 0, 1} to one in {-1, 0, 1};
// it is stored as three 2-bit codes (carry + 1) at bits 0, 2, 4.
constexpr uint32_t kCanonIdentity = 0u | (1u << 2) | (2u << 4);

GL_HD int canon_apply_fn(uint32_t fn, int c) { return (int)((fn >> (2 * (c + 1))) & 3) - 1; }

GL_HD uint32_t canon_compose(uint32_t first, uint32_t then) {
  uint32_t r = 0;
  for (int c = -1; c <= 1; ++c)
    r |= (uint32_t)(canon_apply_fn(then, canon_apply_fn(first, c)) + 1) << (2 * (c + 1));
  return r;
}

// Returns false when the block's outgoing carry is outside {-1, 0, 1}.
GL_HD bool canon_hop_block(const CanonDesc& D, uint32_t b) {
  int64_t carry = D.blk_carry[b == 0 ? D.nblocks - 1 : b - 1];
  bool all_max = true, all_zero = true;
  for (uint32_t k = 0; k < D.block; ++k) {
    const uint32_t j = b * D.block + k;
    const unsigned w = D.widths[j];
    const int64_t mask = (int64_t(1) << w) - 1;
    int64_t d = (int64_t)D.out[j];
    if (carry != 0) {
      const int64_t v = d + carry;
      d = v & mask;
      carry = v >> w;
      D.out[j] = (uint64_t)d;
    }
    all_max = all_max && (d == mask);
    all_zero = all_zero && (d == 0);
  }
  bool ok = carry >= -1 && carry <= 1;
  if (!ok) carry = 0;
  uint32_t fn = 0;
  for (int c = -1; c <= 1; ++c) {
    const int pass = (c == 1 && all_max) ? 1 : (c == -1 && all_zero) ? -1 : 0;
    int64_t out = carry + pass;
    if (out < -1 || out > 1) {
      ok = false;
      out = 0;
    }
    fn |= (uint32_t)(out + 1) << (2 * (c + 1));
  }
  D.blk_fn[b] = (uint8_t)fn;
  return ok;
}

// Composition of the transfer functions of blocks [b0, b1).
GL_HD uint32_t canon_chunk_fn(const CanonDesc& D, uint32_t b0, uint32_t b1) {
  uint32_t f = kCanonIdentity;
  for (uint32_t b = b0; b < b1; ++b) f = canon_compose(f, D.blk_fn[b]);
  return f;
}

// Carry into word 0: the carry out of the top word, iterated from 0 to its
// fixed point (the functions are monotone, so two steps suffice).  Returns
// false if no fixed point was reached.
GL_HD bool canon_wrap_carry(uint32_t total, int& c) {
  c = 0;
  for (int i = 0; i < 3; ++i) c = canon_apply_fn(total, c);
  return canon_apply_fn(total, c) == c;
}

// Resolve the carry-in of every block of [b0, b1) from the carry into b0.
GL_HD void canon_chunk_cin(const CanonDesc& D, uint32_t b0, uint32_t b1, int c) {
  for (uint32_t b = b0; b < b1; ++b) {
    D.blk_cin[b] = (int8_t)c;
    c = canon_apply_fn(D.blk_fn[b], c);
  }
}

// Adds the block's resolved carry-in; reports whether some digit is below its
// maximum and whether some digit of index >= 1 is non-zero.
GL_HD void canon_apply_block(const CanonDesc& D, uint32_t b, bool& not_all_max,
                             bool& high_nonzero) {
  int64_t carry = D.blk_cin[b];
  for (uint32_t k = 0; k < D.block; ++k) {
    const uint32_t j = b * D.block + k;
    const unsigned w = D.widths[j];
    const int64_t mask = (int64_t(1) << w) - 1;
    int64_t d = (int64_t)D.out[j];
    if (carry != 0) {
      const int64_t v = d + carry;
      d = v & mask;
      carry = v >> w;
      D.out[j] = (uint64_t)d;
    }
    not_all_max = not_all_max || (d != mask);
    high_nonzero = high_nonzero || (j >= 1 && d != 0);
  }
}

}  // namespace lnt
