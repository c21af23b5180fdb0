// Transforms of up to 2^14 points in shared memory as register passes of radix
// up to 8 (or 16), shared by the two-pass kernels (lnt_radix16.cu) and the
// SMEM-resident kernel (lnt_resident.cu).
//
// A transform of length L = r0 * r1 * ... (every r a power of two) runs as
// passes over shared memory: pass j takes R = r_j elements at stride span_j / R
// from a block of span_j = L / (r0 ... r_{j-1}) words into registers, does an
// R-point DIF with power-of-two twiddles (ntt_core.cuh), multiplies by
// omega_span^(t * k) and writes back.  The result is in fully bit-reversed
// order; the inverse passes (DIT) take it back to natural order.  Per element a
// pass costs log2(R) shift butterflies and one table multiplication; the
// reference pays one general modular multiplication per radix-2 butterfly
// (core/fft_r2.cuh:17-107).
//
// Small unrolled bodies (one R-point transform) inside runtime loops keep the
// kernels small enough for the instruction cache; fully unrolled 64-point
// passes starved the SM of instructions.  Shared memory is padded by one word
// in 16 (sw below), which makes every pass stride bank-conflict free.
#pragma once
#include <stdint.h>

#include "goldilocks.cuh"
#include "ntt_core.cuh"

namespace lnt {
namespace smem {

__host__ __device__ __forceinline__ int sw(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded(int L) { return L + L / 16; }

struct Passes {
  int m;          // number of passes
  int radix[6];   // r_0 (largest stride) ... r_{m-1} (contiguous)
};

// Default largest pass radix.  8 (three radix-2 stages per pass) keeps a task's
// values, twiddles and addresses within the 64 registers that four row CTAs
// (two column CTAs) per SM allow; 16 needs one twiddle stage less per direction
// but spills there.  The two-pass kernels are built for both (a plan's `radix`)
// and the autotuner picks per length; the resident kernel uses 8.
constexpr int kDefaultRadixLog2 = 3;
constexpr int kMaxRadix = 1 << kDefaultRadixLog2;

// Passes of a length-2^log2L transform with radices of at most 2^b: the first
// pass takes the remainder, every later pass 2^b.
__host__ __device__ inline Passes make_passes(int log2L, int b = kDefaultRadixLog2) {
  Passes p{};
  int first = log2L % b;
  int rest = log2L - first;
  if (first == 0) {
    first = b;
    rest -= b;
  }
  p.radix[p.m++] = 1 << first;
  for (int k = 0; k < rest / b; ++k) p.radix[p.m++] = 1 << b;
  return p;
}

// ---- one task: R elements of one block, forward or inverse ----------------

// The R twiddles of one task, a 16-byte aligned run of the pass table: read as
// R/2 vector loads from one base address.  Element 0's twiddle is
// omega^(t brev(0)) = 1 in every task: it is loaded (the vector load) but not
// multiplied.
#ifndef LNT_TW_UNROLL
#define LNT_TW_UNROLL 8  // twiddle vectors loaded per unrolled step (register pressure)
#endif
constexpr int kTwUnroll = LNT_TW_UNROLL;
template <int R>
__device__ __forceinline__ void mul_task_twiddles(uint64_t (&v)[R], const uint64_t* tw) {
  const ulonglong2* w2 = reinterpret_cast<const ulonglong2*>(tw);
#pragma unroll kTwUnroll
  for (int k = 0; k < R / 2; ++k) {
    const ulonglong2 u = __ldg(w2 + k);
    if (k > 0) v[2 * k] = gl::mul(v[2 * k], u.x);
    v[2 * k + 1] = gl::mul(v[2 * k + 1], u.y);
  }
}

// Shared-memory position of element d (d < R) of a task whose first element is
// `off` (off = b * span + t, t < q, span = q * R, all powers of two):
// sw(off + q d) = sw(off) + q d + (q d >> 4), because the low four bits of
// off + q d never carry out of a padding group of 16 words.  For q >= 16 that
// is sw(off) + d (q + q / 16): one stride per pass, no per-element index math.
template <bool Big>
__device__ __forceinline__ int task_pos(int b0, int q, int qs, int d) {
  if constexpr (Big) {
    return b0 + d * qs;
  } else {
    const int k = q * d;
    return b0 + k + (k >> 4);
  }
}

// forward: DIF, then omega_span^(t k) (tw: this task's twiddles; unused when q == 1)
template <int R, bool Big>
__device__ __forceinline__ void task_dif(uint64_t* base, int b0, int q, int qs, const uint64_t* tw) {
  uint64_t v[R];
#pragma unroll
  for (int d = 0; d < R; ++d) v[d] = base[task_pos<Big>(b0, q, qs, d)];
  dif<R>(v);
  if (q > 1) mul_task_twiddles<R>(v, tw);
#pragma unroll
  for (int r = 0; r < R; ++r) base[task_pos<Big>(b0, q, qs, r)] = v[r];
}

// inverse: omega_span^-(t k), then DIT
template <int R, bool Big>
__device__ __forceinline__ void task_dit(uint64_t* base, int b0, int q, int qs, const uint64_t* itw) {
  uint64_t v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = base[task_pos<Big>(b0, q, qs, r)];
  if (q > 1) mul_task_twiddles<R>(v, itw);
  dit_inv<R>(v);
#pragma unroll
  for (int d = 0; d < R; ++d) base[task_pos<Big>(b0, q, qs, d)] = v[d];
}

// Offset of pass j's twiddles in a pass table (the spans of the passes before it).
__device__ __forceinline__ int pass_table_offset(const Passes& P, int L, int j) {
  int off = 0, span = L;
  for (int i = 0; i < j; ++i) {
    off += span;
    span /= P.radix[i];
  }
  return off;
}

// last forward pass, pointwise square and first inverse pass (a contiguous
// block of R words starting at a multiple of R: positions sw(off) + d)
template <int R>
__device__ __forceinline__ void task_square(uint64_t* base, int off) {
  uint64_t* p = base + sw(off);
  uint64_t v[R];
#pragma unroll
  for (int d = 0; d < R; ++d) v[d] = p[d];
  dif<R>(v);
#pragma unroll
  for (int d = 0; d < R; ++d) v[d] = gl::sqr(v[d]);
  dit_inv<R>(v);
#pragma unroll
  for (int d = 0; d < R; ++d) p[d] = v[d];
}

// last forward pass, pointwise product with a transformed operand f (the same
// positions of the same row, in HBM) and first inverse pass
template <int R>
__device__ __forceinline__ void task_mul(uint64_t* base, int off, const uint64_t* f) {
  uint64_t* p = base + sw(off);
  uint64_t v[R];
#pragma unroll
  for (int d = 0; d < R; ++d) v[d] = p[d];
  dif<R>(v);
#pragma unroll
  for (int d = 0; d < R; ++d) v[d] = gl::mul(v[d], f[off + d]);
  dit_inv<R>(v);
#pragma unroll
  for (int d = 0; d < R; ++d) p[d] = v[d];
}

template <int R, int Mode, bool Big>
__device__ __forceinline__ void pass_tasks(uint64_t* sm, int ld, int ntrans, int L, int span,
                                           const uint64_t* tw) {
  // all sizes are powers of two: index arithmetic by shifts and masks
  const int q = span / R, per = L / R, qs = q + (q >> 4);
  const int lq = __ffs(q) - 1, lper = __ffs(per) - 1;
  const int total = ntrans * per;
  for (int task = threadIdx.x; task < total; task += blockDim.x) {
    const int g = task >> lper, k = task & (per - 1);
    const int b = k >> lq, t = k & (q - 1);
    uint64_t* base = sm + g * ld;
    if constexpr (Mode == 0)
      task_dif<R, Big>(base, sw(b * span + t), q, qs, tw + t * R);
    else if constexpr (Mode == 1)
      task_dit<R, Big>(base, sw(b * span + t), q, qs, tw + t * R);
    else if constexpr (Mode == 2)
      task_square<R>(base, b * span);
    else
      task_mul<R>(base, b * span, tw + (size_t)g * L);
  }
}

// A pass over `ntrans` transforms of length L; transform g lives at sm + g * ld.
// tw: this pass's part of the pass table.
// Mode 0: DIF, 1: DIT, 2: square, 3: product with the transformed rows at tw
template <int R, int Mode>
__device__ void pass(uint64_t* sm, int ld, int ntrans, int L, int span, const uint64_t* tw) {
  if (span / R >= 16)
    pass_tasks<R, Mode, true>(sm, ld, ntrans, L, span, tw);
  else
    pass_tasks<R, Mode, false>(sm, ld, ntrans, L, span, tw);
}

// A pass of radix R (a power of two up to MR, the largest the kernel is built for).
template <int Mode, int MR = kMaxRadix>
__device__ __forceinline__ void pass_r(int R, uint64_t* sm, int ld, int ntrans, int L, int span,
                                       const uint64_t* tw) {
  switch (R) {
    case 2: pass<2, Mode>(sm, ld, ntrans, L, span, tw); break;
    case 4: pass<4, Mode>(sm, ld, ntrans, L, span, tw); break;
    case 8: pass<8, Mode>(sm, ld, ntrans, L, span, tw); break;
    default:
      if constexpr (MR >= 16) pass<16, Mode>(sm, ld, ntrans, L, span, tw);
      break;
  }
}

}  // namespace smem
}  // namespace lnt
