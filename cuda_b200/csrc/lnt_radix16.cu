// Two-pass squaring with register passes (smem_passes.cuh) for n = 2^13 ... 2^26.
//
// Same layout, twiddle tables and carry scheme as lnt_twopass.cu (which
// replaces the reference's FFT_2SMEM pool, kernel_pool.cu:39-48): columns of
// n2 words and rows of n1 words, transformed in shared memory; the result of
// the forward transform is in fully bit-reversed order, like the radix-2
// kernels, so all plans share the 4-step twiddle tables.
//
// row_square_r16: the first pass reads HBM directly (with the 4-step twiddle)
// and the last inverse pass writes HBM directly; the last forward pass, the
// pointwise square and the first inverse pass run in registers back to back.
#include <map>
#include <type_traits>
#include <mutex>
#include <utility>

#include "carry.cuh"
#include "lnt_internal.h"
#include "ntt_core.cuh"
#include "smem_passes.cuh"

namespace lnt {

namespace {

using namespace smem;

// ------------------------------------------------------------------ rows ----

// 256 threads per row of up to 4096 words (four CTAs per SM); longer rows hold
// one or two CTAs per SM, so their CTAs are wider to keep 32 warps per SM.
constexpr int row_threads_for(int L) { return L <= 4096 ? 256 : (L == 8192 ? 512 : 1024); }
// The squaring kernel's CTA for `rows` rows of L words: in a launch that fills
// the GPU, up to 4096 words take two radix-8 tasks per thread per pass (256
// threads for 4096 words, down to one warp); a launch of fewer CTAs than twice
// the SMs (latency) keeps 256; longer rows as row_threads_for.
constexpr int row_square_threads(int L, int rows, bool latency) {
  return L > 4096 ? row_threads_for(L)
                  : (L * rows >= 4096 || latency ? 256
                                                 : (L * rows >= 2048 ? 128 : (L * rows >= 1024 ? 64 : 32)));
}
#ifndef LNT_ROW_MIN_BLOCKS
#define LNT_ROW_MIN_BLOCKS 4  // CTAs per SM the row kernel is compiled for (registers)
#endif
// Radix-16 passes hold 16 values and their twiddles per thread: at the 64
// registers of four row CTAs (two 4-column CTAs) per SM they spill, so their
// kernels are built for half the CTAs per SM (128 registers, no spills).
template <int TH, int MR>
constexpr int row_min_blocks() {
  return TH == 256 ? (MR == 16 ? 2 : LNT_ROW_MIN_BLOCKS)
                   : ((MR == 16 ? 512 : 1024) / TH > 0 ? (MR == 16 ? 512 : 1024) / TH : 1);
}

// Forward pass of `rows` row transforms.  The first pass (span = L) reads HBM
// and applies the 4-step twiddle; later passes read shared memory.  One code
// body serves both, which keeps the kernel small for the instruction cache.
template <int R, bool Big>
__device__ __forceinline__ void row_dif_tasks(uint64_t* sm, int ld, int rows, int L, int span,
                                              const uint64_t* x, const uint64_t* twf,
                                              const uint64_t* twL) {
  const bool first = span == L;
  const int q = span / R, per = L / R, qs = q + (q >> 4);
  const int lq = __ffs(q) - 1, lper = __ffs(per) - 1;
  for (int task = threadIdx.x; task < rows * per; task += blockDim.x) {
    const int g = task >> lper, k = task & (per - 1), b = k >> lq, t = k & (q - 1);
    const int off = b * span + t, b0 = sw(off);
    uint64_t* base = sm + g * ld;
    uint64_t v[R];
    if (first) {
      const size_t rb = (size_t)g * L + off;
#pragma unroll
      for (int d = 0; d < R; ++d) v[d] = gl::mul(x[rb + q * d], twf[rb + q * d]);
    } else {
#pragma unroll
      for (int d = 0; d < R; ++d) v[d] = base[task_pos<Big>(b0, q, qs, d)];
    }
    dif<R>(v);
    if (q > 1) mul_task_twiddles<R>(v, twL + t * R);
#pragma unroll
    for (int r = 0; r < R; ++r) base[task_pos<Big>(b0, q, qs, r)] = v[r];
  }
}

// Inverse pass; the last one (span = L) applies the inverse 4-step twiddle and
// writes HBM.
template <int R, bool Big>
__device__ __forceinline__ void row_dit_tasks(uint64_t* sm, int ld, int rows, int L, int span,
                                              uint64_t* x, const uint64_t* twi, const uint64_t* itwL) {
  const bool last = span == L;
  const int q = span / R, per = L / R, qs = q + (q >> 4);
  const int lq = __ffs(q) - 1, lper = __ffs(per) - 1;
  for (int task = threadIdx.x; task < rows * per; task += blockDim.x) {
    const int g = task >> lper, k = task & (per - 1), b = k >> lq, t = k & (q - 1);
    const int off = b * span + t, b0 = sw(off);
    uint64_t* base = sm + g * ld;
    uint64_t v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = base[task_pos<Big>(b0, q, qs, r)];
    if (q > 1) mul_task_twiddles<R>(v, itwL + t * R);
    dit_inv<R>(v);
    if (last) {
      const size_t rb = (size_t)g * L + off;
#pragma unroll
      for (int d = 0; d < R; ++d) x[rb + q * d] = gl::mul(v[d], twi[rb + q * d]);
    } else {
#pragma unroll
      for (int d = 0; d < R; ++d) base[task_pos<Big>(b0, q, qs, d)] = v[d];
    }
  }
}

#ifndef LNT_ROW_STRIDED
#define LNT_ROW_STRIDED 1
#endif

template <int R>
__device__ void row_dif_pass(uint64_t* sm, int ld, int rows, int L, int span, const uint64_t* x,
                             const uint64_t* twf, const uint64_t* twL) {
  if (LNT_ROW_STRIDED && span / R >= 16)
    row_dif_tasks<R, true>(sm, ld, rows, L, span, x, twf, twL);
  else
    row_dif_tasks<R, false>(sm, ld, rows, L, span, x, twf, twL);
}

template <int R>
__device__ void row_dit_pass(uint64_t* sm, int ld, int rows, int L, int span, uint64_t* x,
                             const uint64_t* twi, const uint64_t* itwL) {
  if (LNT_ROW_STRIDED && span / R >= 16)
    row_dit_tasks<R, true>(sm, ld, rows, L, span, x, twi, itwL);
  else
    row_dit_tasks<R, false>(sm, ld, rows, L, span, x, twi, itwL);
}

template <bool Forward, int MR>
__device__ __forceinline__ void row_pass_r(int R, uint64_t* sm, int ld, int rows, int L, int span,
                                           uint64_t* x, const uint64_t* tw4, const uint64_t* twL) {
  switch (R) {
    case 2:
      if constexpr (Forward) row_dif_pass<2>(sm, ld, rows, L, span, x, tw4, twL);
      else row_dit_pass<2>(sm, ld, rows, L, span, x, tw4, twL);
      break;
    case 4:
      if constexpr (Forward) row_dif_pass<4>(sm, ld, rows, L, span, x, tw4, twL);
      else row_dit_pass<4>(sm, ld, rows, L, span, x, tw4, twL);
      break;
    case 8:
      if constexpr (Forward) row_dif_pass<8>(sm, ld, rows, L, span, x, tw4, twL);
      else row_dit_pass<8>(sm, ld, rows, L, span, x, tw4, twL);
      break;
    default:
      if constexpr (MR >= 16) {
        if constexpr (Forward) row_dif_pass<16>(sm, ld, rows, L, span, x, tw4, twL);
        else row_dit_pass<16>(sm, ld, rows, L, span, x, tw4, twL);
      }
      break;
  }
}

template <int TH, int MR>
__global__ void __launch_bounds__(TH, row_min_blocks<TH, MR>()) row_square_r16(const TwoPassDesc* __restrict__ Ds, Passes P, int rows) {
  extern __shared__ __align__(16) uint64_t sm[];
  const TwoPassDesc& D = Ds[blockIdx.y];
  const int L = (int)D.n1, ld = padded(L);
  const size_t off = (size_t)blockIdx.x * rows * L;
  uint64_t* x = reinterpret_cast<uint64_t*>(D.x) + off;
  int span = L;
  for (int j = 0, seg = 0; j + 1 < P.m; ++j) {
    row_pass_r<true, MR>(P.radix[j], sm, ld, rows, L, span, x, D.twf + off, D.itw1 + seg);
    seg += span;
    span /= P.radix[j];
    __syncthreads();
  }
  pass_r<2, MR>(P.radix[P.m - 1], sm, ld, rows, L, span, nullptr);
  __syncthreads();
  for (int j = P.m - 2; j >= 0; --j) {
    span *= P.radix[j];
    row_pass_r<false, MR>(P.radix[j], sm, ld, rows, L, span, x, D.twi + off,
                      D.iitw1 + pass_table_offset(P, L, j));
    if (j) __syncthreads();
  }
}

// Forward row transforms only (the first half of row_square_r16): the rows
// after all forward passes, in the order the passes leave them, go back to x.
// With col_forward before it this is the full transform of a residue, the
// operand of a product (row_mul_r16).
template <int TH, int MR>
__global__ void __launch_bounds__(TH) row_forward_r16(const TwoPassDesc* __restrict__ Ds, Passes P, int rows) {
  extern __shared__ __align__(16) uint64_t sm[];
  const TwoPassDesc& D = Ds[blockIdx.y];
  const int L = (int)D.n1, ld = padded(L);
  const size_t off = (size_t)blockIdx.x * rows * L;
  uint64_t* x = reinterpret_cast<uint64_t*>(D.x) + off;
  int span = L;
  for (int j = 0, seg = 0; j < P.m; ++j) {
    row_pass_r<true, MR>(P.radix[j], sm, ld, rows, L, span, x, D.twf + off, D.itw1 + seg);
    seg += span;
    span /= P.radix[j];
    __syncthreads();
  }
  for (int i = threadIdx.x; i < rows * L; i += TH) {
    const int g = i / L, k = i - g * L;
    x[i] = sm[g * ld + sw(k)];
  }
}

// row_square_r16 with the pointwise square replaced by the product with the
// transformed rows F of another residue (row_forward_r16's output).
template <int TH, int MR>
__global__ void __launch_bounds__(TH) row_mul_r16(const TwoPassDesc* __restrict__ Ds, Passes P, int rows,
                                                  const uint64_t* __restrict__ F) {
  extern __shared__ __align__(16) uint64_t sm[];
  const TwoPassDesc& D = Ds[blockIdx.y];
  const int L = (int)D.n1, ld = padded(L);
  const size_t off = (size_t)blockIdx.x * rows * L;
  uint64_t* x = reinterpret_cast<uint64_t*>(D.x) + off;
  int span = L;
  for (int j = 0, seg = 0; j + 1 < P.m; ++j) {
    row_pass_r<true, MR>(P.radix[j], sm, ld, rows, L, span, x, D.twf + off, D.itw1 + seg);
    seg += span;
    span /= P.radix[j];
    __syncthreads();
  }
  pass_r<3, MR>(P.radix[P.m - 1], sm, ld, rows, L, span, F + off);
  __syncthreads();
  for (int j = P.m - 2; j >= 0; --j) {
    span *= P.radix[j];
    row_pass_r<false, MR>(P.radix[j], sm, ld, rows, L, span, x, D.twi + off,
                      D.iitw1 + pass_table_offset(P, L, j));
    if (j) __syncthreads();
  }
}

// ------------------------------------------------------- rows of 5 L ----
//
// n = 5 * 2^k: a row holds n1 = 5 L words z[c'], c' = c + L j5.  Its transform
// (root omega_{5L} = omega_n^n2) splits as
//   Z[5 kL + k5] = sum_c omega_L^(c kL) omega_{5L}^(c k5) sum_j5 omega_5^(j5 k5) z[c + L j5]:
// a 5-point transform of the five words c, c + L, ..., c + 4L (fused with the
// 4-step twiddle as the row is loaded), a twiddle, and an L-point transform of
// each of the five planes (the passes above, bit-reversed output), whose last
// pass runs with the square as in row_square_r16.  The inverse runs the same
// steps backwards and stores the row; its factor 1/5 is in the unweights (1/n).

// 5-point transform with the pair form u1 w^k + u4 w^-k = a C + b S (a = u1 + u4,
// b = u1 - u4, C = (w^k + w^-k)/2, S = (w^k - w^-k)/2; likewise u2, u3 with w^2k):
// eight multiplications instead of sixteen.  c = {C1, C2, S1, S2}.  The inverse
// transform (w^-1) is the same with outputs 1, 4 and 2, 3 exchanged.
__device__ __forceinline__ void dft5(uint64_t (&u)[5], const uint64_t* c) {
  const uint64_t a1 = gl::add(u[1], u[4]), b1 = gl::sub(u[1], u[4]);
  const uint64_t a2 = gl::add(u[2], u[3]), b2 = gl::sub(u[2], u[3]);
  const uint64_t t1 = gl::add(gl::mul(a1, c[0]), gl::mul(a2, c[1]));
  const uint64_t t2 = gl::add(gl::mul(a1, c[1]), gl::mul(a2, c[0]));
  const uint64_t s1 = gl::add(gl::mul(b1, c[2]), gl::mul(b2, c[3]));
  const uint64_t s2 = gl::sub(gl::mul(b1, c[3]), gl::mul(b2, c[2]));
  const uint64_t u0 = u[0];
  u[0] = gl::add(u0, gl::add(a1, a2));
  const uint64_t p1 = gl::add(u0, t1), p2 = gl::add(u0, t2);
  u[1] = gl::add(p1, s1);
  u[4] = gl::sub(p1, s1);
  u[2] = gl::add(p2, s2);
  u[3] = gl::sub(p2, s2);
}

// Mode 0: square (a squaring), 1: forward only (the operand F of a product,
// left in x in plane-major order), 2: product with F.  A CTA takes `rows`
// consecutive rows: plane k5 of row g at sm + (5 g + k5) ld.
template <int TH, int MR, int Mode>
__global__ void __launch_bounds__(TH) row5_r16(const TwoPassDesc* __restrict__ Ds, Passes P, int rows,
                                               const uint64_t* __restrict__ F) {
  extern __shared__ __align__(16) uint64_t sm[];
  const TwoPassDesc& D = Ds[blockIdx.y];
  const int L = (int)D.n1 / 5, ld = padded(L), W = 5 * L, lL = __ffs(L) - 1;
  const size_t off = (size_t)blockIdx.x * rows * W;
  uint64_t* x = reinterpret_cast<uint64_t*>(D.x) + off;
  const uint64_t* twf = D.twf + off;
  uint64_t c5[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) c5[k] = D.c5[k];
  // HBM -> planes: 4-step twiddle, 5-point transform, twiddle omega_5L^(c k5)
  for (int item = threadIdx.x; item < rows * L; item += TH) {
    const int g = item >> lL, c = item & (L - 1);
    const int i0 = g * W + c;
    uint64_t u[5];
#pragma unroll
    for (int j5 = 0; j5 < 5; ++j5) u[j5] = gl::mul(x[i0 + j5 * L], twf[i0 + j5 * L]);
    dft5(u, c5);
    uint64_t* base = sm + 5 * g * ld + sw(c);
    base[0] = u[0];
#pragma unroll
    for (int k5 = 1; k5 < 5; ++k5) base[k5 * ld] = gl::mul(u[k5], D.tw5[(k5 - 1) * L + c]);
  }
  __syncthreads();
  int span = L;
  const int last = Mode == 1 ? P.m : P.m - 1;
  for (int j = 0, seg = 0; j < last; ++j) {
    pass_r<0, MR>(P.radix[j], sm, ld, 5 * rows, L, span, D.itw1 + seg);
    seg += span;
    span /= P.radix[j];
    __syncthreads();
  }
  if constexpr (Mode == 1) {
    for (int i = threadIdx.x; i < rows * W; i += TH) {
      const int p = i >> lL, e = i & (L - 1);
      x[i] = sm[p * ld + sw(e)];
    }
  } else {
    // last forward pass, square (or product with F) and first inverse pass
    if constexpr (Mode == 0)
      pass_r<2, MR>(P.radix[P.m - 1], sm, ld, 5 * rows, L, span, nullptr);
    else
      pass_r<3, MR>(P.radix[P.m - 1], sm, ld, 5 * rows, L, span, F + off);
    __syncthreads();
    for (int j = P.m - 2; j >= 0; --j) {
      span *= P.radix[j];
      pass_r<1, MR>(P.radix[j], sm, ld, 5 * rows, L, span, D.iitw1 + pass_table_offset(P, L, j));
      __syncthreads();
    }
    // planes -> HBM: inverse twiddle, inverse 5-point transform, inverse 4-step twiddle
    const uint64_t* twi = D.twi + off;
    for (int item = threadIdx.x; item < rows * L; item += TH) {
      const int g = item >> lL, c = item & (L - 1);
      const int i0 = g * W + c;
      const uint64_t* base = sm + 5 * g * ld + sw(c);
      uint64_t u[5];
      u[0] = base[0];
#pragma unroll
      for (int k5 = 1; k5 < 5; ++k5) u[k5] = gl::mul(base[k5 * ld], D.itw5[(k5 - 1) * L + c]);
      dft5(u, c5);
      x[i0] = gl::mul(u[0], twi[i0]);
      x[i0 + L] = gl::mul(u[4], twi[i0 + L]);
      x[i0 + 2 * L] = gl::mul(u[3], twi[i0 + 2 * L]);
      x[i0 + 3 * L] = gl::mul(u[2], twi[i0 + 3 * L]);
      x[i0 + 4 * L] = gl::mul(u[1], twi[i0 + 4 * L]);
    }
  }
}

// --------------------------------------------------------------- columns ----

// Threads per tile column.  A launch with CTAs enough to fill the GPU
// (throughput: a batch) gives each column one thread per radix-8 task of a pass
// (n2 / 8), at least a warp and at most 128, or 256 for columns of 4096 words
// (one 4-column CTA per SM): short columns then get small CTAs, many per SM,
// instead of CTAs whose threads mostly idle.  A launch with fewer CTAs than
// twice the SMs (one short test: latency) keeps 128 threads a column, whose
// row-wise steps (carries, weights, staging) then run in parallel.
__host__ __device__ constexpr int col_tpc(uint32_t n2, bool latency) {
  return n2 >= 4096 ? 256 : (n2 >= 1024 || latency ? 128 : (n2 == 512 ? 64 : 32));
}
inline bool col_latency_mode(const TwoPassDesc& d, uint32_t count) {
  return (uint64_t)d.ntiles * count < 2ull * device_sms();
}
// CTAs per SM the column kernels are compiled for: 64 registers a thread at
// 1024 threads an SM (128 for radix-16 passes, which spill at 64)
template <int TH, int MR>
constexpr int col_min_blocks() { return (MR == 16 ? 512 : 1024) / TH > 0 ? (MR == 16 ? 512 : 1024) / TH : 1; }

// column stride in words: the coalesced staging (lanes = T columns x 32/T
// rows) then hits distinct banks
__host__ __device__ constexpr int col_ld(int L, int T) {
  return ((padded(L) + 15) / 16) * 16 + (T >= 16 ? 1 : 16 / T);
}

// HBM -> shared memory without a register round trip: every word is an
// 8-byte cp.async, so all of a thread's loads are in flight together.
__device__ __forceinline__ void tile_load(uint64_t* sm, int ld, const int64_t* x, int L, int T,
                                          uint32_t n1, uint32_t c0) {
  const int rs = blockDim.x / T;  // rows per round
  if (blockDim.x % T == 0 && rs % 16 == 0) {
    // fixed column per thread, rows a constant stride apart: both addresses
    // advance by a constant (sw(r + rs) = sw(r) + rs + rs / 16)
    const int c = threadIdx.x % T, r0 = threadIdx.x / T;
    const int64_t* src = x + (size_t)r0 * n1 + c0 + c;
    uint32_t dst = (uint32_t)__cvta_generic_to_shared(sm + c * ld + sw(r0));
    const size_t src_step = (size_t)rs * n1;
    const uint32_t dst_step = (uint32_t)(rs + rs / 16) * 8;
    for (int r = r0; r < L; r += rs, src += src_step, dst += dst_step)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
  } else {
    for (int idx = threadIdx.x; idx < T * L; idx += blockDim.x) {
      const int r = idx / T, c = idx % T;
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(sm + c * ld + sw(r));
      const int64_t* src = x + (size_t)r * n1 + c0 + c;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// HBM -> shared memory through L2 only (ld.global.cg): for a tile another CTA
// of the same launch has just written.
__device__ __forceinline__ void tile_load_cg(uint64_t* sm, int ld, const int64_t* x, int L, int T,
                                             uint32_t n1, uint32_t c0) {
  for (int idx = threadIdx.x; idx < T * L; idx += blockDim.x) {
    const int r = idx / T, c = idx % T;
    sm[c * ld + sw(r)] = (uint64_t)__ldcg(x + (size_t)r * n1 + c0 + c);
  }
}

// shared memory -> HBM: as tile_load, four rounds per loop iteration so the
// shared-memory reads overlap
__device__ __forceinline__ void tile_store(const uint64_t* sm, int ld, int64_t* x, int L, int T,
                                           uint32_t n1, uint32_t c0) {
  const int rs = blockDim.x / T;
  if (blockDim.x % T == 0 && rs % 16 == 0 && L % (4 * rs) == 0) {
    const int c = threadIdx.x % T, r0 = threadIdx.x / T;
    int64_t* dst = x + (size_t)r0 * n1 + c0 + c;
    const uint64_t* src = sm + c * ld + sw(r0);
    const size_t dst_step = (size_t)rs * n1;
    const int src_step = rs + rs / 16;
    for (int r = r0; r < L; r += 4 * rs, dst += 4 * dst_step, src += 4 * src_step) {
      const uint64_t v0 = src[0], v1 = src[src_step], v2 = src[2 * src_step], v3 = src[3 * src_step];
      dst[0] = (int64_t)v0;
      dst[dst_step] = (int64_t)v1;
      dst[2 * dst_step] = (int64_t)v2;
      dst[3 * dst_step] = (int64_t)v3;
    }
    return;
  }
  for (int idx = threadIdx.x; idx < T * L; idx += blockDim.x)
    x[(size_t)(idx / T) * n1 + c0 + idx % T] = (int64_t)sm[(idx % T) * ld + sw(idx / T)];
}

// A row's run of T table entries, read as 16-byte vectors (tile-major tables:
// the run is contiguous and consecutive rows are adjacent, so a warp's loads
// are coalesced).
template <int T>
__device__ __forceinline__ void load_run(const uint64_t* src, uint64_t (&out)[T]) {
  const ulonglong2* v = reinterpret_cast<const ulonglong2*>(src);
#pragma unroll
  for (int k = 0; k < T / 2; ++k) {
    const ulonglong2 u = v[k];
    out[2 * k] = u.x;
    out[2 * k + 1] = u.y;
  }
}

template <int T>
__device__ __forceinline__ void load_widths(const uint8_t* src, unsigned (&out)[T]) {
  if constexpr (T == 8) {
    const uint64_t u = *reinterpret_cast<const uint64_t*>(src);
#pragma unroll
    for (int c = 0; c < 8; ++c) out[c] = (unsigned)((u >> (8 * c)) & 0xFF);
  } else {
    const uint32_t u = *reinterpret_cast<const uint32_t*>(src);
#pragma unroll
    for (int c = 0; c < 4; ++c) out[c] = (u >> (8 * c)) & 0xFF;
  }
}

// ---- column tile bodies: tile t0 (T columns x L rows) staged in shared memory

// Carry-in from the run before each row's run, weight, forward column passes,
// store.  The tile's digits are in `sm`.  `cg_carries`: read the carries from L2
// (written by another CTA of the same launch).
template <int T, int MR>
__device__ __forceinline__ void forward_tile(const TwoPassDesc& D, const Passes& P, uint64_t* sm,
                                             int ld, uint32_t t0, bool apply_carries, bool cg_carries,
                                             uint32_t& status) {
  const int L = (int)D.n2;
  // per row: carry from the previous run, then weight (balanced digit -> field)
  for (int r = threadIdx.x; r < L; r += blockDim.x) {
    const size_t run = (size_t)t0 * L + r;
    uint64_t w[T];
    unsigned wd[T];
    load_run<T>(D.wt + run * T, w);
    load_widths<T>(D.widt + run * T, wd);
    int64_t carry = 0;
    if (apply_carries) {
      const int64_t* src = D.carry + (t0 > 0 ? run - L : (size_t)(D.ntiles - 1) * L + (r ? r - 1 : L - 1));
      carry = cg_carries ? __ldcg(src) : *src;
    }
#pragma unroll
    for (int c = 0; c < T; ++c) {
      uint64_t& v = sm[c * ld + sw(r)];
      int64_t d = (int64_t)v;
      if (carry != 0) {
        if (c + 1 < T) {
          int64_t q;
          d = balance(d + carry, wd[c], q);
          carry = q;
        } else {
          d += carry;
          if (carry > kAbsorbLimit || carry < -kAbsorbLimit) status |= kStatusCarryOverflow;
          carry = 0;
        }
      }
      v = gl::mul_digit(d, w[c]);
    }
  }
  __syncthreads();
  int span = L;
  for (int j = 0, seg = 0; j < P.m; ++j) {
    pass_r<0, MR>(P.radix[j], sm, ld, T, L, span, D.itw2 + seg);
    __syncthreads();
    seg += span;
    span /= P.radix[j];
  }
  tile_store(sm, ld, D.x, L, T, D.n1, t0 * T);
}

// Inverse column passes, unweight, carry each row's run of T words to balanced
// digits (minus two in the run of word 0), store the runs' outgoing carries.
// The tile's transform is in `sm`; its digits are left there.
template <int T, int MR>
__device__ __forceinline__ void inverse_tile(const TwoPassDesc& D, const Passes& P, uint64_t* sm,
                                             int ld, uint32_t t0, bool unsigned_mode) {
  const int L = (int)D.n2;
  int span = 1;
  for (int j = P.m - 1; j >= 0; --j) {
    span *= P.radix[j];
    pass_r<1, MR>(P.radix[j], sm, ld, T, L, span, D.iitw2 + pass_table_offset(P, L, j));
    __syncthreads();
  }
  for (int r = threadIdx.x; r < L; r += blockDim.x) {
    const size_t run = (size_t)t0 * L + r;
    uint64_t uw[T];
    unsigned wd[T];
    load_run<T>(D.uwt + run * T, uw);
    load_widths<T>(D.widt + run * T, wd);
    int64_t carry = (!D.prp && t0 == 0 && r == 0) ? -2 : 0;
#pragma unroll
    for (int c = 0; c < T; ++c) {
      uint64_t& v = sm[c * ld + sw(r)];
      v = (uint64_t)carry_digit(gl::mul(v, uw[c]), unsigned_mode, carry, wd[c], carry);
    }
    D.carry[run] = carry;
  }
  __syncthreads();
}

template <int T, int TH, int MR>
__global__ void __launch_bounds__(TH, col_min_blocks<TH, MR>()) col_forward_r16(
    const TwoPassDesc* __restrict__ Ds, Passes P, int apply_carries) {
  extern __shared__ __align__(16) uint64_t sm[];
  const TwoPassDesc& D = Ds[blockIdx.y];
  const int ld = col_ld((int)D.n2, T);
  uint32_t status = 0;
  tile_load(sm, ld, D.x, (int)D.n2, T, D.n1, blockIdx.x * T);
  __syncthreads();
  forward_tile<T, MR>(D, P, sm, ld, blockIdx.x, apply_carries != 0, false, status);
  if (status) atomicOr(D.status, status);
}

template <int T, int TH, int MR>
__global__ void __launch_bounds__(TH, col_min_blocks<TH, MR>()) col_inverse_r16(
    const TwoPassDesc* __restrict__ Ds, Passes P, int unsigned_mode) {
  extern __shared__ __align__(16) uint64_t sm[];
  const TwoPassDesc& D = Ds[blockIdx.y];
  const int ld = col_ld((int)D.n2, T);
  tile_load(sm, ld, D.x, (int)D.n2, T, D.n1, blockIdx.x * T);
  __syncthreads();
  inverse_tile<T, MR>(D, P, sm, ld, blockIdx.x, unsigned_mode != 0);
  tile_store(sm, ld, D.x, (int)D.n2, T, D.n1, blockIdx.x * T);
}

// ---- carry-fused column kernel: col_inverse of one squaring and col_forward
// of the next in one launch, the tile staying in shared memory in between.
//
// A tile's second half needs the carries of the tile before it (the runs of
// the same rows); tile 0 needs those of the LAST tile (the runs of the rows
// before).  CTAs take tickets in start order (an atomic counter) and no CTA
// ever waits for a CTA that took a later ticket, so every wait ends whatever
// else holds the GPU's CTA slots (other tests, other launches):
//   ticket 0:          first half of the last tile (its digits go back to x,
//                      flag), first half of tile 0 (flag), then tile 0's
//                      second half with the last tile's carries it has just
//                      made itself;
//   ticket t, 0<t<T-1: first half of tile t (flag), wait for tile t-1's flag,
//                      second half;
//   ticket T-1:        wait for the last tile's flag (ticket 0 has stored its
//                      digits) and tile T-2's flag, reload the digits, second
//                      half.
// Flags hold a per-launch epoch, so nothing is cleared between launches.  Every
// wait is bounded in time and reported.
//
// fuse[0]: ticket counter, fuse[1]: epoch, fuse[2 + t]: flag of tile t.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s: far above any launch; then report, never hang

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void publish_flag(uint32_t* flag, uint32_t v) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(flag), "r"(v) : "memory");
  }
}

// Thread 0 polls the flag (acquire), the CTA waits at the barrier.  Gives up
// after kWaitLimitNs, or at once when another CTA already gave up.
__device__ __forceinline__ void wait_flag(const uint32_t* flag, uint32_t want, uint32_t* status) {
  if (threadIdx.x == 0) {
    const uint64_t start = global_ns();
    uint32_t v = 0, iters = 0;
    while (true) {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
      if (v == want) break;
      if ((++iters & 63) == 0) {
        if (*(volatile uint32_t*)status & kStatusFuseTimeout) break;
        if (global_ns() - start > kWaitLimitNs) {
          atomicOr(status, kStatusFuseTimeout);
          break;
        }
      }
      __nanosleep(100);
    }
  }
  __syncthreads();
}

template <int T, int TH, int MR>
__global__ void __launch_bounds__(TH, col_min_blocks<TH, MR>()) col_fused_r16(
    const TwoPassDesc* __restrict__ Ds, Passes P) {
  extern __shared__ __align__(16) uint64_t sm[];
  __shared__ uint32_t s_ticket, s_epoch;
  const TwoPassDesc& D = Ds[blockIdx.y];
  const int L = (int)D.n2, ld = col_ld(L, T);
  const uint32_t n1 = D.n1, ntiles = D.ntiles, last = ntiles - 1;
  uint32_t* ctl = D.fuse;
  if (threadIdx.x == 0) {
    // the epoch is read before the ticket: the last ticket's CTA advances it
    // only after every CTA of the launch has taken its ticket
    uint32_t e;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(e) : "l"(ctl + 1) : "memory");
    s_epoch = e;
    s_ticket = atomicAdd(ctl, 1u);
  }
  __syncthreads();
  const uint32_t ticket = s_ticket, ready = s_epoch + 1;
  if (ticket >= ntiles || ntiles < 2) {  // a counter left over from a launch that did not finish: report, touch nothing
    if (threadIdx.x == 0) atomicOr(D.status, kStatusFuseTimeout);
    return;
  }
  uint32_t status = 0;
  const bool is_last = ticket == last;

  // first halves, each inverse_tile / forward_tile body instantiated once (the
  // kernel stays small for the instruction cache): ticket 0 does the last
  // tile's and then tile 0's, ticket t < T-1 its own, ticket T-1 none
  const int ninv = is_last ? 0 : (ticket == 0 ? 2 : 1);
  for (int i = 0; i < ninv; ++i) {
    const bool lasttile = ticket == 0 && i == 0;
    const uint32_t tile = lasttile ? last : ticket;
    tile_load(sm, ld, D.x, L, T, n1, tile * T);
    __syncthreads();
    inverse_tile<T, MR>(D, P, sm, ld, tile, false);
    // the last tile's digits wait in x for the last ticket
    if (lasttile) tile_store(sm, ld, D.x, L, T, n1, last * T);
    publish_flag(ctl + 2 + tile, ready);
  }
  if (is_last) {
    // the last tile's first half was done by ticket 0 (digits in x)
    wait_flag(ctl + 2 + last, ready, D.status);
    tile_load_cg(sm, ld, D.x, L, T, n1, last * T);
  }
  // second half: carries in from the tile before (tile 0: the last tile, made
  // by this CTA), weight, forward column transform
  if (ticket > 0) wait_flag(ctl + 2 + ticket - 1, ready, D.status);
  forward_tile<T, MR>(D, P, sm, ld, ticket, true, true, status);
  if (is_last && threadIdx.x == 0) {
    // every ticket of this launch is taken and every CTA has read the epoch
    ctl[0] = 0;
    __threadfence();
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(ctl + 1), "r"(ready) : "memory");
  }
  if (status) atomicOr(D.status, status);
}

// Raise a kernel's dynamic shared-memory cap once per device (the cap does not
// change occupancy; the launch's own size does), so launches made while a
// stream is being captured into a graph issue no attribute calls.
template <typename K>
cudaError_t ensure_smem(K* kernel, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair((const void*)kernel, dev);
  auto it = done.find(key);
  if (it != done.end() && it->second >= smem) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) done[key] = smem;
  return e;
}

// Rows per row-kernel CTA: up to 4096 words of rows (the CTA's 256 threads
// then have two tasks each per pass), fewer while the launch would have fewer
// CTAs than the GPU has SMs (one test: latency) or than four per SM (a batch
// of `count` tests: throughput).
int row_rows_per_cta(int L, int n2, uint32_t count) {
  int rows = 4096 / L;
  if (rows < 1) rows = 1;
  const int sms = (int)device_sms();
  const long want = count > 1 ? 4L * sms : sms;
  while (rows > 1 && (long)(n2 / rows) * (long)count < want) rows /= 2;
  return rows;
}

}  // namespace

std::vector<uint32_t> r16_pass_radices(uint32_t log2L, uint32_t radix) {
  const Passes p = make_passes((int)log2L, radix == 16 ? 4 : 3);
  std::vector<uint32_t> r;
  for (int j = 0; j < p.m; ++j) r.push_back((uint32_t)p.radix[j]);
  return r;
}

// Rows up to 2^14 words (139 KB of shared memory, one CTA per SM) and columns
// up to 2^12 (four columns: 139 KB): with B200's 227 KB per CTA the 2^25 and
// 2^26 lengths stay two-pass, where the reference needs 3-factor plans
// (ntt_lengths.cu:118-127).
bool r16_supported(uint32_t log2n1, uint32_t log2n2) {
  return log2n2 >= 6 && log2n2 <= 12 && log2n1 >= 7 && log2n1 <= 14 && log2n1 >= log2n2;
}

uint32_t r16_tile(uint32_t log2n2) { return log2n2 >= 12 ? 4 : 8; }

// Words a carry run needs: the outgoing carry of a run is below 2^(log2 n + W)
// in magnitude (W = ceil(q / n)), each word it ripples through takes off at
// least w_min - 1 bits, and the last word absorbs the remaining +-1.
uint32_t r16_run_words_needed(uint32_t exponent, uint32_t n) {
  uint32_t log2n = 0;
  while ((1ull << log2n) < n) ++log2n;
  const uint32_t wmax = (exponent + n - 1) / n, wmin = exponent / n;
  if (wmin < 3) return 64;
  return (log2n + wmax + wmin - 2) / (wmin - 1) + 1;
}

// log2 of the largest pass radix of a descriptor's plan (3: radix 8, 4: radix 16)
inline int radix_log2(const TwoPassDesc& d) { return d.radix == 16 ? 4 : 3; }

template <int TH, int MR>
cudaError_t row_square_t(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count, cudaStream_t s) {
  const int L = (int)d.n1, rows = row_rows_per_cta(L, (int)d.n2, count);
  const size_t smem = (size_t)rows * padded(L) * 8;
  cudaError_t e = ensure_smem(row_square_r16<TH, MR>, smem);
  if (e != cudaSuccess) return e;
  row_square_r16<TH, MR><<<dim3(d.n2 / rows, count), TH, smem, s>>>(
      dd, make_passes((int)d.log2n1, radix_log2(d)), rows);
  return cudaGetLastError();
}

template <int TH, int MR>
cudaError_t row_forward_t(const TwoPassDesc& d, const TwoPassDesc* dd, cudaStream_t s) {
  const int L = (int)d.n1, rows = row_rows_per_cta(L, (int)d.n2, 1);
  const size_t smem = (size_t)rows * padded(L) * 8;
  cudaError_t e = ensure_smem(row_forward_r16<TH, MR>, smem);
  if (e != cudaSuccess) return e;
  row_forward_r16<TH, MR><<<dim3(d.n2 / rows, 1), TH, smem, s>>>(
      dd, make_passes((int)d.log2n1, radix_log2(d)), rows);
  return cudaGetLastError();
}

template <int TH, int MR>
cudaError_t row_mul_t(const TwoPassDesc& d, const TwoPassDesc* dd, const uint64_t* F, cudaStream_t s) {
  const int L = (int)d.n1, rows = row_rows_per_cta(L, (int)d.n2, 1);
  const size_t smem = (size_t)rows * padded(L) * 8;
  cudaError_t e = ensure_smem(row_mul_r16<TH, MR>, smem);
  if (e != cudaSuccess) return e;
  row_mul_r16<TH, MR><<<dim3(d.n2 / rows, 1), TH, smem, s>>>(
      dd, make_passes((int)d.log2n1, radix_log2(d)), rows, F);
  return cudaGetLastError();
}

template <int MR>
cudaError_t row_forward_m(const TwoPassDesc& d, const TwoPassDesc* dd, cudaStream_t s) {
  switch (row_threads_for((int)d.n1)) {
    case 256: return row_forward_t<256, MR>(d, dd, s);
    case 512: return row_forward_t<512, MR>(d, dd, s);
    default: return row_forward_t<1024, MR>(d, dd, s);
  }
}

template <int MR>
cudaError_t row_mul_m(const TwoPassDesc& d, const TwoPassDesc* dd, const uint64_t* F, cudaStream_t s) {
  switch (row_threads_for((int)d.n1)) {
    case 256: return row_mul_t<256, MR>(d, dd, F, s);
    case 512: return row_mul_t<512, MR>(d, dd, F, s);
    default: return row_mul_t<1024, MR>(d, dd, F, s);
  }
}

template <int MR>
cudaError_t row_square_m(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count, cudaStream_t s) {
  const int rows = row_rows_per_cta((int)d.n1, (int)d.n2, count);
  const bool latency = (uint64_t)(d.n2 / rows) * count < 2ull * device_sms();
  switch (row_square_threads((int)d.n1, rows, latency)) {
    case 32: return row_square_t<32, MR>(d, dd, count, s);
    case 64: return row_square_t<64, MR>(d, dd, count, s);
    case 128: return row_square_t<128, MR>(d, dd, count, s);
    case 256: return row_square_t<256, MR>(d, dd, count, s);
    case 512: return row_square_t<512, MR>(d, dd, count, s);
    default: return row_square_t<1024, MR>(d, dd, count, s);
  }
}

// Rows of 5 L words (radix-8 passes) per CTA: as many as fit 4096 words (a
// power of two), fewer while the launch would have fewer CTAs than the SMs (one
// test) or than four per SM (a batch of `count`); 128 threads for up to 1280
// words a CTA, 256 up to 5120, then 512 and 1024.
template <int Mode>
cudaError_t row5_launch(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                        const uint64_t* F, cudaStream_t s) {
  const int L = (int)d.n1 / 5;
  int rows = 1;
  while (rows * 2 * (int)d.n1 <= 4096 && rows * 2 <= (int)d.n2) rows *= 2;
  const long want = count > 1 ? 4L * device_sms() : (long)device_sms();
  while (rows > 1 && (long)(d.n2 / rows) * (long)count < want) rows /= 2;
  const size_t smem = (size_t)5 * rows * padded(L) * 8;
  const Passes P = make_passes((int)d.log2n1, 3);
  const dim3 grid(d.n2 / rows, count);
  const int words = rows * (int)d.n1;
  auto go = [&](auto kernel, int th) {
    cudaError_t e = ensure_smem(kernel, smem);
    if (e != cudaSuccess) return e;
    kernel<<<grid, th, smem, s>>>(dd, P, rows, F);
    return cudaGetLastError();
  };
  if (words <= 1280) return go(row5_r16<128, 8, Mode>, 128);
  if (words <= 5120) return go(row5_r16<256, 8, Mode>, 256);
  if (words <= 10240) return go(row5_r16<512, 8, Mode>, 512);
  return go(row5_r16<1024, 8, Mode>, 1024);
}

cudaError_t launch_row_forward_r16(const TwoPassDesc& d, const TwoPassDesc* dd, cudaStream_t s) {
  if (d.five) return row5_launch<1>(d, dd, 1, nullptr, s);
  return d.radix == 16 ? row_forward_m<16>(d, dd, s) : row_forward_m<8>(d, dd, s);
}

cudaError_t launch_row_mul_r16(const TwoPassDesc& d, const TwoPassDesc* dd, const uint64_t* F,
                               cudaStream_t s) {
  if (d.five) return row5_launch<2>(d, dd, 1, F, s);
  return d.radix == 16 ? row_mul_m<16>(d, dd, F, s) : row_mul_m<8>(d, dd, F, s);
}

cudaError_t launch_row_square_r16(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                                  cudaStream_t s) {
  if (d.five) return row5_launch<0>(d, dd, count, nullptr, s);
  return d.radix == 16 ? row_square_m<16>(d, dd, count, s) : row_square_m<8>(d, dd, count, s);
}

// The column kernels' thread count for a tile of T columns of n2 words.
template <int T, class F>
cudaError_t col_dispatch(uint32_t n2, bool latency, F&& f) {
  switch (T * col_tpc(n2, latency)) {
    case 128:
      if constexpr (T == 4) return f(std::integral_constant<int, 128>{});
      break;
    case 256: return f(std::integral_constant<int, 256>{});
    case 512: return f(std::integral_constant<int, 512>{});
    case 1024: return f(std::integral_constant<int, 1024>{});
    default: break;
  }
  return cudaErrorInvalidConfiguration;
}
template <int T, int TH, int MR>
cudaError_t col_forward_t(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count, bool apply,
                          cudaStream_t s) {
  const size_t smem = (size_t)T * col_ld((int)d.n2, T) * 8;
  cudaError_t e = ensure_smem(col_forward_r16<T, TH, MR>, smem);
  if (e != cudaSuccess) return e;
  col_forward_r16<T, TH, MR><<<dim3(d.ntiles, count), TH, smem, s>>>(
      dd, make_passes((int)d.log2n2, radix_log2(d)), apply ? 1 : 0);
  return cudaGetLastError();
}

template <int T, int TH, int MR>
cudaError_t col_inverse_t(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                          bool unsigned_mode, cudaStream_t s) {
  const size_t smem = (size_t)T * col_ld((int)d.n2, T) * 8;
  cudaError_t e = ensure_smem(col_inverse_r16<T, TH, MR>, smem);
  if (e != cudaSuccess) return e;
  col_inverse_r16<T, TH, MR><<<dim3(d.ntiles, count), TH, smem, s>>>(
      dd, make_passes((int)d.log2n2, radix_log2(d)), unsigned_mode ? 1 : 0);
  return cudaGetLastError();
}

template <int T, int TH, int MR>
cudaError_t col_fused_t(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count, cudaStream_t s) {
  const size_t smem = (size_t)T * col_ld((int)d.n2, T) * 8;
  cudaError_t e = ensure_smem(col_fused_r16<T, TH, MR>, smem);
  if (e != cudaSuccess) return e;
  col_fused_r16<T, TH, MR><<<dim3(d.ntiles, count), TH, smem, s>>>(
      dd, make_passes((int)d.log2n2, radix_log2(d)));
  return cudaGetLastError();
}

// Tests per launch (the grid's y extent).  A CTA of the fused kernel waits only
// for CTAs that started before it, so the count is not bounded by how many
// CTAs the GPU holds at once.
constexpr uint32_t kFusedTestsPerLaunch = 1024;

template <int T, int MR>
cudaError_t col_fused_tm(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count, cudaStream_t s) {
  return col_dispatch<T>(d.n2, col_latency_mode(d, count),
                         [&](auto th) { return col_fused_t<T, decltype(th)::value, MR>(d, dd, count, s); });
}

template <int MR>
cudaError_t col_fused_m(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count, cudaStream_t s) {
  for (uint32_t first = 0; first < count; first += kFusedTestsPerLaunch) {
    const uint32_t c = count - first < kFusedTestsPerLaunch ? count - first : kFusedTestsPerLaunch;
    const cudaError_t e = d.tile == 8 ? col_fused_tm<8, MR>(d, dd + first, c, s)
                                      : col_fused_tm<4, MR>(d, dd + first, c, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <int MR>
cudaError_t col_forward_m(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count, bool apply,
                          cudaStream_t s) {
  const bool latency = col_latency_mode(d, count);
  if (d.tile == 8)
    return col_dispatch<8>(d.n2, latency,
                           [&](auto th) { return col_forward_t<8, decltype(th)::value, MR>(d, dd, count, apply, s); });
  return col_dispatch<4>(d.n2, latency,
                         [&](auto th) { return col_forward_t<4, decltype(th)::value, MR>(d, dd, count, apply, s); });
}

template <int MR>
cudaError_t col_inverse_m(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                          bool unsigned_mode, cudaStream_t s) {
  const bool latency = col_latency_mode(d, count);
  if (d.tile == 8)
    return col_dispatch<8>(d.n2, latency, [&](auto th) {
      return col_inverse_t<8, decltype(th)::value, MR>(d, dd, count, unsigned_mode, s);
    });
  return col_dispatch<4>(d.n2, latency, [&](auto th) {
    return col_inverse_t<4, decltype(th)::value, MR>(d, dd, count, unsigned_mode, s);
  });
}

cudaError_t launch_col_fused_r16(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                                 cudaStream_t s) {
  return d.radix == 16 ? col_fused_m<16>(d, dd, count, s) : col_fused_m<8>(d, dd, count, s);
}

cudaError_t launch_col_forward_r16(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                                   bool apply, cudaStream_t s) {
  return d.radix == 16 ? col_forward_m<16>(d, dd, count, apply, s)
                       : col_forward_m<8>(d, dd, count, apply, s);
}

cudaError_t launch_col_inverse_r16(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                                   bool unsigned_mode, cudaStream_t s) {
  return d.radix == 16 ? col_inverse_m<16>(d, dd, count, unsigned_mode, s)
                       : col_inverse_m<8>(d, dd, count, unsigned_mode, s);
}

}  // namespace lnt
