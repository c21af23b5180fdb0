// Two-pass squaring with register-resident sub-transforms (n = 2^16 ... 2^24).
//
// Same layout and carry scheme as lnt_twopass.cu (which replaces the
// reference's FFT_2SMEM pool, kernel_pool.cu:39-48), with the transforms
// restructured for the SM: a transform of length L = RA * RB (RA = 64) runs as
//   pass A: each thread holds RA elements at stride RB in registers, a DIF of
//           RA points with power-of-two twiddles (ntt_core.cuh), then one table
//           twiddle omega_L^(i1 * k2);
//   pass B: each thread takes a contiguous block of RB elements, a DIF of RB
//           points.
// The output is in fully bit-reversed order, exactly as the radix-2 kernels
// leave it, so the 4-step twiddle tables are shared.  Per element a transform
// costs 1 table multiplication plus log2(L) shift butterflies, where the
// reference pays one general modular multiplication per radix-2 butterfly
// (core/fft_r2.cuh:17-107).  The row kernel squares between its forward and
// inverse pass B in registers and reads/writes HBM directly in pass A, so a
// row crosses shared memory twice.
#include "carry.cuh"
#include "lnt_internal.h"
#include "ntt_core.cuh"

namespace lnt {

namespace {

template <int L>
struct Split {
  static constexpr int RA = 64;          // pass A radix (stride RB)
  static constexpr int RB = L / 64;      // pass B radix (contiguous)
  static constexpr int PADB = RB + 1;    // padded block stride in shared memory
  static constexpr int WORDS = RA * PADB;
};

// ------------------------------------------------------------------ rows ----

constexpr int kRowThreads = 128;

template <int N1>
__global__ void __launch_bounds__(kRowThreads, 3) row_square_fast(TwoPassDesc D) {
  using S = Split<N1>;
  constexpr int RA = S::RA, RB = S::RB, PADB = S::PADB;
  constexpr int ROWS = kRowThreads / RB;
  extern __shared__ __align__(16) uint64_t sm[];
  const int lr = threadIdx.x / RB, i1 = threadIdx.x % RB;
  const size_t row = (size_t)blockIdx.x * ROWS + lr;
  uint64_t* srow = sm + lr * S::WORDS;
  uint64_t* x = reinterpret_cast<uint64_t*>(D.x) + row * N1;
  const uint64_t* twf = D.twf + row * N1;
  const uint64_t* twi = D.twi + row * N1;

  uint64_t v[RA];
#pragma unroll
  for (int i2 = 0; i2 < RA; ++i2) v[i2] = gl::mul(x[i1 + RB * i2], twf[i1 + RB * i2]);
  dif<RA>(v);
#pragma unroll
  for (int r = 0; r < RA; ++r) srow[i1 + PADB * r] = gl::mul(v[r], D.itw1[i1 * brev_c<RA>(r)]);
  __syncthreads();
  for (int r = i1; r < RA; r += RB) {
    uint64_t u[RB];
#pragma unroll
    for (int s = 0; s < RB; ++s) u[s] = srow[s + PADB * r];
    dif<RB>(u);
#pragma unroll
    for (int s = 0; s < RB; ++s) u[s] = gl::sqr(u[s]);
    dit_inv<RB>(u);
#pragma unroll
    for (int s = 0; s < RB; ++s) srow[s + PADB * r] = u[s];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RA; ++r) v[r] = gl::mul(srow[i1 + PADB * r], D.iitw1[i1 * brev_c<RA>(r)]);
  dit_inv<RA>(v);
#pragma unroll
  for (int i2 = 0; i2 < RA; ++i2) x[i1 + RB * i2] = gl::mul(v[i2], twi[i1 + RB * i2]);
}

// --------------------------------------------------------------- columns ----

constexpr int kColThreads = 256;

template <int N2>
struct ColTile {
  using S = Split<N2>;
  static constexpr int T = kColThreads / S::RB;  // columns per CTA = words per carry run
  // column stride in words: bank-conflict-free coalesced staging
  static constexpr int MOD = T >= 16 ? 1 : 16 / T;
  static constexpr int LD = ((S::WORDS + 15) / 16) * 16 + MOD;
  static constexpr size_t SMEM = (size_t)T * LD * 8;
};

template <int N2>
__device__ __forceinline__ int col_addr(int c, int p) {
  using S = Split<N2>;
  return c * ColTile<N2>::LD + (p % S::RB) + S::PADB * (p / S::RB);
}

template <int N2>
__device__ __forceinline__ void columns_pass_a_forward(uint64_t* sm, const uint64_t* itw) {
  using S = Split<N2>;
  const int c = threadIdx.x / S::RB, i1 = threadIdx.x % S::RB;
  uint64_t* col = sm + c * ColTile<N2>::LD;
  uint64_t v[S::RA];
#pragma unroll
  for (int i2 = 0; i2 < S::RA; ++i2) v[i2] = col[i1 + S::PADB * i2];
  dif<S::RA>(v);
#pragma unroll
  for (int r = 0; r < S::RA; ++r) col[i1 + S::PADB * r] = gl::mul(v[r], itw[i1 * brev_c<S::RA>(r)]);
}

template <int N2>
__device__ __forceinline__ void columns_pass_a_inverse(uint64_t* sm, const uint64_t* iitw) {
  using S = Split<N2>;
  const int c = threadIdx.x / S::RB, i1 = threadIdx.x % S::RB;
  uint64_t* col = sm + c * ColTile<N2>::LD;
  uint64_t v[S::RA];
#pragma unroll
  for (int r = 0; r < S::RA; ++r) v[r] = gl::mul(col[i1 + S::PADB * r], iitw[i1 * brev_c<S::RA>(r)]);
  dit_inv<S::RA>(v);
#pragma unroll
  for (int i2 = 0; i2 < S::RA; ++i2) col[i1 + S::PADB * i2] = v[i2];
}

template <int N2, bool Inverse>
__device__ __forceinline__ void columns_pass_b(uint64_t* sm) {
  using S = Split<N2>;
  constexpr int T = ColTile<N2>::T;
  for (int blk = threadIdx.x; blk < T * S::RA; blk += kColThreads) {
    const int c = blk / S::RA, r = blk % S::RA;
    uint64_t* b = sm + c * ColTile<N2>::LD + S::PADB * r;
    uint64_t u[S::RB];
#pragma unroll
    for (int s = 0; s < S::RB; ++s) u[s] = b[s];
    if constexpr (Inverse)
      dit_inv<S::RB>(u);
    else
      dif<S::RB>(u);
#pragma unroll
    for (int s = 0; s < S::RB; ++s) b[s] = u[s];
  }
}

template <int N2>
__device__ __forceinline__ void tile_load(uint64_t* sm, const int64_t* x, uint32_t n1, uint32_t c0) {
  constexpr int T = ColTile<N2>::T;
  for (int idx = threadIdx.x; idx < T * N2; idx += kColThreads) {
    const int r = idx / T, c = idx % T;
    sm[col_addr<N2>(c, r)] = (uint64_t)x[(size_t)r * n1 + c0 + c];
  }
}

template <int N2>
__device__ __forceinline__ void tile_store(const uint64_t* sm, int64_t* x, uint32_t n1, uint32_t c0) {
  constexpr int T = ColTile<N2>::T;
  for (int idx = threadIdx.x; idx < T * N2; idx += kColThreads) {
    const int r = idx / T, c = idx % T;
    x[(size_t)r * n1 + c0 + c] = (int64_t)sm[col_addr<N2>(c, r)];
  }
}

template <int N2>
__global__ void __launch_bounds__(kColThreads, 1) col_forward_fast(TwoPassDesc D, int apply_carries) {
  constexpr int T = ColTile<N2>::T;
  extern __shared__ __align__(16) uint64_t sm[];
  const uint32_t n1 = D.n1, t0 = blockIdx.x, c0 = t0 * T;
  uint32_t status = 0;

  tile_load<N2>(sm, D.x, n1, c0);
  __syncthreads();
  // per row: carry from the previous run, then weight (balanced digit -> field)
  for (int r = threadIdx.x; r < N2; r += kColThreads) {
    const size_t jrow = (size_t)r * n1 + c0;
    int64_t carry = 0;
    if (apply_carries) {
      const size_t pi = t0 > 0 ? (size_t)(t0 - 1) * N2 + r
                               : (size_t)(D.ntiles - 1) * N2 + (r ? r - 1 : N2 - 1);
      carry = D.carry[pi];
    }
#pragma unroll
    for (int c = 0; c < T; ++c) {
      uint64_t& v = sm[col_addr<N2>(c, r)];
      int64_t d = (int64_t)v;
      if (carry != 0) {
        if (c + 1 < T) {
          int64_t q;
          d = balance(d + carry, D.widths[jrow + c], q);
          carry = q;
        } else {
          d += carry;
          if (carry > kAbsorbLimit || carry < -kAbsorbLimit) status |= kStatusCarryOverflow;
        }
      }
      v = gl::mul(gl::from_signed(d), D.w[jrow + c]);
    }
  }
  __syncthreads();
  columns_pass_a_forward<N2>(sm, D.itw2);
  __syncthreads();
  columns_pass_b<N2, false>(sm);
  __syncthreads();
  tile_store<N2>(sm, D.x, n1, c0);
  if (status) atomicOr(D.status, status);
}

template <int N2>
__global__ void __launch_bounds__(kColThreads, 1) col_inverse_fast(TwoPassDesc D, int unsigned_mode) {
  constexpr int T = ColTile<N2>::T;
  extern __shared__ __align__(16) uint64_t sm[];
  const uint32_t n1 = D.n1, t0 = blockIdx.x, c0 = t0 * T;

  tile_load<N2>(sm, D.x, n1, c0);
  __syncthreads();
  columns_pass_b<N2, true>(sm);
  __syncthreads();
  columns_pass_a_inverse<N2>(sm, D.iitw2);
  __syncthreads();
  // per row: unweight, carry the run of T words to balanced digits, minus two
  for (int r = threadIdx.x; r < N2; r += kColThreads) {
    const size_t jrow = (size_t)r * n1 + c0;
    int64_t carry = (!D.prp && t0 == 0 && r == 0) ? -2 : 0;
#pragma unroll
    for (int c = 0; c < T; ++c) {
      uint64_t& v = sm[col_addr<N2>(c, r)];
      const unsigned w = D.widths[jrow + c];
      int64_t hi, lo, q;
      split_output(gl::mul(v, D.uw[jrow + c]), unsigned_mode != 0, w, hi, lo);
      v = (uint64_t)balance(lo + carry, w, q);
      carry = hi + q;
    }
    D.carry[(size_t)t0 * N2 + r] = carry;
  }
  __syncthreads();
  tile_store<N2>(sm, D.x, n1, c0);
}

template <int N1>
cudaError_t launch_row(const TwoPassDesc& d, cudaStream_t s) {
  constexpr int ROWS = kRowThreads / Split<N1>::RB;
  const size_t smem = (size_t)ROWS * Split<N1>::WORDS * 8;
  cudaError_t e = cudaFuncSetAttribute(row_square_fast<N1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  row_square_fast<N1><<<d.n2 / ROWS, kRowThreads, smem, s>>>(d);
  return cudaGetLastError();
}

template <int N2>
cudaError_t launch_colf(const TwoPassDesc& d, bool apply, cudaStream_t s) {
  const size_t smem = ColTile<N2>::SMEM;
  cudaError_t e = cudaFuncSetAttribute(col_forward_fast<N2>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  col_forward_fast<N2><<<d.ntiles, kColThreads, smem, s>>>(d, apply ? 1 : 0);
  return cudaGetLastError();
}

template <int N2>
cudaError_t launch_coli(const TwoPassDesc& d, bool unsigned_mode, cudaStream_t s) {
  const size_t smem = ColTile<N2>::SMEM;
  cudaError_t e = cudaFuncSetAttribute(col_inverse_fast<N2>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  col_inverse_fast<N2><<<d.ntiles, kColThreads, smem, s>>>(d, unsigned_mode ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace

uint32_t fast_tile(uint32_t log2n2) { return kColThreads / ((1u << log2n2) / 64); }

bool fast_supported(uint32_t log2n1, uint32_t log2n2) {
  return log2n2 >= 8 && log2n2 <= 12 && log2n1 >= 8 && log2n1 <= 12 && log2n1 >= log2n2;
}

cudaError_t launch_row_square_fast(const TwoPassDesc& d, cudaStream_t s) {
  switch (d.log2n1) {
    case 8: return launch_row<256>(d, s);
    case 9: return launch_row<512>(d, s);
    case 10: return launch_row<1024>(d, s);
    case 11: return launch_row<2048>(d, s);
    case 12: return launch_row<4096>(d, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_col_forward_fast(const TwoPassDesc& d, bool apply, cudaStream_t s) {
  switch (d.log2n2) {
    case 8: return launch_colf<256>(d, apply, s);
    case 9: return launch_colf<512>(d, apply, s);
    case 10: return launch_colf<1024>(d, apply, s);
    case 11: return launch_colf<2048>(d, apply, s);
    case 12: return launch_colf<4096>(d, apply, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_col_inverse_fast(const TwoPassDesc& d, bool unsigned_mode, cudaStream_t s) {
  switch (d.log2n2) {
    case 8: return launch_coli<256>(d, unsigned_mode, s);
    case 9: return launch_coli<512>(d, unsigned_mode, s);
    case 10: return launch_coli<1024>(d, unsigned_mode, s);
    case 11: return launch_coli<2048>(d, unsigned_mode, s);
    case 12: return launch_coli<4096>(d, unsigned_mode, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lnt
