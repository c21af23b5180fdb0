// Two-pass (4-step) squaring for n > 4096 words.
//
// Replaces the reference's FFT_2SMEM pool (kernel_pool.cu:39-48): the column
// kernels w_fftc_tw (kernels/w_fftc_tw__r2_8to4k.cu) and tw_ifftc_uw
// (kernels/tw_ifftc_uw__r2_8to4k.cu), the row kernel fftr_sqr_ifftr
// (kernels/fftr_sqr_ifftr__*.cu), and the separate r2b / m2 launches.
//
// Layout: the residue's natural index j = j1 + n1 * j2 is stored row-major,
// row j2 holding columns j1 = 0..n1-1.  Per squaring:
//   col_forward : carry-in from the previous squaring, weight, forward NTT of
//                 every column (length n2, stride n1), bit-reversed row order
//   row_square  : 4-step twiddle, forward NTT of the row, square, inverse NTT,
//                 inverse twiddle (contiguous rows of n1 words)
//   col_inverse : inverse NTT of every column, unweight, carry of each run of
//                 `tile` consecutive words to balanced digits, minus two
// A column-pass CTA owns `tile` adjacent columns, so each of its rows is a run
// of `tile` consecutive words; the run's outgoing carry is stored and added to
// the next run by the next col_forward (no inter-CTA waiting).  Tiles are
// staged in shared memory with coalesced row segments; the reference reads
// columns one word per thread at stride n1.
#include "lnt_internal.h"
#include "carry.cuh"

namespace lnt {

namespace {

constexpr uint32_t kThreads = 256;

// forward DIF over `cols` columns of length L stored at sm[c * ld + i]
__device__ __forceinline__ void columns_forward(uint64_t* sm, uint32_t ld, uint32_t cols,
                                                uint32_t L, uint32_t log2L, const uint64_t* rt) {
  const uint32_t half = L >> 1, total = cols * half;
  uint32_t step = 1;
  for (int lg = (int)log2L - 1; lg >= 0; --lg, step <<= 1) {
    const uint32_t h = 1u << lg;
    for (uint32_t b = threadIdx.x; b < total; b += blockDim.x) {
      const uint32_t c = b >> (log2L - 1), bb = b & (half - 1);
      const uint32_t i = bb & (h - 1);
      uint64_t* col = sm + (size_t)c * ld;
      const uint32_t i0 = ((bb >> lg) << (lg + 1)) + i;
      const uint64_t x = col[i0], y = col[i0 + h];
      col[i0] = gl::add(x, y);
      col[i0 + h] = gl::mul(gl::sub(x, y), rt[i * step]);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void columns_inverse(uint64_t* sm, uint32_t ld, uint32_t cols,
                                                uint32_t L, uint32_t log2L, const uint64_t* irt) {
  const uint32_t half = L >> 1, total = cols * half;
  uint32_t step = half;
  for (uint32_t lg = 0; lg < log2L; ++lg, step >>= 1) {
    const uint32_t h = 1u << lg;
    for (uint32_t b = threadIdx.x; b < total; b += blockDim.x) {
      const uint32_t c = b >> (log2L - 1), bb = b & (half - 1);
      const uint32_t i = bb & (h - 1);
      uint64_t* col = sm + (size_t)c * ld;
      const uint32_t i0 = ((bb >> lg) << (lg + 1)) + i;
      const uint64_t x = col[i0], y = gl::mul(col[i0 + h], irt[i * step]);
      col[i0] = gl::add(x, y);
      col[i0 + h] = gl::sub(x, y);
    }
    __syncthreads();
  }
}

// The run (tile t, row r) receives the carry of the run before it in natural
// order: (t - 1, r), or the last tile of row r - 1, cyclically.
__device__ __forceinline__ size_t predecessor_run(uint32_t t, uint32_t r, uint32_t n2,
                                                  uint32_t ntiles) {
  if (t > 0) return (size_t)(t - 1) * n2 + r;
  return (size_t)(ntiles - 1) * n2 + (r ? r - 1 : n2 - 1);
}

__global__ void __launch_bounds__(kThreads) col_forward(TwoPassDesc D, int apply_carries) {
  extern __shared__ __align__(16) uint64_t sm[];
  const uint32_t T = D.tile, n1 = D.n1, n2 = D.n2, ld = n2 + 1;
  const uint32_t t0 = blockIdx.x, c0 = t0 * T;
  uint32_t status = 0;

  for (uint32_t idx = threadIdx.x; idx < T * n2; idx += blockDim.x) {
    const uint32_t r = idx / T, c = idx % T;
    sm[(size_t)c * ld + r] = (uint64_t)D.x[(size_t)r * n1 + c0 + c];
  }
  __syncthreads();
  if (apply_carries) {
    for (uint32_t r = threadIdx.x; r < n2; r += blockDim.x) {
      int64_t carry = D.carry[predecessor_run(t0, r, n2, D.ntiles)];
      const size_t jrow = (size_t)r * n1 + c0;
      uint32_t c = 0;
      for (; c + 1 < T && carry != 0; ++c) {
        int64_t q;
        uint64_t& v = sm[(size_t)c * ld + r];
        v = (uint64_t)balance((int64_t)v + carry, D.widths[jrow + c], q);
        carry = q;
      }
      if (carry != 0) {
        uint64_t& v = sm[(size_t)(T - 1) * ld + r];
        v = (uint64_t)((int64_t)v + carry);
        if (carry > kAbsorbLimit || carry < -kAbsorbLimit) status |= kStatusCarryOverflow;
      }
    }
    __syncthreads();
  }
  for (uint32_t idx = threadIdx.x; idx < T * n2; idx += blockDim.x) {
    const uint32_t r = idx / T, c = idx % T;
    uint64_t& v = sm[(size_t)c * ld + r];
    v = gl::mul_digit((int64_t)v, D.w[(size_t)r * n1 + c0 + c]);
  }
  __syncthreads();
  columns_forward(sm, ld, T, n2, D.log2n2, D.rt2);
  for (uint32_t idx = threadIdx.x; idx < T * n2; idx += blockDim.x) {
    const uint32_t r = idx / T, c = idx % T;
    D.x[(size_t)r * n1 + c0 + c] = (int64_t)sm[(size_t)c * ld + r];
  }
  if (status) atomicOr(D.status, status);
}

__global__ void __launch_bounds__(kThreads) row_square(TwoPassDesc D) {
  extern __shared__ __align__(16) uint64_t sm[];
  const uint32_t n1 = D.n1, half = n1 >> 1;
  const size_t base = (size_t)blockIdx.x * n1;
  uint64_t* x = reinterpret_cast<uint64_t*>(D.x) + base;
  for (uint32_t j = threadIdx.x; j < n1; j += blockDim.x) sm[j] = gl::mul(x[j], D.twf[base + j]);
  __syncthreads();
  // forward DIF of the row
  uint32_t step = 1;
  for (int lg = (int)D.log2n1 - 1; lg >= 0; --lg, step <<= 1) {
    const uint32_t h = 1u << lg;
    for (uint32_t b = threadIdx.x; b < half; b += blockDim.x) {
      const uint32_t i = b & (h - 1), i0 = ((b >> lg) << (lg + 1)) + i;
      const uint64_t u = sm[i0], v = sm[i0 + h];
      sm[i0] = gl::add(u, v);
      sm[i0 + h] = gl::mul(gl::sub(u, v), D.rt1[i * step]);
    }
    __syncthreads();
  }
  for (uint32_t j = threadIdx.x; j < n1; j += blockDim.x) sm[j] = gl::sqr(sm[j]);
  __syncthreads();
  step = half;
  for (uint32_t lg = 0; lg < D.log2n1; ++lg, step >>= 1) {
    const uint32_t h = 1u << lg;
    for (uint32_t b = threadIdx.x; b < half; b += blockDim.x) {
      const uint32_t i = b & (h - 1), i0 = ((b >> lg) << (lg + 1)) + i;
      const uint64_t u = sm[i0], v = gl::mul(sm[i0 + h], D.irt1[i * step]);
      sm[i0] = gl::add(u, v);
      sm[i0 + h] = gl::sub(u, v);
    }
    __syncthreads();
  }
  for (uint32_t j = threadIdx.x; j < n1; j += blockDim.x) x[j] = gl::mul(sm[j], D.twi[base + j]);
}

__global__ void __launch_bounds__(kThreads) col_inverse(TwoPassDesc D, int unsigned_mode) {
  extern __shared__ __align__(16) uint64_t sm[];
  const uint32_t T = D.tile, n1 = D.n1, n2 = D.n2, ld = n2 + 1;
  const uint32_t t0 = blockIdx.x, c0 = t0 * T;

  for (uint32_t idx = threadIdx.x; idx < T * n2; idx += blockDim.x) {
    const uint32_t r = idx / T, c = idx % T;
    sm[(size_t)c * ld + r] = (uint64_t)D.x[(size_t)r * n1 + c0 + c];
  }
  __syncthreads();
  columns_inverse(sm, ld, T, n2, D.log2n2, D.irt2);
  for (uint32_t idx = threadIdx.x; idx < T * n2; idx += blockDim.x) {
    const uint32_t r = idx / T, c = idx % T;
    uint64_t& v = sm[(size_t)c * ld + r];
    v = gl::mul(v, D.uw[(size_t)r * n1 + c0 + c]);
  }
  __syncthreads();
  for (uint32_t r = threadIdx.x; r < n2; r += blockDim.x) {
    int64_t carry = (!D.prp && t0 == 0 && r == 0) ? -2 : 0;
    const size_t jrow = (size_t)r * n1 + c0;
    for (uint32_t c = 0; c < T; ++c) {
      uint64_t& v = sm[(size_t)c * ld + r];
      const unsigned w = D.widths[jrow + c];
      v = (uint64_t)carry_digit(v, unsigned_mode != 0, carry, w, carry);
    }
    D.carry[(size_t)t0 * n2 + r] = carry;
  }
  __syncthreads();
  for (uint32_t idx = threadIdx.x; idx < T * n2; idx += blockDim.x) {
    const uint32_t r = idx / T, c = idx % T;
    D.x[(size_t)r * n1 + c0 + c] = (int64_t)sm[(size_t)c * ld + r];
  }
}

size_t col_smem(const TwoPassDesc& d) { return (size_t)d.tile * (d.n2 + 1) * 8; }

}  // namespace

cudaError_t launch_col_forward(const TwoPassDesc& d, bool apply_carries, cudaStream_t s) {
  const size_t smem = col_smem(d);
  cudaError_t e = cudaFuncSetAttribute(col_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  col_forward<<<d.ntiles, kThreads, smem, s>>>(d, apply_carries ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_row_square(const TwoPassDesc& d, cudaStream_t s) {
  const size_t smem = (size_t)d.n1 * 8;
  cudaError_t e = cudaFuncSetAttribute(row_square, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  row_square<<<d.n2, kThreads, smem, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_col_inverse(const TwoPassDesc& d, bool unsigned_mode, cudaStream_t s) {
  const size_t smem = col_smem(d);
  cudaError_t e = cudaFuncSetAttribute(col_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  col_inverse<<<d.ntiles, kThreads, smem, s>>>(d, unsigned_mode ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace lnt
