// SMEM-resident squaring loop: one residue of n <= 4096 words per CTA, kept in
// shared memory for every iteration of the launch.
//
// Replaces the reference's FFT_1SMEM pool (kernel_pool.cu:31-38): the fused
// weight/NTT/square/iNTT/unweight kernels (kernels/w_fft_sqr_ifft_uw__r2_8to4k.cu,
// __r4_16to4k.cu, __r8_4096.cu) followed by the separate r2b (kernels/r2b.cu)
// and m2 (kernels/m2.cu) launches, three launches and an HBM round trip per
// iteration.  Here weight -> forward NTT -> square -> inverse NTT -> unweight ->
// carry -> minus two run back to back inside one launch for all iterations, so
// the loop is bound by the SM's integer pipe, not by launch latency.  Many
// residues (a batch) run as many CTAs of the same launch.
#include "lnt_internal.h"
#include "carry.cuh"

namespace lnt {

namespace {

constexpr uint32_t kRunWords = 8;  // words per carry run (one thread each)
constexpr uint32_t kMaxThreads = 512;

__device__ __forceinline__ void ntt_forward(uint64_t* s, const uint64_t* rt, uint32_t n,
                                            uint32_t log2n) {
  // Decimation in frequency: natural order in, bit-reversed order out.
  const uint32_t half = n >> 1;
  uint32_t step = 1;
  for (int lg = (int)log2n - 1; lg >= 0; --lg, step <<= 1) {
    const uint32_t h = 1u << lg;
    for (uint32_t b = threadIdx.x; b < half; b += blockDim.x) {
      const uint32_t i = b & (h - 1);
      const uint32_t i0 = ((b >> lg) << (lg + 1)) + i;
      const uint64_t x = s[i0], y = s[i0 + h];
      s[i0] = gl::add(x, y);
      s[i0 + h] = gl::mul(gl::sub(x, y), rt[i * step]);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void ntt_inverse(uint64_t* s, const uint64_t* irt, uint32_t n,
                                            uint32_t log2n) {
  // Decimation in time with inverse roots: bit-reversed in, natural out.
  const uint32_t half = n >> 1;
  uint32_t step = half;
  for (uint32_t lg = 0; lg < log2n; ++lg, step >>= 1) {
    const uint32_t h = 1u << lg;
    for (uint32_t b = threadIdx.x; b < half; b += blockDim.x) {
      const uint32_t i = b & (h - 1);
      const uint32_t i0 = ((b >> lg) << (lg + 1)) + i;
      const uint64_t x = s[i0], y = gl::mul(s[i0 + h], irt[i * step]);
      s[i0] = gl::add(x, y);
      s[i0 + h] = gl::sub(x, y);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kMaxThreads) resident_square_loop(const ResidentDesc* descs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const ResidentDesc D = descs[blockIdx.x];
  const uint32_t n = D.n, half = n > 1 ? n >> 1 : 1;
  const uint32_t tid = threadIdx.x, bd = blockDim.x;
  uint64_t* s = reinterpret_cast<uint64_t*>(smem_raw);
  uint64_t* w = s + n;
  uint64_t* uw = w + n;
  uint64_t* rt = uw + n;
  uint64_t* irt = rt + half;
  int64_t* runc = reinterpret_cast<int64_t*>(irt + half);
  uint8_t* wd = reinterpret_cast<uint8_t*>(runc + bd);

  const uint32_t runs = n >= kRunWords ? n / kRunWords : 1;  // active carry threads
  const uint32_t K = n / runs;                              // words per run

  for (uint32_t j = tid; j < n; j += bd) {
    s[j] = (uint64_t)D.digits[j];
    w[j] = D.w[j];
    uw[j] = D.uw[j];
    wd[j] = D.widths[j];
  }
  for (uint32_t j = tid; j < half; j += bd) {
    rt[j] = D.rt[j];
    irt[j] = D.irt[j];
  }
  __syncthreads();

  uint32_t status = 0;
  for (uint64_t it = 0; it < D.iterations; ++it) {
    const bool um = D.unsigned_first && it == 0;
    // weight the digits (balanced digits become field elements)
    for (uint32_t j = tid; j < n; j += bd) s[j] = gl::mul(gl::from_signed((int64_t)s[j]), w[j]);
    __syncthreads();
    ntt_forward(s, rt, n, D.log2n);
    for (uint32_t j = tid; j < n; j += bd) s[j] = gl::sqr(s[j]);
    __syncthreads();
    ntt_inverse(s, irt, n, D.log2n);

    // unweight, then carry each run of K words to balanced digits; the LL
    // "minus two" enters as the initial carry of the run holding word 0.
    if (tid < runs) {
      int64_t carry = (!D.prp && tid == 0) ? -2 : 0;
      for (uint32_t k = 0; k < K; ++k) {
        const uint32_t j = tid * K + k;
        int64_t hi, lo, q;
        split_output(gl::mul(s[j], uw[j]), um, wd[j], hi, lo);
        const int64_t d = balance(lo + carry, wd[j], q);
        carry = hi + q;
        s[j] = (uint64_t)d;
      }
      runc[tid] = carry;
    }
    __syncthreads();
    // each run takes the carry of the run before it (cyclically: 2^q == 1 mod M)
    if (tid < runs) {
      int64_t carry = runc[tid == 0 ? runs - 1 : tid - 1];
      const uint32_t j0 = tid * K;
      for (uint32_t k = 0; k + 1 < K && carry != 0; ++k) {
        int64_t q;
        s[j0 + k] = (uint64_t)balance((int64_t)s[j0 + k] + carry, wd[j0 + k], q);
        carry = q;
      }
      if (carry != 0) {
        s[j0 + K - 1] = (uint64_t)((int64_t)s[j0 + K - 1] + carry);
        if (carry > kAbsorbLimit || carry < -kAbsorbLimit) status |= kStatusCarryOverflow;
      }
    }
    __syncthreads();
  }

  for (uint32_t j = tid; j < n; j += bd) D.digits[j] = (int64_t)s[j];
  if (status) atomicOr(D.status, status);
}

}  // namespace

uint32_t resident_threads(uint32_t n) {
  uint32_t runs = n >= kRunWords ? n / kRunWords : 1;
  uint32_t t = runs < 32 ? 32 : runs;
  return t > kMaxThreads ? kMaxThreads : t;
}

size_t resident_smem_bytes(uint32_t n, uint32_t threads) {
  size_t half = n > 1 ? n / 2 : 1;
  return 8 * (3 * (size_t)n + 2 * half) + 8 * (size_t)threads + n;
}

cudaError_t launch_resident(const ResidentDesc* d_descs, uint32_t count, uint32_t max_n,
                            cudaStream_t stream) {
  const uint32_t threads = resident_threads(max_n);
  const size_t smem = resident_smem_bytes(max_n, threads);
  cudaError_t e = cudaFuncSetAttribute(resident_square_loop,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  resident_square_loop<<<count, threads, smem, stream>>>(d_descs);
  return cudaGetLastError();
}

}  // namespace lnt
