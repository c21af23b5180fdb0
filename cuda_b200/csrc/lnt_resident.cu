// SMEM-resident squaring loop: one residue of n <= 4096 words per CTA, kept in
// shared memory for every iteration of the launch.
//
// The transform runs as register passes over shared memory (smem_passes.cuh,
// twiddles from the pass tables in rt / irt): a few barriers per squaring
// instead of one per radix-2 stage.
//
// Replaces the reference's FFT_1SMEM pool (kernel_pool.cu:31-38): the fused
// weight/NTT/square/iNTT/unweight kernels (kernels/w_fft_sqr_ifft_uw__r2_8to4k.cu,
// __r4_16to4k.cu, __r8_4096.cu) followed by the separate r2b (kernels/r2b.cu)
// and m2 (kernels/m2.cu) launches, three launches and an HBM round trip per
// iteration.  Here weight -> forward NTT -> square -> inverse NTT -> unweight ->
// carry -> minus two run back to back inside one launch for all iterations, so
// the loop is bound by the SM's integer pipe, not by launch latency.  Many
// residues (a batch) run as many CTAs of the same launch.
#include <mutex>
#include <set>

#include "lnt_internal.h"
#include "carry.cuh"
#include "smem_passes.cuh"

namespace lnt {

namespace {

using namespace smem;

constexpr uint32_t kRunWords = 8;  // words per carry run (one thread each)
constexpr uint32_t kMaxThreads = 1024;
// CTA size: one thread per 8 words (one radix-8 pass task) when the launch
// fills the GPU with tests; one per 4 words when it carries fewer tests than
// SMs, where latency, not throughput, decides (n = 2048 alone: 11.9 us per
// squaring with 512 threads, 12.9 with 256; nine tests: 48K vs 55K tests/hour).

__global__ void __launch_bounds__(kMaxThreads) resident_square_loop(const ResidentDesc* descs,
                                                                    int latency_mode) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const ResidentDesc D = descs[blockIdx.x];
  const uint32_t n = D.n;
  const uint32_t tid = threadIdx.x, bd = blockDim.x;
  const int ld = padded((int)n);
  uint64_t* s = reinterpret_cast<uint64_t*>(smem_raw);  // the residue, padded layout (sw)
  uint64_t* w = s + ld;
  uint64_t* uw = w + n;
  int64_t* runc = reinterpret_cast<int64_t*>(uw + n);
  uint8_t* wd = reinterpret_cast<uint8_t*>(runc + bd);
  const Passes P = make_passes((int)D.log2n);

  // latency mode: runs of 4 words where the exponent allows, one per thread
  // (n / 4 threads), which halves each thread's carry chain
  const uint32_t run_words = latency_mode && D.short_runs ? 4u : kRunWords;
  const uint32_t runs = n >= run_words ? n / run_words : 1;  // active carry threads
  const uint32_t K = n / runs;                               // words per run

  for (uint32_t j = tid; j < n; j += bd) {
    s[sw(j)] = (uint64_t)D.digits[j];
    w[j] = D.w[j];
    uw[j] = D.uw[j];
    wd[j] = D.widths[j];
  }
  __syncthreads();

  uint32_t status = 0;
  for (uint64_t it = 0; it < D.iterations; ++it) {
    const bool um = D.unsigned_first && it == 0;
    // weight the digits (balanced digits become field elements)
    for (uint32_t j = tid; j < n; j += bd) s[sw(j)] = gl::mul_digit((int64_t)s[sw(j)], w[j]);
    __syncthreads();
    // forward passes, the last one fused with the square and the first inverse pass
    int span = (int)n;
    for (int j = 0, seg = 0; j + 1 < P.m; ++j) {
      pass_r<0>(P.radix[j], s, ld, 1, (int)n, span, D.rt + seg);
      seg += span;
      span /= P.radix[j];
      __syncthreads();
    }
    pass_r<2>(P.radix[P.m - 1], s, ld, 1, (int)n, span, nullptr);
    __syncthreads();
    for (int j = P.m - 2; j >= 0; --j) {
      span *= P.radix[j];
      pass_r<1>(P.radix[j], s, ld, 1, (int)n, span, D.irt + pass_table_offset(P, (int)n, j));
      __syncthreads();
    }

    // unweight, then carry each run of K words to balanced digits; the LL
    // "minus two" enters as the initial carry of the run holding word 0.
    if (tid < runs) {
      int64_t carry = (!D.prp && tid == 0) ? -2 : 0;
      for (uint32_t k = 0; k < K; ++k) {
        const uint32_t j = tid * K + k;
        s[sw(j)] = (uint64_t)carry_digit(gl::mul(s[sw(j)], uw[j]), um, carry, wd[j], carry);
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
        s[sw(j0 + k)] = (uint64_t)balance((int64_t)s[sw(j0 + k)] + carry, wd[j0 + k], q);
        carry = q;
      }
      if (carry != 0) {
        s[sw(j0 + K - 1)] = (uint64_t)((int64_t)s[sw(j0 + K - 1)] + carry);
        if (carry > kAbsorbLimit || carry < -kAbsorbLimit) status |= kStatusCarryOverflow;
      }
    }
    __syncthreads();
  }

  for (uint32_t j = tid; j < n; j += bd) D.digits[j] = (int64_t)s[sw(j)];
  if (status) atomicOr(D.status, status);
}

}  // namespace

uint32_t resident_threads(uint32_t n, uint32_t count, uint32_t sms) {
  uint32_t t = n / (count < sms ? 4u : 8u);
  t = t < 32 ? 32 : t;
  return t > kMaxThreads ? kMaxThreads : t;
}

size_t resident_smem_bytes(uint32_t n, uint32_t threads) {
  return 8 * ((size_t)padded((int)n) + 2 * (size_t)n) + 8 * (size_t)threads + n;
}

cudaError_t launch_resident(const ResidentDesc* d_descs, uint32_t count, uint32_t max_n,
                            cudaStream_t stream) {
  DeviceInfo info;
  cudaError_t e = device_info(info);
  if (e != cudaSuccess) return e;
  const uint32_t sms = (uint32_t)info.sms;
  const uint32_t threads = resident_threads(max_n, count, sms);
  size_t smem = resident_smem_bytes(max_n, threads);
  // Fewer tests than SMs: every test gets an SM of its own.  Left to itself
  // the block scheduler may place two of the CTAs on one SM (their registers
  // and shared memory fit), which halves both tests' speed while other SMs
  // idle; a CTA holding more than half of an SM's shared memory cannot share.
  if (count > 1 && count <= sms) {
    const size_t solo = (size_t)info.smem_per_sm / 2 + 1024;
    if (solo > smem && solo <= (size_t)info.smem_per_block_optin) smem = solo;
  }
  // the kernel's dynamic shared-memory cap, raised once per device to the
  // largest a launch can ask for
  {
    static std::mutex mu;
    static std::set<int> raised;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (!raised.count(dev)) {
      e = cudaFuncSetAttribute(resident_square_loop, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               info.smem_per_block_optin);
      if (e != cudaSuccess) return e;
      raised.insert(dev);
    }
  }
  if (smem > (size_t)info.smem_per_block_optin) return cudaErrorInvalidValue;
  resident_square_loop<<<count, threads, smem, stream>>>(d_descs, count < sms ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace lnt
