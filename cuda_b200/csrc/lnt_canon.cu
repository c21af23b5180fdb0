// Canonical readout kernels: balanced digits (plus pending run carries) ->
// the reference's non-negative digit vector of the same residue.  The
// per-block steps are in canon_core.cuh (shared with the CPU test harness).
// Which of 0 / M the value shows as (both are 0 mod M) is decided by the host
// from the flags, following the reference's carry semantics.
#include "canon_core.cuh"
#include "lnt_internal.h"

namespace lnt {

namespace {

__global__ void canon_local(CanonDesc D) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < D.nblocks) canon_local_block(D, b);
}

__global__ void canon_hop(CanonDesc D) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < D.nblocks && !canon_hop_block(D, b)) atomicOr(D.flags, kCanonError);
}

constexpr uint32_t kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) canon_scan(CanonDesc D) {
  __shared__ uint8_t chunk_fn[kScanThreads];
  __shared__ int8_t chunk_cin[kScanThreads];
  const uint32_t t = threadIdx.x;
  const uint32_t per = (D.nblocks + kScanThreads - 1) / kScanThreads;
  const uint32_t b0 = min(D.nblocks, t * per), b1 = min(D.nblocks, b0 + per);
  chunk_fn[t] = (uint8_t)canon_chunk_fn(D, b0, b1);
  __syncthreads();
  if (t == 0) {
    uint32_t total = kCanonIdentity;
    for (uint32_t i = 0; i < kScanThreads; ++i) total = canon_compose(total, chunk_fn[i]);
    int c;
    if (!canon_wrap_carry(total, c)) atomicOr(D.flags, kCanonError);
    for (uint32_t i = 0; i < kScanThreads; ++i) {
      chunk_cin[i] = (int8_t)c;
      c = canon_apply_fn(chunk_fn[i], c);
    }
  }
  __syncthreads();
  canon_chunk_cin(D, b0, b1, chunk_cin[t]);
}

__global__ void canon_apply(CanonDesc D) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  bool not_all_max = false, high_nonzero = false;
  if (b < D.nblocks) canon_apply_block(D, b, not_all_max, high_nonzero);
  // block-wide vote, one atomic per CTA (every thread reaches both barriers)
  const int any_below = __syncthreads_or(not_all_max ? 1 : 0);
  const int any_high = __syncthreads_or(high_nonzero ? 1 : 0);
  if (threadIdx.x == 0) {
    const uint32_t flags = (any_below ? kCanonNotAllMax : 0u) | (any_high ? kCanonHighNonZero : 0u);
    if (flags) atomicOr(D.flags, flags);
  }
}

__global__ void fill_max_kernel(uint64_t* out, const uint8_t* widths, uint32_t n) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) out[j] = (1ull << widths[j]) - 1;
}

}  // namespace

uint32_t canon_block_size(uint32_t n) { return n < 64 ? n : 64; }

cudaError_t launch_canonicalize(const CanonDesc& d, cudaStream_t s) {
  const uint32_t threads = 128;
  const uint32_t blocks = (d.nblocks + threads - 1) / threads;
  canon_local<<<blocks, threads, 0, s>>>(d);
  canon_hop<<<blocks, threads, 0, s>>>(d);
  canon_scan<<<1, kScanThreads, 0, s>>>(d);
  canon_apply<<<blocks, threads, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_fill_max(uint64_t* out, const uint8_t* widths, uint32_t n, cudaStream_t s) {
  fill_max_kernel<<<(n + 255) / 256, 256, 0, s>>>(out, widths, n);
  return cudaGetLastError();
}

}  // namespace lnt
