// Precomputed tables: IBDWT weights/unweights and 4-step twiddles.
//
// Replaces common/pre_calculation.cu:23-36 (calc_weights_widths) and :69-77
// (calc_brev_factors).  The weights are the same field elements as the
// reference's: w_j = 7^(((p-1)/192/n) * 5 * (n - r_j)), r_j = q j mod n, w_0 = 1,
// uw_j = (w_j n)^-1, uw_0 = n^-1.  With g = 7^(((p-1)/192/n) * 5) (g^n = 2),
// uw_j = g^r_j / (2n) for j > 0.  The weight of word j thus places it at bit
// ceil(qj/n) when r_j != 0; words with r_j = 0, j > 0 (q sharing a factor with
// n) sit exactly on bit qj/n and take weight 1.  The widths (lnt_policy.cpp,
// word_widths) are the exact integer differences of those bits, so every word
// starts where its weight says.
#include "lnt_internal.h"
#include "goldilocks.cuh"

namespace lnt {

namespace {

__global__ void weights_kernel(uint32_t exponent, uint32_t n, uint64_t g, uint64_t inv_n,
                               uint64_t inv_2n, uint64_t* w, uint64_t* uw) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  if (j == 0) {
    w[0] = 1;
    uw[0] = inv_n;
    return;
  }
  const uint32_t r = (uint32_t)(((uint64_t)exponent * j) % n);
  if (r == 0) {
    // qj/n is a whole bit: the word starts exactly there (weight 1).  The formula
    // below would give g^n = 2, one bit off; this happens for j > 0 only when q
    // shares a factor with n (an even q, or q divisible by 5 at n = 5 * 2^k).
    w[j] = 1;
    uw[j] = inv_n;
    return;
  }
  w[j] = gl::pow(g, (uint64_t)(n - r));
  uw[j] = gl::mul(gl::pow(g, (uint64_t)r), inv_2n);
}

// twf[row * n1 + j1] = omega_n^(j1 * k2) with k2 = bit-reverse(row) over log2n2
// bits: the frequency that the forward column NTT leaves in memory row `row`.
__global__ void twiddle_kernel(uint32_t n1, uint32_t n2, uint32_t log2n2, uint64_t root,
                               uint64_t iroot, uint64_t* twf, uint64_t* twi) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)n1 * n2) return;
  const uint32_t row = (uint32_t)(idx / n1), j1 = (uint32_t)(idx % n1);
  const uint32_t k2 = __brev(row) >> (32 - log2n2);
  const uint64_t e = (uint64_t)j1 * k2;
  twf[idx] = gl::pow(root, e);
  twi[idx] = gl::pow(iroot, e);
}

// natural index j = r * n1 + t * tile + c  ->  (t * n2 + r) * tile + c
__global__ void tile_major_kernel(const uint64_t* w, const uint64_t* uw, const uint8_t* widths,
                                  uint32_t n1, uint32_t n2, uint32_t tile, uint64_t* wt,
                                  uint64_t* uwt, uint8_t* widt) {
  const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (size_t)n1 * n2) return;
  const uint32_t r = (uint32_t)(j / n1), col = (uint32_t)(j % n1);
  const uint32_t t = col / tile, c = col % tile;
  const size_t k = ((size_t)t * n2 + r) * tile + c;
  wt[k] = w[j];
  uwt[k] = uw[j];
  widt[k] = widths[j];
}

}  // namespace

cudaError_t launch_tile_major(const uint64_t* w, const uint64_t* uw, const uint8_t* widths,
                              uint32_t n1, uint32_t n2, uint32_t tile, uint64_t* wt, uint64_t* uwt,
                              uint8_t* widt, cudaStream_t s) {
  const uint64_t n = (uint64_t)n1 * n2;
  tile_major_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(w, uw, widths, n1, n2, tile, wt, uwt,
                                                                 widt);
  return cudaGetLastError();
}

cudaError_t launch_weights(uint32_t exponent, uint32_t n, uint64_t* w, uint64_t* uw,
                           cudaStream_t s) {
  const uint64_t c = ((gl::P - 1) / 192 / n) * 5ull;
  const uint64_t g = gl::pow(7, c);
  const uint64_t inv_n = gl::inv(n), inv_2n = gl::inv(2ull * n);
  const uint32_t threads = 256, blocks = (n + threads - 1) / threads;
  weights_kernel<<<blocks, threads, 0, s>>>(exponent, n, g, inv_n, inv_2n, w, uw);
  return cudaGetLastError();
}

namespace {
// tw5[(k5 - 1) L + c] = omega_{5L}^(k5 c): the twiddle between the 5-point
// transform of the words c + L j5 and the L-point transform of plane k5
__global__ void five_twiddle_kernel(uint32_t L, uint64_t root, uint64_t iroot, uint64_t* tw5,
                                    uint64_t* itw5) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 4 * L) return;
  const uint64_t e = (uint64_t)(idx / L + 1) * (idx % L);
  tw5[idx] = gl::pow(root, e);
  itw5[idx] = gl::pow(iroot, e);
}
}  // namespace

cudaError_t launch_five_twiddles(uint32_t L, uint64_t* tw5, uint64_t* itw5, uint64_t c5[4],
                                 cudaStream_t s) {
  // omega_{5L} = 554^((p-1)/5L) = omega_n^n2, the same root family as every other table
  const uint64_t root = gl::pow(554, (gl::P - 1) / (5ull * L)), iroot = gl::inv(root);
  const uint64_t w = gl::pow(root, L), half = gl::inv(2);  // omega_5
  const uint64_t w2 = gl::mul(w, w), w3 = gl::mul(w2, w), w4 = gl::mul(w3, w);
  c5[0] = gl::mul(gl::add(w, w4), half);
  c5[1] = gl::mul(gl::add(w2, w3), half);
  c5[2] = gl::mul(gl::sub(w, w4), half);
  c5[3] = gl::mul(gl::sub(w2, w3), half);
  five_twiddle_kernel<<<(4 * L + 255) / 256, 256, 0, s>>>(L, root, iroot, tw5, itw5);
  return cudaGetLastError();
}

cudaError_t launch_twiddles(uint32_t n1, uint32_t n2, uint32_t log2n2, uint64_t* twf,
                            uint64_t* twi, cudaStream_t s) {
  const uint64_t n = (uint64_t)n1 * n2;
  const uint64_t root = gl::pow(554, (gl::P - 1) / n);
  const uint64_t iroot = gl::inv(root);
  const uint32_t threads = 256;
  const uint64_t blocks = (n + threads - 1) / threads;
  twiddle_kernel<<<(unsigned)blocks, threads, 0, s>>>(n1, n2, log2n2, root, iroot, twf, twi);
  return cudaGetLastError();
}

}  // namespace lnt
