// Instruction cost of the device field operations, for ncu's counters.
//
// Each kernel probe<OP> applies one operation of goldilocks.cuh / ntt_core.cuh
// 1024 times per thread on a dependent chain (4096 threads); probe<0> is the
// bare loop.  Run under
//   ncu --metrics smsp__inst_executed.sum,sm__inst_executed_pipe_alu.sum,
//                 sm__inst_executed_pipe_fma.sum --clock-control none cuda_b200/opcount
// and subtract probe<0>: warp instructions x 32 / (4096 x 1024) is the cost of one
// operation per thread, in total and per pipe.  Not part of the library.
#include <cstdint>
#include <cstdio>

#include "../csrc/goldilocks.cuh"
#include "../csrc/ntt_core.cuh"

using namespace lnt;

namespace {

constexpr int kIters = 1024;
constexpr int kThreads = 32 * 128;

template <int OP>
__global__ void probe(const uint64_t* in, uint64_t* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // < kThreads; in holds 2 kThreads
  uint64_t x = in[i], y = in[i + kThreads];
  uint64_t v[8];
  for (int k = 0; k < 8; ++k) v[k] = in[(i + 37 * k) & (kThreads - 1)];
#pragma unroll 1
  for (int it = 0; it < kIters; ++it) {
    if constexpr (OP == 0) x ^= y;
    if constexpr (OP == 1) x = gl::mul(x, y);
    if constexpr (OP == 2) x = gl::add(x, y);
    if constexpr (OP == 3) x = gl::sub(x, y);
    if constexpr (OP == 4) x = shl_c<24>(x);
    if constexpr (OP == 5) x = shl_c<48>(x);
    if constexpr (OP == 6) x = shl_c<72>(x);
    if constexpr (OP == 7) x = gl::mul_digit((int64_t)(int32_t)x, y);
    if constexpr (OP == 8) dif<8>(v);
    if constexpr (OP == 9) dit_inv<8>(v);
    if constexpr (OP == 10) {
      const uint64_t a = gl::add(x, y), b = gl::sub(x, y);
      x = a;
      y = b;
    }
  }
  uint64_t r = x;
  for (int k = 0; k < 8; ++k) r ^= v[k];
  out[i] = r;
}

}  // namespace

int main() {
  uint64_t *in = nullptr, *out = nullptr;
  if (cudaMalloc(&in, 2 * kThreads * sizeof(uint64_t)) != cudaSuccess ||
      cudaMalloc(&out, kThreads * sizeof(uint64_t)) != cudaSuccess) {
    std::printf("no device memory\n");
    return 1;
  }
  static uint64_t h[2 * kThreads];
  uint64_t s = 12345;
  for (auto& e : h) {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    e = s % gl::P;
  }
  cudaMemcpy(in, h, sizeof h, cudaMemcpyHostToDevice);
  probe<0><<<32, 128>>>(in, out);
  probe<1><<<32, 128>>>(in, out);
  probe<2><<<32, 128>>>(in, out);
  probe<3><<<32, 128>>>(in, out);
  probe<4><<<32, 128>>>(in, out);
  probe<5><<<32, 128>>>(in, out);
  probe<6><<<32, 128>>>(in, out);
  probe<7><<<32, 128>>>(in, out);
  probe<8><<<32, 128>>>(in, out);
  probe<9><<<32, 128>>>(in, out);
  probe<10><<<32, 128>>>(in, out);
  const cudaError_t e = cudaDeviceSynchronize();
  std::printf("opcount: %s\n", cudaGetErrorString(e));
  cudaFree(in);
  cudaFree(out);
  return e == cudaSuccess ? 0 : 1;
}
