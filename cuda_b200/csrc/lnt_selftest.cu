// Device arithmetic self-test: lnt_arith_selftest.
//
// The kernels reduce modulo p = 2^64 - 2^32 + 1 with PTX carry chains and
// multiplier-pipe sums (goldilocks.cuh reduce_words / reduce_words3, the shift
// twiddles of ntt_core.cuh).  Some of their branches are rare on residue data:
// a word >= p before the canonical step, a carry and a borrow in the same
// reduction, a digit product whose fold carries.  Random residues reach each
// about once in 2^32 operations.  This entry point runs the device functions
// on operands chosen to reach those branches (0, 1, p - 1, the 2^32 and 2^63
// boundaries, values just below p, products with all-ones high words) and on
// seeded random operands.  It compares every result with the host build of the
// same function: the portable C path, which the CPU tests check against the
// oracle and an independent 128-bit implementation.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/lucasntt.h"
#include "goldilocks.cuh"
#include "lnt_internal.h"
#include "ntt_core.cuh"

namespace {

// results per operand pair: mul, add, sub, ten shifts, three digit products
constexpr int kOps = 16;

template <unsigned S>
__host__ __device__ uint64_t shift_op(uint64_t x) {
  return lnt::shl_c<S>(x);
}

__host__ __device__ void arith_ops(uint64_t a, uint64_t b, uint64_t* r) {
  r[0] = gl::mul(a, b);
  r[1] = gl::add(a, b);
  r[2] = gl::sub(a, b);
  r[3] = shift_op<3>(a);
  r[4] = shift_op<24>(a);
  r[5] = shift_op<32>(a);
  r[6] = shift_op<45>(a);
  r[7] = shift_op<48>(a);
  r[8] = shift_op<64>(a);
  r[9] = shift_op<72>(a);
  r[10] = shift_op<95>(a);
  r[11] = shift_op<120>(a);
  r[12] = shift_op<168>(a);
  // digits |d| < 2^32: the low word of b as signed, as unsigned, and negated
  const uint32_t b0 = (uint32_t)b;
  r[13] = gl::mul_digit((int64_t)(int32_t)b0, a);
  r[14] = gl::mul_digit((int64_t)b0, a);
  r[15] = gl::mul_digit(-(int64_t)b0, a);
}

__global__ void arith_selftest_kernel(const uint64_t* a, const uint64_t* b, uint32_t count,
                                      uint64_t* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) arith_ops(a[i], b[i], out + (size_t)i * kOps);
}

// operands that reach the rare branches of the reductions
std::vector<uint64_t> edge_values() {
  const uint64_t P = gl::P;
  return {0ull,
          1ull,
          2ull,
          3ull,
          0x7FFFFFFFull,
          0x80000000ull,
          0xFFFFFFFEull,
          0xFFFFFFFFull,
          0x100000000ull,
          0x100000001ull,
          0x1FFFFFFFFull,
          0x7FFFFFFFFFFFFFFFull,
          0x8000000000000000ull,
          0xFFFFFFFE00000000ull,
          0xFFFFFFFE00000001ull,
          0xFFFFFFFEFFFFFFFFull,
          P - 0x100000000ull,
          P - 3,
          P - 2,
          P - 1,
          0xFFFFFFFF00000000ull,  // p - 1
          0x00000000FFFFFFFFull * 0x10001ull,
          0x0000FFFF0000FFFFull,
          0xAAAAAAAAAAAAAAAAull % P,
          0x5555555555555555ull};
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

namespace lnt {
void set_last_error(const std::string& msg);
}

extern "C" int lnt_arith_selftest(int device, uint64_t* checked, uint64_t* mismatches) {
  if (!checked || !mismatches) {
    lnt::set_last_error("lnt_arith_selftest: null argument");
    return LNT_ERR_INVALID_ARGUMENT;
  }
  *checked = *mismatches = 0;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    lnt::set_last_error("lnt_arith_selftest: no CUDA device");
    return LNT_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) {
    lnt::set_last_error("lnt_arith_selftest: no such device");
    return LNT_ERR_INVALID_ARGUMENT;
  }
  // every pair of edge values, then seeded random pairs: uniform field
  // elements, values within 2^33 of p, and small values
  const std::vector<uint64_t> edge = edge_values();
  std::vector<uint64_t> a, b;
  for (uint64_t x : edge)
    for (uint64_t y : edge) {
      a.push_back(x);
      b.push_back(y);
    }
  uint64_t s = 0x4C75636173ull;
  for (int i = 0; i < 3 * 8192; ++i) {
    uint64_t x = splitmix(s), y = splitmix(s);
    switch (i % 3) {
      case 0: x %= gl::P; y %= gl::P; break;
      case 1: x = gl::P - 1 - (x >> 31); y = gl::P - 1 - (y >> 31); break;
      default: x >>= 30; y %= gl::P; break;
    }
    a.push_back(x);
    b.push_back(y);
  }
  const uint32_t n = (uint32_t)a.size();
  std::vector<uint64_t> got((size_t)n * kOps);

  cudaError_t e = cudaSetDevice(device);
  uint64_t *da = nullptr, *db = nullptr, *dout = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&da, n * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMalloc(&db, n * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMalloc(&dout, got.size() * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMemcpy(da, a.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(db, b.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    arith_selftest_kernel<<<(n + 255) / 256, 256>>>(da, db, n, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(got.data(), dout, got.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost);
  cudaFree(da);
  cudaFree(db);
  cudaFree(dout);
  if (e != cudaSuccess) {
    lnt::set_last_error(std::string("lnt_arith_selftest: ") + cudaGetErrorString(e));
    return LNT_ERR_CUDA;
  }

  std::string first;
  uint64_t bad = 0;
  for (uint32_t i = 0; i < n; ++i) {
    uint64_t want[kOps];
    arith_ops(a[i], b[i], want);
    for (int k = 0; k < kOps; ++k)
      if (got[(size_t)i * kOps + k] != want[k]) {
        if (bad++ == 0) {
          char line[160];
          std::snprintf(line, sizeof line,
                        "op %d of a = %016llx, b = %016llx: device %016llx, host %016llx", k,
                        (unsigned long long)a[i], (unsigned long long)b[i],
                        (unsigned long long)got[(size_t)i * kOps + k], (unsigned long long)want[k]);
          first = line;
        }
      }
  }
  *checked = (uint64_t)n * kOps;
  *mismatches = bad;
  if (bad) {
    lnt::set_last_error("lnt_arith_selftest: " + std::to_string(bad) + " mismatches; first: " + first);
    return LNT_ERR_NUMERIC;
  }
  return LNT_OK;
}
