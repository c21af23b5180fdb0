// Allocation-free canonical readout: lnt_canonicalize_noalloc.
//
// The canonical readout (lnt_canon.cu) needs per-block scratch (block carries,
// carry transfer functions, resolved carry-ins, a flag word).  The regular path
// keeps that scratch in each test's own cudaMalloc'd buffers.  Some callers
// cannot allocate device memory at the time they need a residue in the
// reference's digit format: a serving process whose HBM is entirely handed to
// its own pool or admission budget, a latency-critical step where cudaMalloc's
// implicit device synchronisation is unacceptable, or a checkpoint written by a
// path that must not allocate (outside the allocator's reach).  For them this entry point takes every buffer from the
// caller and keeps the scratch in one fixed array of device memory that belongs
// to the library: g_noalloc_scratch below, sized for residues of up to
// 2^24 words (about 2.5 MiB, held by every GPU that loads the library until the
// process exits).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/lucasntt.h"
#include "canon_core.cuh"
#include "lnt_internal.h"

namespace lnt {
void set_last_error(const std::string& msg);
}

namespace {

constexpr uint32_t kMaxLog2 = 24;
constexpr uint32_t kMaxWords = 1u << kMaxLog2;
constexpr uint32_t kBlock = 64;  // canon_block_size(n) for n >= 64
constexpr uint32_t kMaxBlocks = kMaxWords / kBlock;
constexpr size_t kCarryBytes = (size_t)kMaxBlocks * sizeof(int64_t);
constexpr size_t kFnOffset = kCarryBytes;
constexpr size_t kCinOffset = kFnOffset + kMaxBlocks;
constexpr size_t kFlagsOffset = kCinOffset + kMaxBlocks;  // 256-byte aligned
constexpr size_t kScratchBytes = kFlagsOffset + 256;

static_assert(kFlagsOffset % 256 == 0, "flag word alignment");

// Host code must not use this name as an address: it is a host-side stand-in.
// The device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// The device address of the scratch array on the current device (set-up on
// the first call per device).  The address is kept for the life of the process:
// a cudaDeviceReset (or anything else that tears down the device's primary
// context) invalidates it, and this entry point must not be called after one.
cudaError_t scratch_on_current_device(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

// The reference's choice between the two representations of 0 mod M, decided
// on the device from the readout flags (no host round trip): an LL residue of
// all-maximal digits is 0; a PRP residue of all-zero digits is M unless the
// test started from zero.
__global__ void noalloc_digit0_flag(const uint64_t* out, uint32_t* flags) {
  if (out[0] != 0) atomicOr(flags, 1u << 31);
}

__global__ void noalloc_fix_zero(uint64_t* out, const uint8_t* widths, uint32_t n,
                                 const uint32_t* flags, int prp, int zero_start) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t f = *flags;
  const bool all_max = !(f & lnt::kCanonNotAllMax);
  const bool all_zero = !(f & lnt::kCanonHighNonZero) && !(f & (1u << 31));
  if (!prp && all_max) out[j] = 0;
  if (prp && !zero_start && all_zero) out[j] = (1ull << widths[j]) - 1;
}

}  // namespace

extern "C" int lnt_canonicalize_noalloc(const int64_t* words, const uint8_t* widths, uint32_t n,
                                        int prp, int zero_start, uint64_t* digits,
                                        void* cuda_stream) {
  if (!words || !widths || !digits) {
    lnt::set_last_error("lnt_canonicalize_noalloc: null device pointer");
    return LNT_ERR_INVALID_ARGUMENT;
  }
  if (n < 2 || (n & (n - 1)) || n > kMaxWords) {
    lnt::set_last_error("lnt_canonicalize_noalloc: n must be a power of two in [2, 2^24] (" +
                        std::to_string(n) + " given)");
    return LNT_ERR_INVALID_ARGUMENT;
  }
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  cudaError_t e;
  if (s != nullptr) {
    // the scratch address is the current device's: the stream must be on it
    int cur = 0, sdev = 0;
    if ((e = cudaGetDevice(&cur)) != cudaSuccess || (e = cudaStreamGetDevice(s, &sdev)) != cudaSuccess) {
      lnt::set_last_error(std::string("lnt_canonicalize_noalloc: ") + cudaGetErrorString(e));
      return LNT_ERR_CUDA;
    }
    if (sdev != cur) {
      lnt::set_last_error("lnt_canonicalize_noalloc: the stream belongs to device " + std::to_string(sdev) +
                          ", the current device is " + std::to_string(cur));
      return LNT_ERR_INVALID_ARGUMENT;
    }
  }
  unsigned char* base = nullptr;
  e = scratch_on_current_device(&base);
  if (e != cudaSuccess) {
    lnt::set_last_error(std::string("lnt_canonicalize_noalloc: scratch set-up: ") +
                        cudaGetErrorString(e));
    return LNT_ERR_CUDA;
  }
  lnt::CanonDesc c{};
  c.x = words;
  c.carry = nullptr;
  c.widths = widths;
  c.out = digits;
  c.blk_carry = reinterpret_cast<int64_t*>(base);
  c.blk_fn = base + kFnOffset;
  c.blk_cin = reinterpret_cast<int8_t*>(base + kCinOffset);
  c.flags = reinterpret_cast<uint32_t*>(base + kFlagsOffset);
  c.n = n;
  c.block = lnt::canon_block_size(n);
  c.nblocks = n / c.block;
  // the array keeps the previous call's contents: the flag word must start at 0
  if ((e = cudaMemsetAsync(c.flags, 0, sizeof(uint32_t), s)) != cudaSuccess ||
      (e = lnt::launch_canonicalize(c, s)) != cudaSuccess) {
    lnt::set_last_error(std::string("lnt_canonicalize_noalloc: ") + cudaGetErrorString(e));
    return LNT_ERR_CUDA;
  }
  noalloc_digit0_flag<<<1, 1, 0, s>>>(digits, c.flags);
  noalloc_fix_zero<<<(n + 255) / 256, 256, 0, s>>>(digits, widths, n, c.flags, prp, zero_start);
  // the flag word comes back on the caller's stream (not the legacy stream,
  // which would wait for every blocking stream of the device)
  uint32_t flags = 0;
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(&flags, c.flags, sizeof(flags), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    lnt::set_last_error(std::string("lnt_canonicalize_noalloc: ") + cudaGetErrorString(e));
    return LNT_ERR_CUDA;
  }
  if (flags & lnt::kCanonError) {
    // `digits` is left partly written; lnt_get_digits of a test may still
    // succeed on such words (it falls back to an exact carry on the host)
    lnt::set_last_error("lnt_canonicalize_noalloc: words too far from normalised digits");
    return LNT_ERR_NUMERIC;
  }
  return LNT_OK;
}
