// Per-device properties the launchers size their grids by, queried once per
// device and cached (launches made while a stream is captured into a graph
// then issue no attribute queries).
#include <map>
#include <mutex>

#include "lnt_internal.h"

namespace lnt {

cudaError_t device_info(DeviceInfo& out) {
  static std::mutex mu;
  static std::map<int, DeviceInfo> cache;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(dev);
  if (it == cache.end()) {
    DeviceInfo d;
    if ((e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&d.smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) !=
            cudaSuccess ||
        (e = cudaDeviceGetAttribute(&d.smem_per_block_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                    dev)) != cudaSuccess)
      return e;
    it = cache.emplace(dev, d).first;
  }
  out = it->second;
  return cudaSuccess;
}

uint32_t device_sms() {
  DeviceInfo d;
  return device_info(d) == cudaSuccess && d.sms > 0 ? (uint32_t)d.sms : 148u;
}

}  // namespace lnt
