// ABI housekeeping: error strings and version.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>

#include "common.cuh"

namespace fsi {
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int device_sm_count() {
  static std::atomic<int> cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  int n = cached[dev].load(std::memory_order_relaxed);
  if (n <= 0) {
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cached[dev].store(n, std::memory_order_relaxed);
  }
  return n;
}
}  // namespace fsi

extern "C" uint64_t fsi_launch_count(void) { return fsi::g_launches.load(std::memory_order_relaxed); }

extern "C" int fsi_abi_version(void) { return FSI_ABI_VERSION; }

extern "C" int fsi_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return (int)fsi::g_last_error.size();
  const size_t n = std::min(len - 1, fsi::g_last_error.size());
  std::memcpy(buf, fsi::g_last_error.data(), n);
  buf[n] = 0;
  return (int)n;
}
