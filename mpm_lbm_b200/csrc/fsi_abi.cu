// ABI housekeeping: error strings and version.
#include <algorithm>
#include <cstring>
#include <string>

#include "common.cuh"

namespace fsi {
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
}  // namespace fsi

extern "C" int fsi_abi_version(void) { return FSI_ABI_VERSION; }

extern "C" int fsi_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return (int)fsi::g_last_error.size();
  const size_t n = std::min(len - 1, fsi::g_last_error.size());
  std::memcpy(buf, fsi::g_last_error.data(), n);
  buf[n] = 0;
  return (int)n;
}
