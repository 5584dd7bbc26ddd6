// Shared host/device helpers: error reporting, launch checks, atomics.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/fsi_b200.h"

namespace fsi {

void set_error(const std::string& msg);
// counts kernel launches issued through this library (see fsi_launch_count)
void count_launch();

inline int cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FSI_OK;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return FSI_E_CUDA;
}

// every kernel launch of the library is followed by exactly one launch_check
inline int launch_check(const char* what) {
  const int rc = cuda_check(cudaGetLastError(), what);
  if (rc == FSI_OK) count_launch();
  return rc;
}

inline int invalid(const std::string& msg) {
  set_error(msg);
  return FSI_E_INVALID;
}

#if defined(__CUDACC__)
// max of non-negative floats through their integer bit patterns
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
  atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
#endif

}  // namespace fsi
