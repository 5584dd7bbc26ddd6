// Shared host/device helpers: error reporting, launch checks, atomics.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>

#include "../../include/fsi_b200.h"

namespace fsi {

void set_error(const std::string& msg);
// counts kernel launches issued through this library (see fsi_launch_count)
void count_launch();
// SMs of the current device (148 on B200; queried once per device)
int device_sm_count();

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
// Programmatic dependent launch (sm_90+): a kernel launched with
// launch_pdl() may be scheduled while the kernel before it in the stream is
// still running; it must call griddep_wait() before touching memory that
// kernel writes (the wait returns once that grid has completed and its writes
// are visible; in a kernel launched normally it returns at once).
// griddep_launch() lets the next such kernel be scheduled; every CTA calls it
// after its own wait, so the chain never runs more than one grid ahead.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

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

#if defined(__CUDACC__)
// launch with programmatic stream serialization (see griddep_wait)
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
#endif

}  // namespace fsi
