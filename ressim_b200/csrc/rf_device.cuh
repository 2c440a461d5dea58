// rf_device.cuh — CUDA utilities shared by the kernels: error checks and deterministic block
// reductions.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace rf {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& m) : std::runtime_error(m) {}
};

#define RF_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      throw ::rf::CudaError(std::string(#call) + " failed: " + cudaGetErrorString(e_) + " at " + \
                            __FILE__ + ":" + std::to_string(__LINE__));                           \
  } while (0)

constexpr int kBlock = 256;
// Full systems of at most this many rows take the direct route (fim/linear/mod.rs:15).
constexpr int kDirectSolveRows = 512;

inline int blocks_for(long long n, int block = kBlock) {
  long long b = (n + block - 1) / block;
  if (b < 1) b = 1;
  return int(b);
}

// Block-wide sum of one double (fixed reduction tree: deterministic for a fixed launch shape).
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int t = threadIdx.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((t & 31) == 0) sh[t >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (t < 32) {
    r = (t < BLOCK / 32) ? sh[t] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

template <int BLOCK>
__device__ __forceinline__ double block_max(double v, double* sh) {
  const int t = threadIdx.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((t & 31) == 0) sh[t >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (t < 32) {
    r = (t < BLOCK / 32) ? sh[t] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
  }
  __syncthreads();
  return r;
}

}  // namespace rf
