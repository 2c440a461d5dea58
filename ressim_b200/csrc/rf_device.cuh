// rf_device.cuh — CUDA utilities shared by the kernels: error checks, deterministic block
// reductions and a bounded software grid barrier for cooperative (co-resident) launches.
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

inline int blocks_for(long long n, int block = kBlock) {
  long long b = (n + block - 1) / block;
  if (b < 1) b = 1;
  return int(b);
}

// Device status word written by bounded waits and checks.  Nonzero means a kernel gave up a
// wait (code 1) or detected an inconsistency; the host reads it after each solve.
struct DeviceStatus {
  int code;
  int where;
};

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

// Software grid barrier for cooperative launches (all blocks co-resident).  `count` is a 64-bit
// arrival counter set to zero before each launch (stream-ordered memset); barrier k of a launch
// completes when it reaches (k + 1) * gridDim.x.  Arrival is a release reduction and the wait an
// acquire load followed by a fence, so the block's writes before the barrier are visible to every
// block's plain loads after it.  The
// spin is bounded: after kBarrierPollLimit polls it records code 1 in `status` and releases; once
// the status is set every later barrier returns at once, so a failed launch runs its bounded
// loops to the end instead of hanging, and the host reports the failure after the launch.
struct GridBarrier {
  unsigned long long* count;
  volatile DeviceStatus* status;
};

constexpr long long kBarrierPollLimit = 1ll << 24;

__device__ __forceinline__ void grid_sync(const GridBarrier& b, unsigned long long& target, int where) {
  __syncthreads();
  target += gridDim.x * gridDim.y * gridDim.z;
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(b.count) : "memory");
    if (b.status->code == 0) {
      long long polls = 0;
      while (true) {
        unsigned long long v;
        asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(b.count) : "memory");
        if (v >= target) break;
        if ((++polls & 255) == 0) {
          if (b.status->code != 0) break;
          if (polls > kBarrierPollLimit) {
            b.status->where = where;
            b.status->code = 1;
            break;
          }
        }
      }
    }
    // make every thread's later plain loads see the other blocks' writes (L1 is not coherent)
    __threadfence();
  }
  __syncthreads();
}

}  // namespace rf
