// rf_fiber.hpp — batched stepping of an ensemble group (rf_fiber.cu): the items the variants' fibers
// file for a batched launch and the group that collects them.
#pragma once

#include <cuda_runtime.h>

#include <utility>
#include <vector>

namespace rf {

// Kinds of batched launches: the pressure BiCGStab and the block-ILU0 sweep (rf_level.cu), the
// block-ILU0 and pressure-ILU0 factorisation (rf_linear.cu).
constexpr int kBatchPressure = 0;
constexpr int kBatchBlockSweep = 1;
constexpr int kBatchFactor = 2;
constexpr int kBatchKinds = 3;
// Items per launch: the kernel parameter carries their arguments by value.
constexpr int kBatchItems = 24;
constexpr size_t kBatchArgBytes = 320;

struct BatchItem {
  int kind = 0;
  int type = 0;  // 0 double, 1 float
  int threads = 0;
  size_t smem = 0;
  alignas(16) unsigned char args[kBatchArgBytes];
};

struct BatchGroup {
  cudaStream_t stream = nullptr;
  std::vector<int> members;  // variant indices
  std::vector<BatchItem> pending;
  std::vector<char> stacks;
  bool failed = false;  // a batched launch failed (the step reports RF_ERR_CUDA)
  // launch counts always; opt-in timing of the batched launches (events on the group's stream)
  bool profiling = false;
  long long launches[kBatchKinds] = {}, items[kBatchKinds] = {};
  double ms_by_kind[kBatchKinds] = {};
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> timed;
  cudaEvent_t timing_event();
  void resolve_timing();
  void reset_stats();
  BatchGroup() = default;
  BatchGroup(const BatchGroup&) = delete;
  BatchGroup& operator=(const BatchGroup&) = delete;
  ~BatchGroup();
};

// File an item with the calling fiber's group and suspend until the group launches it; false
// (nothing filed) when the caller is not a batch fiber.
bool fiber_submit(const BatchItem& item);
// The same for launch arguments `args` (bytes <= kBatchArgBytes) of a kernel kind.
bool fiber_file(int kind, int type, const void* args, size_t bytes, int threads, size_t smem);
// Run fn(args[i]) for i < count as fibers on the calling thread until all have returned.
void run_fibers(BatchGroup& g, void (*fn)(void*), void* const* args, int count, size_t stack_bytes);
// One launch of `count` items of one kind and value type on `stream` (rf_level.cu); false when
// the launch failed.
bool launch_batch_items(int kind, int type, const BatchItem* const* items, int count, cudaStream_t stream);
// The factorisation's batched launch (rf_linear.cu).
bool launch_factor_batch(const BatchItem* const* items, int count, cudaStream_t stream);

}  // namespace rf
