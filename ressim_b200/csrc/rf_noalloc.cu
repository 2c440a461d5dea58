// rf_noalloc.cu — a dense pressure solve for callers that may not allocate device memory.
//
// Some hosts cannot call cudaMalloc while they run: an application that reserves its whole
// device-memory budget at start-up and hands it to its own pool, an embedding framework whose
// allocator owns the GPU, or a time-critical loop that must not block, since cudaMalloc and
// cudaFree can synchronise the device.  For them this file offers x = A^{-1} b for a dense
// row-major n x n pressure matrix, n <= RF_NOALLOC_MAX_ROWS (299, the size up to which the
// reference's CPR inverts its pressure block densely, gmres_block_jacobi.rs:903-917).  It runs
// the same kernels as a context's CPR coarse stage (k_dense_lu and k_dense_inv_cols, the inverse
// by LU with partial pivoting in nalgebra's order, then k_dense_matvec), with all scratch (the LU
// work copy, the inverse, the row permutation and a status word) in one file-scope static device
// array.  The caller passes A, b
// and x in device memory; the call itself allocates nothing, on the device or the host.
//
// The array is part of the loaded library, so every GPU that loads it keeps about 1.4 MB for it
// until the process exits.  Host code may not pass the array's name to a kernel (on the host it is
// only a stand-in symbol): the first call on each device, with that device current, looks up the
// device address with cudaGetSymbolAddress and keeps it.  Every call synchronises its stream and
// reads a status word back into host memory, so no call may be made while its stream is being
// captured into a CUDA graph.  All calls share the one array and it keeps the previous call's
// contents: the status word is cleared on every call, everything else is overwritten before it is
// read.  Calls that overlap on the GPU (other host threads, or unordered streams) race on the
// array; serialise them.  When a pivot is exactly zero the call fails and leaves x as it was.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/ressim_fim.h"

namespace rf {
void dense_invert_launch(int n, double* a, double* inv, int* perm, int* ok, cudaStream_t stream);
__global__ void k_dense_matvec(int n, const double* __restrict__ a, const double* __restrict__ x,
                               double* __restrict__ y, const int* __restrict__ ok);
}  // namespace rf

namespace {

constexpr int kMaxRows = RF_NOALLOC_MAX_ROWS;
constexpr size_t kMat = size_t(kMaxRows) * kMaxRows;
// [LU work copy: kMat doubles][inverse: kMat doubles][permutation: kMaxRows ints][status: 1 int]
constexpr size_t kScratchBytes = 2 * kMat * sizeof(double) + (kMaxRows + 1) * sizeof(int);

static __device__ __align__(256) unsigned char g_dense_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
static void* g_scratch_addr[kMaxDevices] = {};
static std::mutex g_setup_mu;

int32_t report(char* err, size_t len, int32_t code, const char* msg) {
  if (err && len) std::snprintf(err, len, "%s", msg);
  return code;
}

}  // namespace

extern "C" int32_t rf_dense_solve_noalloc(int32_t n, const double* a, const double* b, double* x, void* stream,
                                          char* err, size_t err_len) {
  if (n < 1 || n > kMaxRows) {
    char msg[160];
    std::snprintf(msg, sizeof msg,
                  "rf_dense_solve_noalloc: n = %d is outside 1..%d (the fixed scratch holds at most %d rows)",
                  int(n), kMaxRows, kMaxRows);
    return report(err, err_len, RF_ERR_INVALID, msg);
  }
  if (!a || !b || !x) return report(err, err_len, RF_ERR_INVALID, "rf_dense_solve_noalloc: null device pointer");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return report(err, err_len, RF_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return report(err, err_len, RF_ERR_INVALID, "rf_dense_solve_noalloc: device index out of range");
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_dense_scratch);
      if (e != cudaSuccess) return report(err, err_len, RF_ERR_CUDA, cudaGetErrorString(e));
      g_scratch_addr[dev] = p;
    }
    base = g_scratch_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* lu = static_cast<double*>(base);
  double* inv = lu + kMat;
  int* perm = reinterpret_cast<int*>(inv + kMat);
  int* status = perm + kMaxRows;
  // the LU factorisation works in place, so it runs on a copy of A; the status word must start
  // at zero (the kernel writes 1 on success and 0 on an exactly zero pivot)
  if ((e = cudaMemcpyAsync(lu, a, sizeof(double) * size_t(n) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(status, 0, sizeof(int), s)) != cudaSuccess)
    return report(err, err_len, RF_ERR_CUDA, cudaGetErrorString(e));
  rf::dense_invert_launch(n, lu, inv, perm, status, s);
  // the product skips its writes when the factorisation failed, so x keeps the caller's values
  rf::k_dense_matvec<<<(n + 63) / 64, 64, 0, s>>>(n, inv, b, x, status);
  if ((e = cudaGetLastError()) != cudaSuccess) return report(err, err_len, RF_ERR_CUDA, cudaGetErrorString(e));
  int ok = 0;
  if ((e = cudaMemcpyAsync(&ok, status, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return report(err, err_len, RF_ERR_CUDA, cudaGetErrorString(e));
  if (!ok) return report(err, err_len, RF_ERR_INVALID, "rf_dense_solve_noalloc: the matrix is singular (zero pivot)");
  return RF_OK;
}
