// Process-wide dynamic shared-memory limits of the library's kernels.
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

#include "fem_internal.h"

namespace femb200 {

void raise_smem_limit(const void* kernel) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (!done.insert({dev, kernel}).second) return;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

}  // namespace femb200
