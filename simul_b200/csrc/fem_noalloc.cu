// Allocation-free FP64 dot product: fem_dot_f64_noalloc.
//
// Some callers of this library cannot call cudaMalloc: a host application that
// owns the device memory pool (a framework allocator that reserved all of HBM
// at start-up), a real-time loop that forbids allocation after initialisation,
// or a plug-in that must not create device allocations behind its host's back.
// A context (fem_ctx_create) allocates its scratch, so those callers get this
// one entry point instead.  It is the same deterministic two-level reduction
// the residual and CG kernels use for their FP64 dots and norms: every block
// sums a fixed tile in a fixed order, writes one partial, and the last block to
// finish adds the partials in index order.  Here the per-block partials and the
// arrival counter live in the file-scope array g_noalloc_scratch instead of
// context-owned memory.
//
// Limits and sharing:
//  - at most kMaxBlocks = 2048 blocks of kTile = 4096 elements, so
//    n <= 8,388,608; larger n is rejected with FEM_ERR_INVALID;
//  - the array (2048 partials + counter, about 16 KB) is held by every GPU that
//    loads the library until the process exits;
//  - the first call on a device looks up the array's device address there
//    (cudaGetSymbolAddress); make that first call before any stream capture;
//    the address is kept for the life of the process, so a cudaDeviceReset
//    (which unloads the module, and the array with it) must not be followed
//    by further calls;
//  - the reduction follows the solver's scheme (fixed-order per-block
//    partials, the last block adds them in index order) with its own
//    4096-element tiles, so its result agrees with the solver's norms to
//    rounding, not bit for bit;
//  - every call shares the array and it keeps the last call's contents; the
//    counter is cleared at the start of each call, the partials are
//    overwritten.  Calls that overlap on the GPU (two streams, or two host
//    threads issuing at once) race on the array and return wrong sums:
//    serialise them.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/femb200.h"
#include "fem_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;
constexpr int kMaxBlocks = 2048;
constexpr int64_t kMaxN = (int64_t)kMaxBlocks * kTile;
constexpr int kScratchWords = kMaxBlocks + 32;  // partials, then the counter word

static __device__ __align__(256) double g_noalloc_scratch[kScratchWords];

__global__ void __launch_bounds__(kThreads) dot_noalloc_kernel(const double* __restrict__ a,
                                                               const double* __restrict__ b,
                                                               int64_t n, double* scratch,
                                                               double* out) {
  __shared__ double sh[kThreads / 32];
  __shared__ bool am_last;
  unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + kMaxBlocks);
  const int64_t base = (int64_t)blockIdx.x * kTile;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const int64_t i = base + (int64_t)k * kThreads + threadIdx.x;
    if (i < n) acc += a[i] * b[i];
  }
  auto block_sum = [&](double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
      r = (l < kThreads / 32) ? sh[l] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
  };
  const double part = block_sum(acc);
  if (threadIdx.x == 0) {
    scratch[blockIdx.x] = part;
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double tot = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads) tot += __ldcg(scratch + i);
  tot = block_sum(tot);
  if (threadIdx.x == 0) {
    *out = tot;
    *counter = 0u;
  }
}

std::mutex g_mu;
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {};

}  // namespace

extern "C" int fem_dot_f64_noalloc(const double* a, const double* b, int64_t n, double* result,
                                   void* stream) {
  using femb200::set_global_error;
  if (!a || !b || !result) return set_global_error(FEM_ERR_INVALID, "fem_dot_f64_noalloc: null pointer");
  if (n < 0 || n > kMaxN)
    return set_global_error(FEM_ERR_INVALID,
                            "fem_dot_f64_noalloc: n = %lld outside [0, %lld], the allocation-free maximum",
                            (long long)n, (long long)kMaxN);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return set_global_error(FEM_ERR_CUDA, "fem_dot_f64_noalloc: cudaGetDevice failed (%s)",
                            cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return set_global_error(FEM_ERR_INVALID,
                            "fem_dot_f64_noalloc: device ordinal %d exceeds the allocation-free limit of %d devices",
                            dev, kMaxDevices);
  double* scratch;
  {
    // set-up, once per device, with that device current: the host-side symbol
    // is a stand-in, the kernel needs the array's device address
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return set_global_error(FEM_ERR_CUDA, "fem_dot_f64_noalloc: cudaGetSymbolAddress failed (%s)",
                                cudaGetErrorString(e));
      g_scratch_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  if (n == 0) {
    e = cudaMemsetAsync(result, 0, sizeof(double), s);
    if (e != cudaSuccess)
      return set_global_error(FEM_ERR_CUDA, "fem_dot_f64_noalloc: %s", cudaGetErrorString(e));
    return FEM_OK;
  }
  // the arrival counter must start at zero; the partials are overwritten
  e = cudaMemsetAsync(scratch + kMaxBlocks, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess)
    return set_global_error(FEM_ERR_CUDA, "fem_dot_f64_noalloc: %s", cudaGetErrorString(e));
  const int grid = (int)((n + kTile - 1) / kTile);
  dot_noalloc_kernel<<<grid, kThreads, 0, s>>>(a, b, n, scratch, result);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_global_error(FEM_ERR_CUDA, "fem_dot_f64_noalloc: launch failed (%s)", cudaGetErrorString(e));
  return FEM_OK;
}
