// Deterministic block and grid reductions shared by the kernel files.
#pragma once
#include <cuda_runtime.h>

#include "fem_internal.h"

namespace femb200 {

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = (l < NT / 32) ? sh[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;  // valid in thread 0
}

// Publishes this block's partial(s) and reports whether it is the last block
// to arrive; the last block then owns the fixed-order final sum.
__device__ __forceinline__ bool publish_partial(const Reduce& red, int site, int nval,
                                                const double* vals, bool* am_last) {
  if (threadIdx.x == 0) {
    for (int v = 0; v < nval; ++v)
      red.partials[(size_t)(site * 2 + v) * red.max_blocks + blockIdx.x] = vals[v];
    __threadfence();
    unsigned int t = atomicAdd(&red.counters[site], 1u);
    *am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  return *am_last;
}

template <int NT>
__device__ __forceinline__ double final_sum(const Reduce& red, int site, int v, double* sh) {
  __threadfence();
  double acc = 0.0;
  const double* p = red.partials + (size_t)(site * 2 + v) * red.max_blocks;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += NT) acc += __ldcg(p + i);
  return block_sum<NT>(acc, sh);
}

}  // namespace femb200
