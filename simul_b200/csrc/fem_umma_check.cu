// Known-answer check of the tcgen05 path: one M = 128 tile
// D = A B^T (A: 128 x K, B: N x K, BF16 row-major in HBM, D FP32) through the
// same shared-memory layout, descriptors, TMEM allocation and epilogue loads
// the learned-preconditioner layers use.  Exposed as fem_selftest_umma so
// tests can compare it with a host product before the layers are trusted.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/femb200.h"
#include "fem_internal.h"
#include "fem_umma.cuh"

namespace femb200 {

constexpr int kMaxPolls = 1 << 22;

__global__ void __launch_bounds__(128) umma_check_kernel(const __nv_bfloat16* __restrict__ A,
                                                         const __nv_bfloat16* __restrict__ B, float* D,
                                                         int N, int K, int ncols, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  unsigned char* sA = smem;
  unsigned char* sB = smem + 128 * K * 2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) umma::tmem_alloc(&tmem_base, (uint32_t)ncols);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  for (int i = tid; i < 128 * K; i += 128) {
    const int row = i / K, k = i - row * K;
    *reinterpret_cast<__nv_bfloat16*>(sA + umma::kmajor_off(row, k, K)) = A[i];
  }
  for (int i = tid; i < N * K; i += 128) {
    const int row = i / K, k = i - row * K;
    *reinterpret_cast<__nv_bfloat16*>(sB + umma::kmajor_off(row, k, K)) = B[i];
  }
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (tid == 0) {
    const uint32_t idesc = umma::idesc_bf16(128, N);
    const uint32_t a0 = umma::smem_u32(sA), b0 = umma::smem_u32(sB);
    for (int s = 0; s < K / 16; ++s)
      umma::mma_bf16(tbase, umma::smem_desc(a0 + 256 * s, K), umma::smem_desc(b0 + 256 * s, K), idesc,
                     s > 0 ? 1u : 0u);
    umma::commit(&mbar);
  }
  __syncwarp();
  const bool ok = umma::mbar_wait(&mbar, 0, kMaxPolls);
  umma::fence_after_sync();
  if (ok) {
    const int row = 32 * warp + lane;
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      umma::tmem_ld16(umma::taddr(tbase, 32 * warp, c0), v);
#pragma unroll
      for (int j = 0; j < 16; ++j) D[(size_t)row * N + c0 + j] = v[j];
    }
  } else if (lane == 0) {
    atomicExch(err, 1);
  }
  umma::drain_mma(&mbar, 0, ok, kMaxPolls);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, (uint32_t)ncols);
}

}  // namespace femb200

using namespace femb200;

int fem_selftest_umma(const void* A, const void* B, float* D, int32_t N, int32_t K, void* stream) {
  if (!A || !B || !D) return set_global_error(FEM_ERR_INVALID, "null operand");
  if (N < 16 || N > 256 || N % 16 || K < 16 || K > 256 || K % 16)
    return set_global_error(FEM_ERR_INVALID, "N and K must be multiples of 16 in [16, 256] (got %d, %d)", N, K);
  int ncols = 32;
  while (ncols < N) ncols *= 2;
  const size_t smem = (size_t)(128 + N) * K * 2;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* err = nullptr;
  if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return set_global_error(FEM_ERR_CUDA, "cudaMalloc failed");
  cudaMemsetAsync(err, 0, sizeof(int), s);
  cudaFuncSetAttribute(umma_check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  umma_check_kernel<<<1, 128, smem, s>>>(static_cast<const __nv_bfloat16*>(A),
                                        static_cast<const __nv_bfloat16*>(B), D, N, K, ncols, err);
  cudaError_t e = cudaGetLastError();
  int h_err = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(err);
  if (e != cudaSuccess) return set_global_error(FEM_ERR_CUDA, "umma check: %s", cudaGetErrorString(e));
  if (h_err) return set_global_error(FEM_ERR_BUDGET, "umma check: MMA completion wait timed out");
  return FEM_OK;
}
