// Fused PCG step: everything one CG iteration does after the tangent matvec,
// as ONE cooperative kernel instead of a chain of small launches.
//
// At the sizes of the hot path (1e5 - 1e6 nodes) every vector pass of CG is
// L2-resident and takes a few microseconds, so a chain of six dependent
// launches (update, restriction, coarse residual, coarse product, z and r.z,
// direction update) costs more in launch gaps, ramp-up and tails than in
// work.  Here the chain runs inside one grid of 1-2 CTAs per SM, launched
// cooperatively (all CTAs resident), with a grid-wide barrier between the
// phases that depend on a global result.  Every wait is bounded (2 s); a CTA
// that gives up marks the CG state broken down (status 5) and returns, and
// the host reports the solve as failed.
//
// Reductions stay deterministic: every partial sum covers a fixed set of
// nodes (one lattice-cell slice, or one chunk of kStepThreads nodes) and the
// partials are added in index order, so results do not depend on which CTA
// ran which piece.  Data written inside the kernel is read back through L2
// (ld.global.cg) because L1 is not coherent across SMs.
//
// No reference counterpart: the reference solves the assembled system with
// spsolve / ILU-CG (backend/fea/fem/solver/static_solver.py:399-462).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "fem_internal.h"
#include "fem_lattice.cuh"

namespace femb200 {

namespace {

constexpr int kStepWarps = kStepThreads / 32;
constexpr unsigned long long kBarrierNs = 2000000000ull;  // 2 s
constexpr int kMaxSlices = 8;

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier of a cooperative launch.  bar[0] counts arrivals, bar[1]
// is the generation: the last CTA to arrive resets the count, then advances
// the generation; the others wait for the generation to move.  Returns false
// when the wait ran out (the CG state is then marked broken down).
__device__ bool grid_sync(unsigned int* bar, CGState* cg) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int gen = ld_acquire(bar + 1);
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      for (unsigned int k = 1;; ++k) {
        if (ld_acquire(bar + 1) != gen) break;
        if ((k & 63u) == 0 && global_ns() - t0 > kBarrierNs) {
          cg->status = 5;
          atomicExch(&cg->done, 3);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the CTA in a fixed order, returned to every thread.
__device__ __forceinline__ double block_total(double v, double* sh) {
  v = warp_sum_d(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int k = 0; k < kStepWarps; ++k) t += sh[k];
  return t;
}

// Sum of part[0 .. n) in index order (strided per thread, then the fixed
// block order), returned to every thread of the CTA.
__device__ __forceinline__ double ordered_total(const double* part, int n, double* sh) {
  double v = 0.0;
  for (int k = threadIdx.x; k < n; k += kStepThreads) v += __ldcg(part + k);
  return block_total(v, sh);
}

__global__ void __launch_bounds__(kStepThreads) tl_step_kernel(const __grid_constant__ StepArgs a) {
  CGState* cg = a.cg;
  if (*(volatile int*)&cg->done) return;
  extern __shared__ __align__(16) float s_rc[];
  __shared__ double s_red[kStepWarps];
  const CoarseDev& c = a.c;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gwarp = blockIdx.x * kStepWarps + warp, n_gwarps = gridDim.x * kStepWarps;
  const float alpha = (float)cg->alpha;
  const double rz_old = cg->rz;
  const int iter_new = cg->iter + 1;
  float4* x4 = reinterpret_cast<float4*>(a.x);
  float4* r4 = reinterpret_cast<float4*>(a.r);
  float4* p4 = reinterpret_cast<float4*>(a.p);
  float4* z4 = reinterpret_cast<float4*>(a.z);
  const float4* q4 = reinterpret_cast<const float4*>(a.q);
  const float4* d4 = reinterpret_cast<const float4*>(a.dinv);
  const int S = c.r_slices;
  const int n_items = c.n_cells * S;

  // A: x += alpha p, r -= alpha q over each cell's nodes; per (cell, slice)
  // warp: ||r||^2 share and the 24 restriction shares of the new r
  for (int item = gwarp; item < n_items; item += n_gwarps) {
    const int cell = item / S, sl = item - cell * S;
    const int3 ijk = c.cell_ijk[cell];
    const int n0 = c.cell_node_ptr[cell], n1 = c.cell_node_ptr[cell + 1];
    float acc[24];
#pragma unroll
    for (int k = 0; k < 24; ++k) acc[k] = 0.f;
    double rr = 0.0;
    for (int i = n0 + 32 * sl + lane; i < n1; i += 32 * S) {
      const int node = __ldg(c.cell_nodes + i);
      float4 xv = __ldcg(x4 + node), rv = __ldcg(r4 + node);
      const float4 pv = __ldcg(p4 + node), qv = __ldcg(q4 + node);
      xv.x += alpha * pv.x; xv.y += alpha * pv.y; xv.z += alpha * pv.z;
      rv.x -= alpha * qv.x; rv.y -= alpha * qv.y; rv.z -= alpha * qv.z;
      __stcg(x4 + node, xv);
      __stcg(r4 + node, rv);
      rr += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z;
      const float4 X = __ldg(a.m.X32 + node);
      float t[3];
      cell_local(c, ijk, X.x, X.y, X.z, t);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float w = tri_weight(t[0], t[1], t[2], k);
        acc[3 * k] += w * rv.x;
        acc[3 * k + 1] += w * rv.y;
        acc[3 * k + 2] += w * rv.z;
      }
    }
    float mine = 0.f;
#pragma unroll
    for (int k = 0; k < 24; ++k) {
      const float v = warp_sum_f(acc[k]);
      if (lane == k) mine = v;
    }
    rr = warp_sum_d(rr);
    if (lane < 24) __stcg(c.cell_r + (size_t)item * 24 + lane, mine);
    if (lane == 0) __stcg(a.part + item, rr);
  }
  if (!grid_sync(a.bar, cg)) return;

  // B: coarse residual r_c, one warp per coarse node: lane 4k + j adds the
  // node's k-th cell share over slices j, j + 4, ...; a fixed butterfly
  // combines the lanes.  CTA 0 adds the ||r||^2 shares and runs the
  // convergence test.
  for (int cn = gwarp; cn < c.n_cn; cn += n_gwarps) {
    const int ent = __ldg(c.cn_cells + cn * 8 + (lane >> 2));
    float v0 = 0.f, v1 = 0.f, v2 = 0.f;
    if (ent >= 0) {
      const float* src = c.cell_r + (size_t)(ent >> 3) * S * 24 + 3 * (ent & 7);
      for (int sl = lane & 3; sl < S; sl += 4) {
        const float* q = src + (size_t)sl * 24;
        v0 += __ldcg(q);
        v1 += __ldcg(q + 1);
        v2 += __ldcg(q + 2);
      }
    }
    v0 = warp_sum_f(v0);
    v1 = warp_sum_f(v1);
    v2 = warp_sum_f(v2);
    if (lane < 3) __stcg(c.rc + 3 * cn + lane, lane == 0 ? v0 : (lane == 1 ? v1 : v2));
  }
  if (blockIdx.x == 0) {
    const double trr = ordered_total(a.part, n_items, s_red);
    if (threadIdx.x == 0) {
      cg->rr = trr;
      cg->iter = iter_new;
      if (!isfinite(trr)) {
        cg->done = 3;
        cg->status = 3;
      } else if (trr <= cg->tol2) {
        cg->done = 1;
      } else if (iter_new >= cg->max_iter) {
        cg->done = 2;
      }
    }
  }
  if (!grid_sync(a.bar, cg)) return;
  if (*(volatile int*)&cg->done) return;

  // C: y_c = Ainv r_c (FP32 inverse), r_c staged in shared memory, one warp
  // per row
  const int n = c.n_dof;
  for (int k = threadIdx.x; k < n; k += kStepThreads) s_rc[k] = __ldcg(c.rc + k);
  __syncthreads();
  for (int row = gwarp; row < n; row += n_gwarps) {
    float s0 = 0.f, s1 = 0.f;
    {
      const float* Arow = c.Ainv + (size_t)row * n;
      int j = lane;
      for (; j + 32 < n; j += 64) {
        s0 += __ldg(Arow + j) * s_rc[j];
        s1 += __ldg(Arow + j + 32) * s_rc[j + 32];
      }
      if (j < n) s0 += __ldg(Arow + j) * s_rc[j];
    }
    float s = s0 + s1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) __stcg(c.yc + row, s);
  }
  if (!grid_sync(a.bar, cg)) return;

  // D: z = D^-1 r + P y_c (zero on fixed DOFs); r.z share per chunk of
  // kStepThreads nodes
  double* rz_part = a.part + n_items;
  const int Nn = a.m.n_nodes;
  for (int base = blockIdx.x * kStepThreads; base < Nn; base += gridDim.x * kStepThreads) {
    const int i = base + threadIdx.x;
    double rz = 0.0;
    if (i < Nn) {
      const float4 rv = __ldcg(r4 + i);
      const float4 dv = __ldg(d4 + i);
      float t[3];
      const int cell = node_lattice(c, i, t);
      float cz[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int cnode = __ldg(c.cell_corner + cell * 8 + k);
        const float w = tri_weight(t[0], t[1], t[2], k);
        cz[0] += w * __ldcg(c.yc + 3 * cnode);
        cz[1] += w * __ldcg(c.yc + 3 * cnode + 1);
        cz[2] += w * __ldcg(c.yc + 3 * cnode + 2);
      }
      const int fx = (int)a.m.fixed[i];
      float4 zv;
      zv.x = (fx & 1) ? 0.f : dv.x * rv.x + cz[0];
      zv.y = (fx & 2) ? 0.f : dv.y * rv.y + cz[1];
      zv.z = (fx & 4) ? 0.f : dv.z * rv.z + cz[2];
      zv.w = 0.f;
      __stcg(z4 + i, zv);
      rz = (double)rv.x * zv.x + (double)rv.y * zv.y + (double)rv.z * zv.z;
    }
    const double v = block_total(rz, s_red);
    if (threadIdx.x == 0) __stcg(rz_part + base / kStepThreads, v);
  }
  if (!grid_sync(a.bar, cg)) return;

  // E: every CTA adds the r.z shares in order (same value everywhere):
  // beta = rz_new / rz_old (Fletcher-Reeves), p = z + beta p
  const double trz = ordered_total(rz_part, a.n_chunks, s_red);
  const float beta = (float)(trz / rz_old);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    cg->beta = trz / rz_old;
    cg->rz = trz;
    if (!isfinite(trz) || !(trz > 0.0)) {
      cg->done = 3;
      cg->status = 3;
    }
  }
  const int gt = blockIdx.x * kStepThreads + threadIdx.x, n_gt = gridDim.x * kStepThreads;
  for (int i = gt; i < Nn; i += n_gt) {
    float4 pv = __ldcg(p4 + i);
    const float4 zv = __ldcg(z4 + i);
    pv.x = zv.x + beta * pv.x;
    pv.y = zv.y + beta * pv.y;
    pv.z = zv.z + beta * pv.z;
    __stcg(p4 + i, pv);
  }
}

__global__ void __launch_bounds__(kStepThreads) jacobi_step_kernel(const __grid_constant__ StepArgs a) {
  CGState* cg = a.cg;
  if (*(volatile int*)&cg->done) return;
  __shared__ double s_red[kStepWarps];
  const float alpha = (float)cg->alpha;
  const double rz_old = cg->rz, tol2 = cg->tol2;
  const int iter_new = cg->iter + 1, max_iter = cg->max_iter;
  float4* x4 = reinterpret_cast<float4*>(a.x);
  float4* r4 = reinterpret_cast<float4*>(a.r);
  float4* p4 = reinterpret_cast<float4*>(a.p);
  const float4* q4 = reinterpret_cast<const float4*>(a.q);
  const float4* d4 = reinterpret_cast<const float4*>(a.dinv);
  const int Nn = a.m.n_nodes;
  double* rr_part = a.part;
  double* rz_part = a.part + a.n_chunks;

  // A: x += alpha p, r -= alpha q; ||r||^2 and r.D^-1 r per chunk
  for (int base = blockIdx.x * kStepThreads; base < Nn; base += gridDim.x * kStepThreads) {
    const int i = base + threadIdx.x;
    double rr = 0.0, rz = 0.0;
    if (i < Nn) {
      float4 xv = __ldcg(x4 + i), rv = __ldcg(r4 + i);
      const float4 pv = __ldcg(p4 + i), qv = __ldcg(q4 + i), dv = __ldg(d4 + i);
      xv.x += alpha * pv.x; xv.y += alpha * pv.y; xv.z += alpha * pv.z;
      rv.x -= alpha * qv.x; rv.y -= alpha * qv.y; rv.z -= alpha * qv.z;
      __stcg(x4 + i, xv);
      __stcg(r4 + i, rv);
      rr = (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z;
      rz = (double)rv.x * (dv.x * rv.x) + (double)rv.y * (dv.y * rv.y) + (double)rv.z * (dv.z * rv.z);
    }
    const double vr = block_total(rr, s_red);
    const double vz = block_total(rz, s_red);
    if (threadIdx.x == 0) {
      __stcg(rr_part + base / kStepThreads, vr);
      __stcg(rz_part + base / kStepThreads, vz);
    }
  }
  if (!grid_sync(a.bar, cg)) return;

  // B: every CTA adds the shares in order and takes the same decision
  const double trr = ordered_total(rr_part, a.n_chunks, s_red);
  const double trz = ordered_total(rz_part, a.n_chunks, s_red);
  int done = 0;
  if (!isfinite(trr) || !isfinite(trz)) done = 3;
  else if (trr <= tol2) done = 1;
  else if (iter_new >= max_iter) done = 2;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    cg->rr = trr;
    cg->iter = iter_new;
    cg->beta = trz / rz_old;
    cg->rz = trz;
    if (done == 3) cg->status = 3;
    if (done) cg->done = done;
  }
  if (done) return;
  const float beta = (float)(trz / rz_old);
  const int gt = blockIdx.x * kStepThreads + threadIdx.x, n_gt = gridDim.x * kStepThreads;
  for (int i = gt; i < Nn; i += n_gt) {
    float4 pv = __ldcg(p4 + i);
    const float4 rv = __ldcg(r4 + i), dv = __ldg(d4 + i);
    pv.x = dv.x * rv.x + beta * pv.x;
    pv.y = dv.y * rv.y + beta * pv.y;
    pv.z = dv.z * rv.z + beta * pv.z;
    __stcg(p4 + i, pv);
  }
}

size_t tl_step_smem(int n_dof) { return sizeof(float) * ((size_t)n_dof + 2); }

cudaError_t launch_coop(const void* fn, int grid, size_t smem, const StepArgs& a, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kStepThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[] = {const_cast<StepArgs*>(&a)};
  return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace

int step_grid(int kind, int n_dof) {
  int dev = 0, coop = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  int per_sm = 0;
  cudaError_t e;
  if (kind == 1) {
    raise_smem_limit_k(tl_step_kernel);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tl_step_kernel, kStepThreads, tl_step_smem(n_dof));
  } else {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_step_kernel, kStepThreads, 0);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  // two CTAs per SM at most: enough threads for the vector phases, and few
  // arrivals per barrier
  return sms * std::min(per_sm, 2);
}

void prepare_step_kernels(int kind, int n_dof) {
  if (kind == 1) raise_smem_limit_k(tl_step_kernel);
  (void)n_dof;
}


cudaError_t launch_tl_step(const StepArgs& a, cudaStream_t s) {
  const int g = step_grid(1, a.c.n_dof);
  if (g <= 0) return cudaErrorNotSupported;
  return launch_coop(reinterpret_cast<const void*>(tl_step_kernel), g, tl_step_smem(a.c.n_dof), a, s);
}

cudaError_t launch_jacobi_step(const StepArgs& a, cudaStream_t s) {
  const int g = step_grid(0, 0);
  if (g <= 0) return cudaErrorNotSupported;
  return launch_coop(reinterpret_cast<const void*>(jacobi_step_kernel), g, 0, a, s);
}

}  // namespace femb200
