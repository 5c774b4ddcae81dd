// Element-block tangent matvec (TET4, FP32): y = K_T x.
//
// eb_matvec_kernel: one CTA per element block (eb consecutive elements of
// the internal order, which is Morton-sorted, so a block is a compact piece
// of the mesh), one thread per element:
//   1. each thread loads its element's inputs (local vertex indices, slot
//      positions, tangent payload, material), then the block's local nodes
//      (the distinct vertices of its elements) are staged in shared memory:
//      coordinates with the fixed-DOF bits (X32) and the input vector, one
//      pass instead of four dependent gathers per element;
//   2. each thread evaluates its element (geometry, dF, dP, four slot
//      vectors) and stores the slot vectors at their node-major positions in
//      shared memory;
//   3. each local node's slot range is added in its fixed order.  A node all
//      of whose elements are in the block ("interior") is complete and goes
//      to y; a node shared with other blocks writes this block's partial row.
// eb_complete_kernel adds each shared node's partial rows in block order and
// writes y.  Inside CG the element pass also forms p.Ap element by element
// (sum over slots of p_a . f_a, equal to the node sum because p and y are
// both zero on fixed DOFs), one FP64 share per block; the completion kernel
// adds the shares in block order and sets alpha = rz / pAp.  No atomics touch
// the product, so results are bitwise reproducible; the grid-wide reduction
// runs over the completion kernel's few CTAs instead of one per element
// block.  Compared with the two-phase pass the per-element slot vectors stay
// in shared memory instead of going through L2 and back.  This replaces the
// reference's ti.atomic_add scatter (backend/fea/fem/material/neo_hookean.py:190)
// as the two other variants do.
#include <cuda_runtime.h>

#include <algorithm>

#include "fem_internal.h"
#include "fem_reduce.cuh"

namespace femb200 {

__device__ __forceinline__ void mask_xyz(float4& v, int fx) {
  if (fx & 1) v.x = 0.f;
  if (fx & 2) v.y = 0.f;
  if (fx & 4) v.z = 0.f;
}

// Inputs of one element read from global memory before the block's vertex
// staging, so their latency overlaps it.
struct EbElem {
  uint2 lc, sp;
  float pay[kPay];
  float scl;
  int mid;
};

template <int MODEL>
__device__ __forceinline__ void eb_load_elem(const MvArgs& a, int e, EbElem& q) {
  q.lc = __ldg(a.eb.lconn + e);
  q.sp = __ldg(a.eb.lspos + e);
  q.mid = (int)__ldg(a.m.mat_id + e);
  q.scl = __ldg(a.m.scale + e);
  // mixed tables: the payload words of the largest model (zeros beyond an element's own)
  const int npay = MODEL >= 0 ? model_pay_words(MODEL) : kPay;
#pragma unroll
  for (int k = 0; k < kPay; ++k) q.pay[k] = (k < npay) ? __ldg(a.payload + (size_t)k * a.m.n_elems + e) : 0.f;
}

// NT threads per CTA, one element each (NT elements per block).
template <int NT, int MODEL, bool CG>
__global__ void __launch_bounds__(NT, 1024 / NT) eb_matvec_kernel(const __grid_constant__ MvArgs a) {
  chain_enter();
  if (CG) {
    if (a.cg->done) return;
  }
  extern __shared__ __align__(16) unsigned char s_dyn[];
  const EbDev& t = a.eb;
  const MeshDev& m = a.m;
  float4* s_stage = reinterpret_cast<float4*>(s_dyn);  // [4 NT] slot vectors, node-major
  float4* s_x = s_stage + 4 * NT;                       // [lmax] coordinates, w = fixed bits
  float4* s_p = s_x + t.lmax;                           // [lmax] input vector
  uint16_t* s_row = reinterpret_cast<uint16_t*>(s_p + t.lmax);  // [lmax + 1]
  __shared__ double sred[NT / 32];
  __shared__ bool am_last;
  const int b = blockIdx.x;
  const int e = b * NT + (int)threadIdx.x;
  const bool has_e = e < m.n_elems;
  EbElem q;
  if (has_e) eb_load_elem<MODEL>(a, e, q);
  const int n0 = __ldg(t.node_ptr + b);
  const int L = __ldg(t.node_ptr + b + 1) - n0;
  const float4* __restrict__ xin = reinterpret_cast<const float4*>(a.x);
  // staging: coordinates by threads [0, L), the input vector by [L, 2L)
  // (about two local nodes per thread-pair-slot: every thread has one load)
  for (int i = threadIdx.x; i < 2 * L; i += NT) {
    const int ln = i < L ? i : i - L;
    const int n = __ldg(t.nodes + n0 + ln);
    if (i < L) {
      s_x[ln] = __ldg(m.X32 + n);
    } else {
      float4 P = __ldg(xin + n);
      if (a.mask_input) mask_xyz(P, (int)__ldg(m.fixed + n));
      s_p[ln] = P;
    }
  }
  for (int i = threadIdx.x; i <= L; i += NT) s_row[i] = __ldg(t.lrow + n0 + b + i);
  __syncthreads();

  double pap = 0.0;
  if (has_e) {
    const int li[4] = {(int)(q.lc.x & 0xffffu), (int)(q.lc.x >> 16), (int)(q.lc.y & 0xffffu), (int)(q.lc.y >> 16)};
    float xv[4][3], pv[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 X = s_x[li[k]];
      const float4 P = s_p[li[k]];
      xv[k][0] = X.x;
      xv[k][1] = X.y;
      xv[k][2] = X.z;
      pv[k][0] = P.x;
      pv[k][1] = P.y;
      pv[k][2] = P.z;
    }
    const DevMat<float>& mat = a.matF[q.mid];
    TetGeom<float> g;
    tet_geom(xv[0], xv[1], xv[2], xv[3], g);
    float D[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int d = 0; d < 3; ++d) D[k][d] = pv[k + 1][d] - pv[0][d];
    float dF[9];
    grad_from_diffs(D, g, dF);
    float dP[9];
    dP_any<MODEL>(mat, q.scl, q.pay, dF, dP);
    float f[4][3];
    slot_vectors(dP, g, g.s6, f);
    if (CG) {
      float pe = 0.f;
#pragma unroll
      for (int k = 0; k < 4; ++k) pe += pv[k][0] * f[k][0] + pv[k][1] * f[k][1] + pv[k][2] * f[k][2];
      pap = (double)pe;
    }
    s_stage[q.sp.x & 0xffffu] = make_float4(f[0][0], f[0][1], f[0][2], 0.f);
    s_stage[q.sp.x >> 16] = make_float4(f[1][0], f[1][1], f[1][2], 0.f);
    s_stage[q.sp.y & 0xffffu] = make_float4(f[2][0], f[2][1], f[2][2], 0.f);
    s_stage[q.sp.y >> 16] = make_float4(f[3][0], f[3][1], f[3][2], 0.f);
  }
  __syncthreads();

  // node sums: two adjacent lanes per local node, even and odd slots of its
  // range, combined even + odd (a fixed order)
  float4* __restrict__ yout = reinterpret_cast<float4*>(a.y);
#pragma unroll 1
  for (int base = 0; base < 2 * L; base += NT) {
    const int i = base + (int)threadIdx.x;
    const bool act = i < 2 * L;
    const int ln = i >> 1, half = i & 1;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    if (act) {
      const int j1 = s_row[ln + 1];
#pragma unroll 2
      for (int j = s_row[ln] + half; j < j1; j += 2) {
        const float4 v = s_stage[j];
        a0 += v.x;
        a1 += v.y;
        a2 += v.z;
      }
    }
    a0 += __shfl_xor_sync(0xffffffffu, a0, 1);
    a1 += __shfl_xor_sync(0xffffffffu, a1, 1);
    a2 += __shfl_xor_sync(0xffffffffu, a2, 1);
    if (act && half == 0) {
      const int4 info = __ldg(t.ninfo + n0 + ln);  // node, partial slot, first partial, count
      if (info.y < 0) {
        float4 yv = make_float4(a0, a1, a2, 0.f);
        mask_xyz(yv, (int)s_x[ln].w);
        yout[info.x] = yv;
      } else {
        __stcg(t.parts + info.y, make_float4(a0, a1, a2, 0.f));
      }
    }
  }

  if (CG) {
    chain_release();
    const double bsum = block_sum<NT>(pap, sred);
    if (threadIdx.x == 0) t.pap_part[b] = bsum;
  }
}

// Shared nodes: the partial rows of every block touching the node, added in
// block order.  CG: p.Ap from the element blocks' shares (each CTA adds a
// contiguous slice in order, the last CTA adds the slices in order) and alpha.
constexpr int kEbCompleteThreads = 256;

template <bool CG>
__global__ void __launch_bounds__(kEbCompleteThreads) eb_complete_kernel(const __grid_constant__ MvArgs a) {
  chain_enter();
  if (CG) {
    if (a.cg->done) return;
  }
  __shared__ double sred[kEbCompleteThreads / 32];
  __shared__ bool am_last;
  const EbDev& t = a.eb;
  float4* __restrict__ yout = reinterpret_cast<float4*>(a.y);
  for (int i = blockIdx.x * kEbCompleteThreads + threadIdx.x; i < t.n_shared; i += gridDim.x * kEbCompleteThreads) {
    const int4 sn = __ldg(t.snode + i);
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll 1
    for (int k = 0; k < sn.z; ++k) {
      const float4 v = __ldcg(t.parts + sn.y + k);
      s0 += v.x;
      s1 += v.y;
      s2 += v.z;
    }
    float4 yv = make_float4(s0, s1, s2, 0.f);
    mask_xyz(yv, (int)a.m.fixed[sn.x]);
    yout[sn.x] = yv;
  }
  if (CG) {
    chain_release();
    const int per = (t.n_blk + gridDim.x - 1) / gridDim.x;
    const int k0 = blockIdx.x * per, k1 = min(t.n_blk, k0 + per);
    double acc = 0.0;
    // per <= kEbCompleteThreads: thread k adds share k0 + k, block_sum adds the threads in order
    if (k0 + (int)threadIdx.x < k1) acc = __ldcg(t.pap_part + k0 + threadIdx.x);
    double bsum = block_sum<kEbCompleteThreads>(acc, sred);
    if (publish_partial(a.red, a.red_site, 1, &bsum, &am_last)) {
      double tot = final_sum<kEbCompleteThreads>(a.red, a.red_site, 0, sred);
      if (threadIdx.x == 0) {
        CGState* st = a.cg;
        st->pAp = tot;
        if (!(tot > 0.0) || !isfinite(tot)) {
          st->done = 3;
          st->status = 3;
          st->alpha = 0.0;
        } else {
          st->alpha = st->rz / tot;
        }
        a.red.counters[a.red_site] = 0u;
      }
    }
  }
}

// CTAs of the completion kernel: enough that each adds at most
// kEbCompleteThreads of the element blocks' p.Ap shares, at least 2 per SM
static int eb_complete_grid(const EbDev& t) {
  static int n_sm = 0;
  if (n_sm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (n_sm <= 0) n_sm = 148;
  }
  const int need = (t.n_blk + kEbCompleteThreads - 1) / kEbCompleteThreads;
  const int by_nodes = (t.n_shared + kEbCompleteThreads - 1) / kEbCompleteThreads;
  return std::max(1, std::max(need, std::min(by_nodes, 2 * n_sm)));
}

template <int NT, int MODEL, bool CG>
static void eb_go(const MvArgs& a, cudaStream_t s) {
  const size_t smem = eb_smem_bytes(NT, a.eb.lmax);
  raise_smem_limit_k(eb_matvec_kernel<NT, MODEL, CG>);
  launch_chain(eb_matvec_kernel<NT, MODEL, CG>, a.eb.n_blk, NT, smem, s, a);
}

template <int NT, bool CG>
static void eb_model(const MvArgs& a, int model, cudaStream_t s) {
  switch (model) {
    case M_LE: eb_go<NT, M_LE, CG>(a, s); break;
    case M_NH: eb_go<NT, M_NH, CG>(a, s); break;
    case M_MR: eb_go<NT, M_MR, CG>(a, s); break;
    case M_J2: eb_go<NT, M_J2, CG>(a, s); break;
    case M_TI: eb_go<NT, M_TI, CG>(a, s); break;
    case M_FMR: eb_go<NT, M_FMR, CG>(a, s); break;
    default: eb_go<NT, -1, CG>(a, s); break;
  }
}

template <bool CG>
static void eb_size(const MvArgs& a, int model, cudaStream_t s) {
  switch (a.eb.eb) {
    case 256: eb_model<256, CG>(a, model, s); break;
    case 512: eb_model<512, CG>(a, model, s); break;
    case 768: eb_model<768, CG>(a, model, s); break;
    default: eb_model<1024, CG>(a, model, s); break;
  }
}

void launch_matvec_eb(const MvArgs& a, int model, cudaStream_t s) {
  const int g = eb_complete_grid(a.eb);
  if (a.cg) {
    eb_size<true>(a, model, s);
    launch_chain(eb_complete_kernel<true>, g, kEbCompleteThreads, 0, s, a);
  } else {
    eb_size<false>(a, model, s);
    launch_chain(eb_complete_kernel<false>, g, kEbCompleteThreads, 0, s, a);
  }
}

template <int NT>
static void prepare_eb_nt(int model) {
  auto set = [](auto k) { raise_smem_limit_k(k); };
  switch (model) {
    case M_LE: set(eb_matvec_kernel<NT, M_LE, true>); break;
    case M_NH: set(eb_matvec_kernel<NT, M_NH, true>); break;
    case M_MR: set(eb_matvec_kernel<NT, M_MR, true>); break;
    case M_J2: set(eb_matvec_kernel<NT, M_J2, true>); break;
    case M_TI: set(eb_matvec_kernel<NT, M_TI, true>); break;
    case M_FMR: set(eb_matvec_kernel<NT, M_FMR, true>); break;
    default: set(eb_matvec_kernel<NT, -1, true>); break;
  }
}

void prepare_eb_kernels(int model) {
  prepare_eb_nt<256>(model);
  prepare_eb_nt<512>(model);
  prepare_eb_nt<768>(model);
  prepare_eb_nt<1024>(model);
}

}  // namespace femb200
