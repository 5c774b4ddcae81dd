// sm_100a kernels of the TET4 static-solve path.
//
// Element kernels run one CTA per node block (nb consecutive internal nodes,
// nb = blockDim.x).  A CTA walks its element list in chunks of nb elements:
// every thread evaluates one element (F -> stress -> four slot vectors) into
// shared memory, then every thread sums, for the node it owns, the slot
// vectors of that chunk in the fixed order of the node's slot list.  No
// atomics touch the outputs, so results are bitwise reproducible; elements
// shared by two blocks are evaluated by both (about 1.4x redundant work at
// nb = 256 on Morton-ordered meshes) instead of staging per-element forces in
// HBM.  This replaces the reference's ti.atomic_add scatter
// (e.g. backend/fea/fem/material/neo_hookean.py:190).
#include <cuda_runtime.h>

#include <algorithm>

#include "fem_internal.h"
#include "fem_reduce.cuh"

namespace femb200 {

// Loads this block's node slot lists (one contiguous range of node_slots)
// into shared memory and returns the calling thread's node range within it.
// The caller's first __syncthreads makes the copy visible.
template <int NB>
__device__ __forceinline__ void load_block_slots(const MeshDev& m, int b, uint32_t* s_slots,
                                                 int& cur, int& end) {
  const int n0 = b * NB;
  const int n1 = min(n0 + NB, m.n_nodes);
  const int s0 = __ldg(m.node_row + n0);
  const int s1 = __ldg(m.node_row + n1);
  for (int i = threadIdx.x; i < s1 - s0; i += NB) s_slots[i] = __ldg(m.node_slots + s0 + i);
  const int node = n0 + (int)threadIdx.x;
  cur = end = 0;
  if (node < m.n_nodes) {
    cur = __ldg(m.node_row + node) - s0;
    end = __ldg(m.node_row + node + 1) - s0;
  }
}

// Adds, in slot-list order, the slot vectors of the current chunk that belong
// to this thread's node.  Entries are sorted by local element index, so every
// chunk consumes a prefix of what is left.
template <int NB, typename T, typename TA>
__device__ __forceinline__ void gather_chunk(const uint32_t* s_slots, const T (*sf)[NB], int base,
                                             int& cur, int end, TA& a0, TA& a1, TA& a2) {
  const int lim = base + NB;
  while (cur < end) {
    const uint32_t ent = s_slots[cur];
    const int li = (int)(ent >> 2);
    if (li >= lim) break;
    const int t = li - base;
    const int s = (int)(ent & 3u);
    a0 += sf[3 * s + 0][t];
    a1 += sf[3 * s + 1][t];
    a2 += sf[3 * s + 2][t];
    ++cur;
  }
}

// gather_chunk for W values per slot: sf[W * slot + k][thread]
template <int NB, int W>
__device__ __forceinline__ void gather_chunk_w(const uint32_t* s_slots, const float (*sf)[NB], int base, int& cur,
                                               int end, float (&acc)[W]) {
  const int lim = base + NB;
  while (cur < end) {
    const uint32_t ent = s_slots[cur];
    const int li = (int)(ent >> 2);
    if (li >= lim) break;
    const int t = li - base;
    const int s = (int)(ent & 3u);
#pragma unroll
    for (int k = 0; k < W; ++k) acc[k] += sf[W * s + k][t];
    ++cur;
  }
}

// ───────────────────────── residual (FP64) ─────────────────────────

// Element e's four slot forces (FP64, the negative internal force of its
// vertices) from u; with write_state also its tangent payload and J2 trial
// history.
template <int MODEL>
__device__ __forceinline__ void res_element(const ResArgs& a, int e, bool write_state, double f[4][3]) {
  const MeshDev& m = a.m;
  const int4 cn = __ldg(m.conn + e);
  const int nid[4] = {cn.x, cn.y, cn.z, cn.w};
  double xv[4][3], uv[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      xv[k][d] = __ldg(m.X64 + 3 * nid[k] + d);
      uv[k][d] = __ldg(a.u + 3 * nid[k] + d);
    }
  TetGeom<double> g;
  tet_geom(xv[0], xv[1], xv[2], xv[3], g);
  double D[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int d = 0; d < 3; ++d) D[k][d] = uv[k + 1][d] - uv[0][d];
  double Hg[9];
  grad_from_diffs(D, g, Hg);
  const DevMat<double>& mat = a.matD[__ldg(m.mat_id + e)];
  const double scale = (double)__ldg(m.scale + e);
  const int model = MODEL >= 0 ? MODEL : mat.model;
  double S[9];
  float pay[kPay];
  if (model == M_NH) {
    nh_stress(mat, scale, Hg, S, pay);
  } else if (model == M_MR || model == M_FMR) {
    mr_stress(mat, scale, Hg, S, pay);
  } else if (model == M_J2) {
    double ep[6], epn[6], epe_n;
#pragma unroll
    for (int k = 0; k < 6; ++k) ep[k] = a.ep_c[(size_t)k * m.n_elems + e];
    const double epe = a.epe_c[e];
    j2_stress(mat, scale, Hg, ep, epe, S, epn, epe_n, pay);
    if (write_state) {
#pragma unroll
      for (int k = 0; k < 6; ++k) a.ep_t[(size_t)k * m.n_elems + e] = epn[k];
      a.epe_t[e] = epe_n;
    }
  } else if (model == M_TI) {
    ti_stress(mat, scale, Hg, S);
  } else {
    le_stress(mat, scale, Hg, S);
  }
  if (write_state) {
    const int npay = model_pay_words(model);
#pragma unroll
    for (int k = 0; k < kPay; ++k)
      if (k < npay) a.payload[(size_t)k * m.n_elems + e] = pay[k];
  }
  slot_vectors(S, g, -g.s6, f);
}

template <int NB, int MODEL>
__global__ void __launch_bounds__(NB) residual_kernel(const __grid_constant__ ResArgs a) {
  // dynamic: 12 x NB doubles of slot vectors, then the block's slot lists
  extern __shared__ __align__(16) unsigned char s_dyn[];
  double(*sf)[NB] = reinterpret_cast<double(*)[NB]>(s_dyn);
  uint32_t* s_slots = reinterpret_cast<uint32_t*>(s_dyn + sizeof(double) * 12 * NB);
  __shared__ double sred[NB / 32];
  __shared__ bool am_last;
  const MeshDev& m = a.m;
  const int b = blockIdx.x;
  const int tid = threadIdx.x;
  const int node = b * NB + tid;
  const bool has_node = node < m.n_nodes;
  int cur, end;
  load_block_slots<NB>(m, b, s_slots, cur, end);
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
  const int e0 = m.blk_ptr[b], e1 = m.blk_ptr[b + 1];
  const int home_end = e0 + m.blk_home[b];
  for (int c0 = e0; c0 < e1; c0 += NB) {
    const int idx = c0 + tid;
    if (idx < e1) {
      double f[4][3];
      res_element<MODEL>(a, __ldg(m.blk_elems + idx), idx < home_end, f);
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int d = 0; d < 3; ++d) sf[3 * s + d][tid] = f[s][d];
    }
    __syncthreads();
    gather_chunk<NB>(s_slots, sf, c0 - e0, cur, end, acc0, acc1, acc2);
    __syncthreads();
  }
  double r2 = 0.0;
  if (has_node) {
    const uint8_t fx = m.fixed[node];
    const double accs[3] = {acc0, acc1, acc2};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double fn = accs[d];
      if (a.fneg) a.fneg[3 * node + d] = fn;
      const double r = ((fx >> d) & 1) ? 0.0 : a.f_ext[3 * node + d] + fn;
      a.R[3 * node + d] = r;
      r2 += r * r;
    }
  }
  double bsum = block_sum<NB>(r2, sred);
  if (publish_partial(a.red, a.red_site, 1, &bsum, &am_last)) {
    double tot = final_sum<NB>(a.red, a.red_site, 0, sred);
    if (tid == 0) {
      *a.rnorm2 = tot;
      a.red.counters[a.red_site] = 0u;
    }
  }
}

// Two-phase FP64 residual.  res_elem_kernel: one thread per element, each
// element evaluated once (the fused node-block kernel above evaluates an
// element shared by several node blocks in each of them), its four slot
// forces stored at their positions in node-slot order (stage_d, three doubles
// per slot).  res_gather_kernel: kGatherLanes lanes per node add the node's
// contiguous slot range (lane k: slots k, k + kGatherLanes, ...; then xor
// steps in a fixed order), R = f_ext + f on free DOFs and the fixed-order
// FP64 sum of ||R||^2.  Bitwise reproducible; the node sums are associated
// differently from the fused kernel's (agreement to rounding).
template <int MODEL>
__global__ void __launch_bounds__(128) res_elem_kernel(const __grid_constant__ ResArgs a) {
  // persistent: one wave of CTAs walks the elements in grid-stride order
  for (int e = (int)blockIdx.x * 128 + (int)threadIdx.x; e < a.m.n_elems; e += (int)gridDim.x * 128) {
    double f[4][3];
    res_element<MODEL>(a, e, true, f);
    const int4 sp = __ldg(a.m.spos + e);
    const int pos[4] = {sp.x, sp.y, sp.z, sp.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int d = 0; d < 3; ++d) __stcg(a.stage_d + 3 * (size_t)pos[k] + d, f[k][d]);
  }
}

// ───────────────────────── tangent matvec (FP32) ─────────────────────────
// x and y hold one float4 per node (xyz, 0); X32.w carries the node's
// fixed-DOF bits, so one 16-byte load per vertex brings geometry and mask.

template <int NB, int MODEL, bool CG>
__global__ void __launch_bounds__(NB) matvec_kernel(const __grid_constant__ MvArgs a) {
  chain_enter();
  if (CG) {
    if (a.cg->done) return;
  }
  extern __shared__ __align__(16) unsigned char s_dyn[];
  uint32_t* s_slots = reinterpret_cast<uint32_t*>(s_dyn);
  __shared__ float sf[12][NB];
  __shared__ double sred[NB / 32];
  __shared__ bool am_last;
  const MeshDev& m = a.m;
  const int b = blockIdx.x;
  const int tid = threadIdx.x;
  const int node = b * NB + tid;
  const bool has_node = node < m.n_nodes;
  int cur, end;
  load_block_slots<NB>(m, b, s_slots, cur, end);
  float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f;
  const int e0 = m.blk_ptr[b], e1 = m.blk_ptr[b + 1];
  const float4* __restrict__ xin = reinterpret_cast<const float4*>(a.x);
  for (int c0 = e0; c0 < e1; c0 += NB) {
    const int idx = c0 + tid;
    if (idx < e1) {
      const int e = __ldg(m.blk_elems + idx);
      const int4 cn = __ldg(m.conn + e);
      const int nid[4] = {cn.x, cn.y, cn.z, cn.w};
      float xv[4][3], pv[4][3];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float4 X = __ldg(m.X32 + nid[k]);
        const float4 P = __ldg(xin + nid[k]);
        xv[k][0] = X.x;
        xv[k][1] = X.y;
        xv[k][2] = X.z;
        const int fx = a.mask_input ? (int)X.w : 0;
        pv[k][0] = (fx & 1) ? 0.f : P.x;
        pv[k][1] = (fx & 2) ? 0.f : P.y;
        pv[k][2] = (fx & 4) ? 0.f : P.z;
      }
      TetGeom<float> g;
      tet_geom(xv[0], xv[1], xv[2], xv[3], g);
      float D[3][3];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int d = 0; d < 3; ++d) D[k][d] = pv[k + 1][d] - pv[0][d];
      float dF[9];
      grad_from_diffs(D, g, dF);
      const DevMat<float>& mat = a.matF[__ldg(m.mat_id + e)];
      const float scale = __ldg(m.scale + e);
      float pay[kPay];
      {
        const int npay = model_pay_words(MODEL >= 0 ? MODEL : mat.model);
#pragma unroll
        for (int k = 0; k < kPay; ++k)
          pay[k] = (k < npay) ? __ldg(a.payload + (size_t)k * m.n_elems + e) : 0.f;
      }
      float dP[9];
      dP_any<MODEL>(mat, scale, pay, dF, dP);
      float f[4][3];
      slot_vectors(dP, g, g.s6, f);
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int d = 0; d < 3; ++d) sf[3 * s + d][tid] = f[s][d];
    }
    __syncthreads();
    gather_chunk<NB>(s_slots, sf, c0 - e0, cur, end, acc0, acc1, acc2);
    __syncthreads();
  }
  double pap = 0.0;
  if (has_node) {
    const uint8_t fx = m.fixed[node];
    const float4 yv = make_float4((fx & 1) ? 0.f : acc0, (fx & 2) ? 0.f : acc1,
                                  (fx & 4) ? 0.f : acc2, 0.f);
    reinterpret_cast<float4*>(a.y)[node] = yv;
    if (CG) {
      const float4 pv = xin[node];
      pap = (double)yv.x * pv.x + (double)yv.y * pv.y + (double)yv.z * pv.z;
    }
  }
  if (CG) {
    double bsum = block_sum<NB>(pap, sred);
    if (publish_partial(a.red, a.red_site, 1, &bsum, &am_last)) {
      double tot = final_sum<NB>(a.red, a.red_site, 0, sred);
      if (tid == 0) {
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

// ───────────────────────── two-phase tangent matvec (FP32) ─────────────────────────
// Phase 1: one thread per element, no barriers and no redundant evaluation;
// each slot vector is stored at its position in the node-major slot list.
// Phase 2: one thread per node sums its contiguous slot range in list order,
// so the result is the same fixed-order (bitwise reproducible) sum.

// Streaming (coalesced SoA) inputs of one element: connectivity, slot
// positions, material, modulus scale and tangent payload.
struct MvIn {
  int4 cn, sp;
  float pay[kPay];
  float scl;
  int mid;
};

// The per-element words after the connectivity and slot positions.
template <int MODEL>
__device__ __forceinline__ void mv_load_rest(const MvArgs& a, int e, MvIn& q) {
  const MeshDev& m = a.m;
  q.mid = (int)__ldg(m.mat_id + e);
  q.scl = __ldg(m.scale + e);
  // mixed tables: the payload words of the largest model (zeros beyond an element's own)
  const int npay = MODEL >= 0 ? model_pay_words(MODEL) : kPay;
#pragma unroll
  for (int k = 0; k < kPay; ++k) q.pay[k] = (k < npay) ? __ldg(a.payload + (size_t)k * m.n_elems + e) : 0.f;
}

template <int MODEL>
__device__ __forceinline__ void mv_load(const MvArgs& a, int e, MvIn& q) {
  q.cn = __ldg(a.m.conn + e);
  q.sp = __ldg(a.m.spos + e);
  mv_load_rest<MODEL>(a, e, q);
}

// The four slot vectors f (tangent action on x) of one element from its
// vertices' coordinates (w: fixed-DOF bits) and x values.
template <int MODEL, bool MASK>
__device__ __forceinline__ void elem_mv_forces_v(const MvArgs& a, const float4 (&X)[4], const float4 (&P)[4],
                                                 int mid, float scl, const float (&pay)[kPay], float f[4][3]) {
  float xv[4][3], pv[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    xv[k][0] = X[k].x;
    xv[k][1] = X[k].y;
    xv[k][2] = X[k].z;
    // CG directions are zero on fixed DOFs already; only a standalone
    // matvec masks its input
    const int fx = MASK ? (int)X[k].w : 0;
    pv[k][0] = (fx & 1) ? 0.f : P[k].x;
    pv[k][1] = (fx & 2) ? 0.f : P[k].y;
    pv[k][2] = (fx & 4) ? 0.f : P[k].z;
  }
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
  dP_any<MODEL>(a.matF[mid], scl, pay, dF, dP);
  slot_vectors(dP, g, g.s6, f);
}

// The four slot vectors f (tangent action on x) of the element whose
// streaming inputs are q: its vertices' coordinates and x are gathered here.
template <int MODEL, bool MASK>
__device__ __forceinline__ void elem_mv_forces_q(const MvArgs& a, const MvIn& q, float f[4][3]) {
  const int nid[4] = {q.cn.x, q.cn.y, q.cn.z, q.cn.w};
  const float4* __restrict__ xin = reinterpret_cast<const float4*>(a.x);
  float4 X[4], P[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    X[k] = __ldg(a.m.X32 + nid[k]);
    P[k] = __ldg(xin + nid[k]);
  }
  elem_mv_forces_v<MODEL, MASK>(a, X, P, q.mid, q.scl, q.pay, f);
}

// The four slot vectors f (tangent action on x) of element e.
template <int MODEL, bool MASK>
__device__ __forceinline__ void elem_mv_forces(const MvArgs& a, int e, float f[4][3]) {
  MvIn q;
  mv_load<MODEL>(a, e, q);
  elem_mv_forces_q<MODEL, MASK>(a, q, f);
}

template <int MODEL, bool MASK>
__device__ __forceinline__ void elem_mv_one(const MvArgs& a, int e) {
  const int4 sp = __ldg(a.m.spos + e);
  float f[4][3];
  elem_mv_forces<MODEL, MASK>(a, e, f);
  __stcg(a.stage + sp.x, make_float4(f[0][0], f[0][1], f[0][2], 0.f));
  __stcg(a.stage + sp.y, make_float4(f[1][0], f[1][1], f[1][2], 0.f));
  __stcg(a.stage + sp.z, make_float4(f[2][0], f[2][1], f[2][2], 0.f));
  __stcg(a.stage + sp.w, make_float4(f[3][0], f[3][1], f[3][2], 0.f));
}

// 5 CTAs per SM: 48 registers (no spills) instead of 52 lift occupancy from
// 50 % to 62.5 % for this latency-bound gather-compute-scatter kernel.
template <int MODEL, bool CG>
__global__ void __launch_bounds__(256, 5) elem_mv_kernel(const __grid_constant__ MvArgs a) {
  chain_enter();
  if (CG) {
    if (a.cg->done) return;
  }
  const int e = blockIdx.x * 256 + threadIdx.x;
  if (e >= a.m.n_elems) return;
  if (!CG && a.mask_input)
    elem_mv_one<MODEL, true>(a, e);
  else
    elem_mv_one<MODEL, false>(a, e);
}

// Persistent element pass: one wave of CTAs (resident CTAs per SM x SMs)
// walks the elements in grid-stride order.  Each thread loads the
// connectivity and slot positions of its next element before it evaluates
// the current one, so the current element's vertex gathers and its payload
// loads are in flight together (one memory round trip per element instead
// of two dependent ones).
template <int MODEL, bool CG>
__global__ void __launch_bounds__(256, 4) elem_mv_persist_kernel(const __grid_constant__ MvArgs a) {
  chain_enter();
  if (CG) {
    if (a.cg->done) return;
  }
  const int n = a.m.n_elems;
  const int stride = (int)gridDim.x * 256;
  int e = (int)blockIdx.x * 256 + (int)threadIdx.x;
  if (e >= n) return;
  const bool mask = !CG && a.mask_input;
  int4 cn = __ldg(a.m.conn + e), sp = __ldg(a.m.spos + e);
  for (;;) {
    const int en = e + stride;
    int4 cn_n = cn, sp_n = sp;
    if (en < n) {
      cn_n = __ldg(a.m.conn + en);
      sp_n = __ldg(a.m.spos + en);
    }
    MvIn q;
    q.cn = cn;
    q.sp = sp;
    mv_load_rest<MODEL>(a, e, q);
    float f[4][3];
    if (mask)
      elem_mv_forces_q<MODEL, true>(a, q, f);
    else
      elem_mv_forces_q<MODEL, false>(a, q, f);
    __stcg(a.stage + sp.x, make_float4(f[0][0], f[0][1], f[0][2], 0.f));
    __stcg(a.stage + sp.y, make_float4(f[1][0], f[1][1], f[1][2], 0.f));
    __stcg(a.stage + sp.z, make_float4(f[2][0], f[2][1], f[2][2], 0.f));
    __stcg(a.stage + sp.w, make_float4(f[3][0], f[3][1], f[3][2], 0.f));
    if (en >= n) break;
    e = en;
    cn = cn_n;
    sp = sp_n;
  }
}

// Warp-aggregated element pass.  The elements are taken 32 at a time (one
// "element warp" w: elements 32 w .. 32 w + 31) and each has its list of
// distinct vertices (rows, node-major).  A hardware warp walks the element
// warps in grid-stride order (persistent, one wave of CTAs); for each it
//   1. loads every row's coordinates (w: fixed-DOF bits) and x value once
//      into shared memory (a vertex shared by several of the 32 elements is
//      read once instead of once per element);
//   2. lane l evaluates element 32 w + l from those rows and puts its slot
//      vectors at their places in the warp's node-major slot order;
//   3. each row is the sum of its slot range in that order, written to its
//      place among the vertex's partial rows (the node gather adds those).
constexpr int kWaggWarps = 8;

template <int MODEL, bool CG>
__global__ void __launch_bounds__(32 * kWaggWarps, 4) elem_wagg_kernel(const __grid_constant__ MvArgs a) {
  chain_enter();
  if (CG) {
    if (a.cg->done) return;
  }
  __shared__ float4 s_slot[kWaggWarps][128];
  __shared__ float4 s_xv[kWaggWarps][128];
  __shared__ float4 s_pv[kWaggWarps][128];
  const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
  const int n = a.m.n_elems;
  const bool mask = !CG && a.mask_input;
  const float4* __restrict__ xin = reinterpret_cast<const float4*>(a.x);
  float4* sw = s_slot[warp];
  float4* sx = s_xv[warp];
  float4* sp4 = s_pv[warp];
  for (int w = (int)blockIdx.x * kWaggWarps + warp; w * 32 < n; w += (int)gridDim.x * kWaggWarps) {
    const int e = w * 32 + lane;
    const bool valid = e < n;
    const int q0 = __ldg(a.wa.wptr + w), q1 = __ldg(a.wa.wptr + w + 1);
    // the element's own streaming words first, so they are in flight with the row loads
    MvIn q;
    uint32_t lr = 0u, sp = 0u;
    if (valid) {
      lr = __ldg(a.wa.lrow + e);
      sp = __ldg(a.wa.lspos + e);
      mv_load_rest<MODEL>(a, e, q);
    }
    for (int i = q0 + lane; i < q1; i += 32) {
      const int node = __ldg(a.wa.wnode + i);
      sx[i - q0] = __ldg(a.m.X32 + node);
      sp4[i - q0] = __ldg(xin + node);
    }
    __syncwarp();
    if (valid) {
      float4 X[4], P[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int r = (int)((lr >> (8 * k)) & 0xffu);
        X[k] = sx[r];
        P[k] = sp4[r];
      }
      float f[4][3];
      if (mask)
        elem_mv_forces_v<MODEL, true>(a, X, P, q.mid, q.scl, q.pay, f);
      else
        elem_mv_forces_v<MODEL, false>(a, X, P, q.mid, q.scl, q.pay, f);
      sw[sp & 0xffu] = make_float4(f[0][0], f[0][1], f[0][2], 0.f);
      sw[(sp >> 8) & 0xffu] = make_float4(f[1][0], f[1][1], f[1][2], 0.f);
      sw[(sp >> 16) & 0xffu] = make_float4(f[2][0], f[2][1], f[2][2], 0.f);
      sw[sp >> 24] = make_float4(f[3][0], f[3][1], f[3][2], 0.f);
    }
    __syncwarp();
#pragma unroll 1
    for (int i = q0 + lane; i < q1; i += 32) {
      const int2 en = __ldg(a.wa.went + i);  // partial position, slot range
      const int j1 = en.y >> 16;
      float a0 = 0.f, a1 = 0.f, a2 = 0.f;
      for (int j = en.y & 0xffff; j < j1; ++j) {
        const float4 v = sw[j];
        a0 += v.x;
        a1 += v.y;
        a2 += v.z;
      }
      __stcg(a.wa.parts + en.x, make_float4(a0, a1, a2, 0.f));
    }
    __syncwarp();  // the shared rows and slots are refilled by the next element warp
  }
}

// kGatherLanes lanes per node: lane k of a node's group adds slots k,
// k + kGatherLanes, ... of its slot list (a node's slots are contiguous, so a
// warp reads one contiguous stretch), then xor steps combine the group in a
// fixed order.  Several lanes per node keep several times as many loads in
// flight as one thread per node.
constexpr int kGatherLanes = 4;
constexpr int kGatherNodes = 256 / kGatherLanes;  // nodes per CTA

// Node n's product row from its contiguous slot range (lanes sub of its
// kGatherLanes-lane group), stored to y; inside CG also the direction by
// recurrence and the node's p.Ap term (returned by the group's lane 0).
// Every lane of the warp calls it (the group sum uses shuffles).
template <bool CG>
__device__ __forceinline__ double gather_node(const MvArgs& a, int n, int sub) {
  const MeshDev& m = a.m;
  double pap = 0.0;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  if (n < m.n_nodes) {
    const int j0 = __ldg(m.node_row + n), j1 = __ldg(m.node_row + n + 1);
    constexpr int kBatch = 8;
    for (int j = j0 + sub; j < j1; j += kBatch * kGatherLanes) {
      float4 v[kBatch];
#pragma unroll
      for (int k = 0; k < kBatch; ++k)
        v[k] = (j + k * kGatherLanes < j1) ? __ldcg(a.stage + j + k * kGatherLanes) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int k = 0; k < kBatch; ++k) {
        a0 += v[k].x;
        a1 += v[k].y;
        a2 += v[k].z;
      }
    }
  }
#pragma unroll
  for (int o = 1; o < kGatherLanes; o <<= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  }
  if (n < m.n_nodes && sub == 0) {
    const uint8_t fx = m.fixed[n];
    float4 yv = make_float4((fx & 1) ? 0.f : a0, (fx & 2) ? 0.f : a1, (fx & 4) ? 0.f : a2, 0.f);
    if (CG && a.p_rec) {
      // direction by recurrence: x = z, q = K z + beta q_old, p = z + beta p_old
      // (beta = 0 after the start: plain copies, whatever the old vectors hold)
      const double beta_d = a.cg->beta;
      const float beta = (float)beta_d;
      float4 pv = reinterpret_cast<const float4*>(a.x)[n];
      if (beta_d != 0.0) {
        const float4 qo = reinterpret_cast<const float4*>(a.y)[n];
        const float4 po = reinterpret_cast<const float4*>(a.p_rec)[n];
        yv.x += beta * qo.x; yv.y += beta * qo.y; yv.z += beta * qo.z;
        pv.x += beta * po.x; pv.y += beta * po.y; pv.z += beta * po.z;
      }
      reinterpret_cast<float4*>(a.p_rec)[n] = pv;
      reinterpret_cast<float4*>(a.y)[n] = yv;
      pap = (double)yv.x * pv.x + (double)yv.y * pv.y + (double)yv.z * pv.z;
    } else {
      reinterpret_cast<float4*>(a.y)[n] = yv;
      if (CG) {
        const float4 pv = reinterpret_cast<const float4*>(a.x)[n];
        pap = (double)yv.x * pv.x + (double)yv.y * pv.y + (double)yv.z * pv.z;
      }
    }
  }
  return pap;
}

// The last block's p.Ap: alpha = rz / pAp, or a breakdown flag.
__device__ __forceinline__ void gather_finish(const MvArgs& a, double pap, double* sred, bool* am_last) {
  double bsum = block_sum<256>(pap, sred);
  if (publish_partial(a.red, a.red_site, 1, &bsum, am_last)) {
    double tot = final_sum<256>(a.red, a.red_site, 0, sred);
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

template <bool CG>
__global__ void __launch_bounds__(256) node_gather_kernel(const __grid_constant__ MvArgs a) {
  chain_enter();
  if (CG) {
    if (a.cg->done) return;
  }
  __shared__ double sred[8];
  __shared__ bool am_last;
  const int n = blockIdx.x * kGatherNodes + threadIdx.x / kGatherLanes;
  const double pap = gather_node<CG>(a, n, threadIdx.x % kGatherLanes);
  if (CG) {
    chain_release();
    gather_finish(a, pap, sred, &am_last);
  }
}

// Persistent node gather: one wave of CTAs walks the node groups in
// grid-stride order, so the grid reduction adds one partial per resident
// CTA instead of one per 64-node group.
template <bool CG>
__global__ void __launch_bounds__(256) node_gather_persist_kernel(const __grid_constant__ MvArgs a) {
  chain_enter();
  if (CG) {
    if (a.cg->done) return;
  }
  __shared__ double sred[8];
  __shared__ bool am_last;
  double pap = 0.0;
  const int sub = threadIdx.x % kGatherLanes;
  for (int g = blockIdx.x; g * kGatherNodes < a.m.n_nodes; g += gridDim.x)
    pap += gather_node<CG>(a, g * kGatherNodes + threadIdx.x / kGatherLanes, sub);
  if (CG) {
    chain_release();
    gather_finish(a, pap, sred, &am_last);
  }
}

// One node's residual row (LANES lanes of a group add its slot range; the
// group's lane 0 stores R and fneg) and its ||R||^2 term (lane 0).
template <int LANES>
__device__ __forceinline__ double res_gather_node(const ResArgs& a, int n, int sub) {
  const MeshDev& m = a.m;
  double acc[3] = {0.0, 0.0, 0.0};
  if (n < m.n_nodes) {
    const int j0 = __ldg(m.node_row + n), j1 = __ldg(m.node_row + n + 1);
    for (int j = j0 + sub; j < j1; j += LANES)
#pragma unroll
      for (int d = 0; d < 3; ++d) acc[d] += __ldcg(a.stage_d + 3 * (size_t)j + d);
  }
#pragma unroll
  for (int o = 1; o < LANES; o <<= 1)
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d] += __shfl_xor_sync(0xffffffffu, acc[d], o);
  double r2 = 0.0;
  if (n < m.n_nodes && sub == 0) {
    const uint8_t fx = m.fixed[n];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (a.fneg) a.fneg[3 * n + d] = acc[d];
      const double r = ((fx >> d) & 1) ? 0.0 : a.f_ext[3 * n + d] + acc[d];
      a.R[3 * n + d] = r;
      r2 += r * r;
    }
  }
  return r2;
}

// Persistent over node groups (grid-stride): one ||R||^2 partial per
// resident CTA, added in index order by the last block.
template <int LANES>
__global__ void __launch_bounds__(256) res_gather_kernel(const __grid_constant__ ResArgs a) {
  __shared__ double sred[8];
  __shared__ bool am_last;
  constexpr int kNodes = 256 / LANES;
  const int sub = (int)threadIdx.x % LANES;
  double r2 = 0.0;
  for (int g = blockIdx.x; g * kNodes < a.m.n_nodes; g += gridDim.x)
    r2 += res_gather_node<LANES>(a, g * kNodes + (int)threadIdx.x / LANES, sub);
  double bsum = block_sum<256>(r2, sred);
  if (publish_partial(a.red, a.red_site, 1, &bsum, &am_last)) {
    double tot = final_sum<256>(a.red, a.red_site, 0, sred);
    if (threadIdx.x == 0) {
      *a.rnorm2 = tot;
      a.red.counters[a.red_site] = 0u;
    }
  }
}

// ───────────────────────── Jacobi diagonal (FP32) ─────────────────────────
//
// BLOCK = false: dinv = 1 / diag(K_T) on free DOFs.  BLOCK = true: the
// node's 3 x 3 diagonal block of K_T (6 entries per element slot, gathered
// in the same fixed order), restricted to the free DOFs and inverted in
// FP64: dinv = the inverse's diagonal, boff = its off-diagonals (01, 02, 12);
// fixed rows and columns are zero.  A block that is not positive definite
// falls back to the scalar inverse of its diagonal.

template <int NB, int MODEL, bool BLOCK>
__global__ void __launch_bounds__(NB) diag_kernel(const __grid_constant__ DiagArgs a) {
  constexpr int W = BLOCK ? 6 : 3;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  uint32_t* s_slots = reinterpret_cast<uint32_t*>(s_dyn);
  __shared__ float sf[4 * W][NB];
  const MeshDev& m = a.m;
  const int b = blockIdx.x;
  const int tid = threadIdx.x;
  const int node = b * NB + tid;
  const bool has_node = node < m.n_nodes;
  int cur, end;
  load_block_slots<NB>(m, b, s_slots, cur, end);
  float acc[W];
#pragma unroll
  for (int k = 0; k < W; ++k) acc[k] = 0.f;
  const int e0 = m.blk_ptr[b], e1 = m.blk_ptr[b + 1];
  for (int c0 = e0; c0 < e1; c0 += NB) {
    const int idx = c0 + tid;
    if (idx < e1) {
      const int e = __ldg(m.blk_elems + idx);
      const int4 cn = __ldg(m.conn + e);
      const int nid[4] = {cn.x, cn.y, cn.z, cn.w};
      float xv[4][3];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float4 X = __ldg(m.X32 + nid[k]);
        xv[k][0] = X.x;
        xv[k][1] = X.y;
        xv[k][2] = X.z;
      }
      TetGeom<float> g;
      tet_geom(xv[0], xv[1], xv[2], xv[3], g);
      const DevMat<float>& mat = a.matF[__ldg(m.mat_id + e)];
      const float scale = __ldg(m.scale + e);
      float pay[kPay];
      {
        const int npay = model_pay_words(MODEL >= 0 ? MODEL : mat.model);
#pragma unroll
        for (int k = 0; k < kPay; ++k)
          pay[k] = (k < npay) ? __ldg(a.payload + (size_t)k * m.n_elems + e) : 0.f;
      }
      float w[4][3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        w[1][j] = g.c[0][j];
        w[2][j] = g.c[1][j];
        w[3][j] = g.c[2][j];
        w[0][j] = -(g.c[0][j] + g.c[1][j] + g.c[2][j]);
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          float dF[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) dF[k] = 0.f;
#pragma unroll
          for (int j = 0; j < 3; ++j) dF[3 * i + j] = w[s][j] * g.inv_det;
          float dP[9];
          dP_any<MODEL>(mat, scale, pay, dF, dP);
          if (BLOCK) {
            // force component k at the slot's node for a unit displacement in
            // direction i: entries (i, k), k >= i -> 00 01 02 | 11 12 | 22
#pragma unroll
            for (int k = i; k < 3; ++k) {
              const int ent = (i == 0) ? k : (i == 1 ? 2 + k : 5);
              sf[W * s + ent][tid] =
                  g.s6 * (dP[3 * k] * w[s][0] + dP[3 * k + 1] * w[s][1] + dP[3 * k + 2] * w[s][2]);
            }
          } else {
            sf[W * s + i][tid] =
                g.s6 * (dP[3 * i] * w[s][0] + dP[3 * i + 1] * w[s][1] + dP[3 * i + 2] * w[s][2]);
          }
        }
      }
    }
    __syncthreads();
    gather_chunk_w<NB, W>(s_slots, sf, c0 - e0, cur, end, acc);
    __syncthreads();
  }
  if (!has_node) return;
  diag_store<BLOCK>(acc, m.fixed[node], node, a.dinv, a.boff);
}

// ───────────────────────── PCG vector kernels ─────────────────────────
// FP32 node vectors hold one float4 per node (xyz, 0); fixed DOFs carry
// dinv = 0, so z, p and x stay zero there without masks.  One node per thread.

constexpr int kVecThreads = 256;

__global__ void __launch_bounds__(kVecThreads) cg_init_kernel(const double* __restrict__ b,
                                                              float* r, float* x, float* p,
                                                              const float* __restrict__ dinv,
                                                              int n_nodes, CGState* cg, double rtol,
                                                              int maxit, Reduce red, int site,
                                                              int jac) {
  // b holds 3 doubles per node
  __shared__ double sred[kVecThreads / 32];
  __shared__ bool am_last;
  const int i = blockIdx.x * kVecThreads + threadIdx.x;
  double rz = 0.0, rr = 0.0;
  if (i < n_nodes) {
    const float4 rv = make_float4((float)b[3 * i], (float)b[3 * i + 1], (float)b[3 * i + 2], 0.f);
    const float4 dv = reinterpret_cast<const float4*>(dinv)[i];
    const float4 zv = make_float4(dv.x * rv.x, dv.y * rv.y, dv.z * rv.z, 0.f);
    reinterpret_cast<float4*>(r)[i] = rv;
    if (jac) reinterpret_cast<float4*>(p)[i] = zv;
    reinterpret_cast<float4*>(x)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    rz = jac ? (double)rv.x * zv.x + (double)rv.y * zv.y + (double)rv.z * zv.z : 0.0;
    rr = (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z;
  }
  double v[2];
  v[0] = block_sum<kVecThreads>(rz, sred);
  v[1] = block_sum<kVecThreads>(rr, sred);
  if (publish_partial(red, site, 2, v, &am_last)) {
    double trz = final_sum<kVecThreads>(red, site, 0, sred);
    double trr = final_sum<kVecThreads>(red, site, 1, sred);
    if (threadIdx.x == 0) {
      cg->rz = trz;
      cg->rr = trr;
      cg->rr0 = trr;
      cg->tol2 = rtol * rtol * trr;
      cg->alpha = 0.0;
      cg->beta = 0.0;
      cg->pAp = 0.0;
      cg->iter = 0;
      cg->max_iter = maxit;
      cg->zsel = 0;
      cg->n_alt = 0;
      cg->locked = 0;
      cg->trips = 0;
      cg->status = isfinite(trr) ? 0 : 3;
      cg->done = (!isfinite(trr)) ? 3 : ((trr == 0.0 || (jac && !(trz > 0.0))) ? 1 : 0);
      red.counters[site] = 0u;
    }
  }
}

__global__ void __launch_bounds__(kVecThreads) cg_update_kernel(float* x, float* r,
                                                                const float* __restrict__ p,
                                                                const float* __restrict__ y,
                                                                const float* __restrict__ dinv,
                                                                int n_nodes, CGState* cg, Reduce red,
                                                                int site, int jac) {
  chain_enter();
  if (cg->done) return;
  __shared__ double sred[kVecThreads / 32];
  __shared__ bool am_last;
  const float alpha = (float)cg->alpha;
  const int i = blockIdx.x * kVecThreads + threadIdx.x;
  double rz = 0.0, rr = 0.0;
  if (i < n_nodes) {
    float4 xv = reinterpret_cast<float4*>(x)[i];
    float4 rv = reinterpret_cast<float4*>(r)[i];
    const float4 pv = reinterpret_cast<const float4*>(p)[i];
    const float4 yv = reinterpret_cast<const float4*>(y)[i];
    const float4 dv = reinterpret_cast<const float4*>(dinv)[i];
    xv.x += alpha * pv.x; xv.y += alpha * pv.y; xv.z += alpha * pv.z;
    rv.x -= alpha * yv.x; rv.y -= alpha * yv.y; rv.z -= alpha * yv.z;
    reinterpret_cast<float4*>(x)[i] = xv;
    reinterpret_cast<float4*>(r)[i] = rv;
    if (jac) rz = (double)rv.x * (dv.x * rv.x) + (double)rv.y * (dv.y * rv.y) + (double)rv.z * (dv.z * rv.z);
    rr = (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z;
  }
  double v[2];
  v[0] = block_sum<kVecThreads>(rz, sred);
  v[1] = block_sum<kVecThreads>(rr, sred);
  if (publish_partial(red, site, 2, v, &am_last)) {
    double trz = final_sum<kVecThreads>(red, site, 0, sred);
    double trr = final_sum<kVecThreads>(red, site, 1, sred);
    if (threadIdx.x == 0) {
      if (jac) {
        cg->beta = trz / cg->rz;
        cg->rz = trz;
      }
      cg->rr = trr;
      cg->iter += 1;
      if (!isfinite(trr) || (jac && !isfinite(trz))) {
        cg->done = 3;
        cg->status = 3;
      } else if (trr <= cg->tol2) {
        cg->done = 1;
      } else if (cg->iter >= cg->max_iter) {
        cg->done = 2;
      }
      red.counters[site] = 0u;
    }
  }
}

__global__ void __launch_bounds__(kVecThreads) cg_pupdate_kernel(float* p,
                                                                 const float* __restrict__ r,
                                                                 const float* __restrict__ dinv,
                                                                 int n_nodes, const CGState* cg) {
  chain_enter();
  if (cg->done) return;
  const float beta = (float)cg->beta;
  const int i = blockIdx.x * kVecThreads + threadIdx.x;
  if (i < n_nodes) {
    float4 pv = reinterpret_cast<float4*>(p)[i];
    const float4 rv = reinterpret_cast<const float4*>(r)[i];
    const float4 dv = reinterpret_cast<const float4*>(dinv)[i];
    pv.x = dv.x * rv.x + beta * pv.x;
    pv.y = dv.y * rv.y + beta * pv.y;
    pv.z = dv.z * rv.z + beta * pv.z;
    reinterpret_cast<float4*>(p)[i] = pv;
  }
}

// ───────────────────────── element-parallel helpers (FP64) ─────────────────────────

template <int MODEL>
__global__ void stress_kernel(const MeshDev m, const DevMat<double>* matD, const double* u,
                              const double* ep_c, const double* epe_c, const int* perm_elem,
                              double* F_out, double* sig_out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n_elems) return;
  const int4 cn = m.conn[e];
  const int nid[4] = {cn.x, cn.y, cn.z, cn.w};
  double xv[4][3], uv[4][3];
  for (int k = 0; k < 4; ++k)
    for (int d = 0; d < 3; ++d) {
      xv[k][d] = m.X64[3 * nid[k] + d];
      uv[k][d] = u[3 * nid[k] + d];
    }
  TetGeom<double> g;
  tet_geom(xv[0], xv[1], xv[2], xv[3], g);
  double D[3][3];
  for (int k = 0; k < 3; ++k)
    for (int d = 0; d < 3; ++d) D[k][d] = uv[k + 1][d] - uv[0][d];
  double Hg[9], F[9];
  grad_from_diffs(D, g, Hg);
  for (int k = 0; k < 9; ++k) F[k] = Hg[k] + ((k % 4 == 0) ? 1.0 : 0.0);
  const DevMat<double>& mat = matD[m.mat_id[e]];
  const double scale = (double)m.scale[e];
  const int model = MODEL >= 0 ? MODEL : mat.model;
  double sig[9];
  float pay[kPay];
  if (model == M_NH || model == M_MR || model == M_FMR) {
    // Cauchy stress sigma = P F^T / J_s (the stress kernels of neo_hookean.py:99-129 and
    // mooney_rivlin.py:150-190 evaluate the same tensor directly)
    double P[9];
    if (model == M_NH)
      nh_stress(mat, scale, Hg, P, pay);
    else
      mr_stress(mat, scale, Hg, P, pay);
    const double J = det3(F);
    const double Js = J > kJFloor ? J : kJFloor;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        sig[3 * i + j] =
            (P[3 * i] * F[3 * j] + P[3 * i + 1] * F[3 * j + 1] + P[3 * i + 2] * F[3 * j + 2]) / Js;
  } else if (model == M_J2) {
    double ep[6], epn[6], epe_n;
    for (int k = 0; k < 6; ++k) ep[k] = ep_c[(size_t)k * m.n_elems + e];
    j2_stress(mat, scale, Hg, ep, epe_c[e], sig, epn, epe_n, pay);
  } else if (model == M_TI) {
    ti_stress(mat, scale, Hg, sig);
  } else {
    le_stress(mat, scale, Hg, sig);
  }
  const int eu = perm_elem[e];
  for (int k = 0; k < 9; ++k) {
    if (F_out) F_out[(size_t)9 * eu + k] = F[k];
    if (sig_out) sig_out[(size_t)9 * eu + k] = sig[k];
  }
}

// Nodal von Mises stress: per node, the von Mises stress of each element on
// it (from the elements' Cauchy stresses in caller order) added in the
// node's fixed slot order; average = 1 divides by the number of elements.
// Written in caller node order.  core/mesh.py:459-492 accumulates the sum
// with atomics and never divides (its average step is a comment).
__global__ void nodal_mises_kernel(const MeshDev m, const int* perm_elem, const int* perm_node,
                                   const double* sig_user, int average, double* out_user) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= m.n_nodes) return;
  const int b = n / m.nb;
  const int base = m.blk_ptr[b];
  const int j0 = m.node_row[n], j1 = m.node_row[n + 1];
  double acc = 0.0;
  const int ngp = m.npe == 8 ? kHexGauss : 1;
  for (int j = j0; j < j1; ++j) {
    const int li = (int)(m.node_slots[j] >> m.slot_shift);
    const int e = m.blk_elems[base + li];
    // the element's Gauss-point mean stress (core/mesh.py:470-474)
    const double* sp = sig_user + (size_t)9 * ngp * perm_elem[e];
    double s[9];
    for (int k = 0; k < 9; ++k) s[k] = sp[k];
    for (int g = 1; g < ngp; ++g)
      for (int k = 0; k < 9; ++k) s[k] += sp[9 * g + k];
    if (ngp > 1)
      for (int k = 0; k < 9; ++k) s[k] /= (double)ngp;
    const double s11 = s[0], s22 = s[4], s33 = s[8], s12 = s[1], s23 = s[5], s13 = s[2];
    acc += sqrt(0.5 * ((s11 - s22) * (s11 - s22) + (s22 - s33) * (s22 - s33) + (s33 - s11) * (s33 - s11) +
                       6.0 * (s12 * s12 + s23 * s23 + s13 * s13)));
  }
  if (average && j1 > j0) acc /= (double)(j1 - j0);
  out_user[perm_node[n]] = acc;
}

__global__ void refq_kernel(const MeshDev m, const int* perm_elem, double* dNdX, double* vol) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n_elems) return;
  const int4 cn = m.conn[e];
  const int nid[4] = {cn.x, cn.y, cn.z, cn.w};
  double xv[4][3];
  for (int k = 0; k < 4; ++k)
    for (int d = 0; d < 3; ++d) xv[k][d] = m.X64[3 * nid[k] + d];
  TetGeom<double> g;
  tet_geom(xv[0], xv[1], xv[2], xv[3], g);
  const int eu = perm_elem[e];
  if (dNdX) {
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) {
        const double v = g.c[k][j] * g.inv_det;
        dNdX[(size_t)12 * eu + 3 * (k + 1) + j] = v;
        s += v;
      }
      dNdX[(size_t)12 * eu + j] = -s;
    }
  }
  if (vol) vol[eu] = g.vol;
}

// ───────────────────────── small helpers ─────────────────────────

template <typename TI, typename TO>
__global__ void gather3_kernel(const TI* in_user, TO* out_int, const int* perm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int src = perm[i];
  for (int d = 0; d < 3; ++d) out_int[3 * i + d] = (TO)in_user[3 * src + d];
}

template <typename TI, typename TO>
__global__ void scatter3_kernel(const TI* in_int, TO* out_user, const int* perm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int dst = perm[i];
  for (int d = 0; d < 3; ++d) out_user[3 * dst + d] = (TO)in_int[3 * i + d];
}

__global__ void gather_mask_kernel(const uint8_t* in_user, uint8_t* out_int, const int* perm,
                                   int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int src = perm[i];
  uint8_t bits = 0;
  for (int d = 0; d < 3; ++d) bits |= (in_user[3 * src + d] ? 1 : 0) << d;
  out_int[i] = bits;
}

__global__ void apply_bc_kernel(double* u, const double* fixed_vals, const uint8_t* fixed, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t fx = fixed[i];
  for (int d = 0; d < 3; ++d)
    if ((fx >> d) & 1) u[3 * i + d] = fixed_vals[3 * i + d];
}

__global__ void u_update_kernel(double* u, const double* u_base, const float* du, double alpha,
                                int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 d = reinterpret_cast<const float4*>(du)[i];
  u[3 * i] = u_base[3 * i] + alpha * (double)d.x;
  u[3 * i + 1] = u_base[3 * i + 1] + alpha * (double)d.y;
  u[3 * i + 2] = u_base[3 * i + 2] + alpha * (double)d.z;
}

// one float4 per node -> three doubles per node
__global__ void f4_to_d3_kernel(const float* __restrict__ in, double* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 v = reinterpret_cast<const float4*>(in)[i];
  out[3 * i] = v.x;
  out[3 * i + 1] = v.y;
  out[3 * i + 2] = v.z;
}

// x += x0 (one float4 per node)
__global__ void f4_add_kernel(float* x, const float* __restrict__ x0, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = reinterpret_cast<float4*>(x)[i];
  const float4 w = reinterpret_cast<const float4*>(x0)[i];
  v.x += w.x;
  v.y += w.y;
  v.z += w.z;
  reinterpret_cast<float4*>(x)[i] = v;
}

// load-step extrapolation: u = u_last + du_last
__global__ void extrap_kernel(double* u, const double* u_last, const double* du_last, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) u[i] = u_last[i] + du_last[i];
}

// *differ |= 1 where a and b differ
__global__ void differ_kernel(const double* a, const double* b, int n, unsigned int* differ) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && a[i] != b[i]) atomicOr(differ, 1u);
}

// after a converged solve that started at u_start: du_last = u - u_start, u_last = u
__global__ void extrap_record_kernel(const double* u, const double* u_start, double* u_last, double* du_last,
                                     int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  du_last[i] = u[i] - u_start[i];
  u_last[i] = u[i];
}

// float4-per-node <-> 3-per-node caller layout
__global__ void gather_f4_kernel(const float* in_user, float* out_int, const int* perm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int src = perm[i];
  reinterpret_cast<float4*>(out_int)[i] =
      make_float4(in_user[3 * src], in_user[3 * src + 1], in_user[3 * src + 2], 0.f);
}

template <typename TO>
__global__ void scatter_f4_kernel(const float* in_int, TO* out_user, const int* perm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int dst = perm[i];
  const float4 v = reinterpret_cast<const float4*>(in_int)[i];
  out_user[3 * dst] = (TO)v.x;
  out_user[3 * dst + 1] = (TO)v.y;
  out_user[3 * dst + 2] = (TO)v.z;
}

__global__ void x32_mask_kernel(float4* X32, const uint8_t* fixed, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  X32[i].w = (float)fixed[i];
}

__global__ void gather3_masked_kernel(const double* in_user, double* out_int, const int* perm,
                                      const uint8_t* fixed, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int src = perm[i];
  const uint8_t fx = fixed[i];
  for (int d = 0; d < 3; ++d) out_int[3 * i + d] = ((fx >> d) & 1) ? 0.0 : in_user[3 * src + d];
}

__global__ void dinv_identity_kernel(float* dinv, const uint8_t* fixed, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t fx = fixed[i];
  reinterpret_cast<float4*>(dinv)[i] =
      make_float4((fx & 1) ? 0.f : 1.f, (fx & 2) ? 0.f : 1.f, (fx & 4) ? 0.f : 1.f, 0.f);
}

__global__ void __launch_bounds__(256) bc_delta_kernel(const double* u, const double* fixed_vals,
                                                       const uint8_t* fixed, float* dc, int n,
                                                       Reduce red, int site, double* dc2) {
  __shared__ double sred[8];
  __shared__ bool am_last;
  const int i = blockIdx.x * 256 + threadIdx.x;
  double acc = 0.0;
  if (i < n) {
    const uint8_t fx = fixed[i];
    float dv[3];
    for (int d = 0; d < 3; ++d) {
      const double v = ((fx >> d) & 1) ? fixed_vals[3 * i + d] - u[3 * i + d] : 0.0;
      dv[d] = (float)v;
      acc += v * v;
    }
    reinterpret_cast<float4*>(dc)[i] = make_float4(dv[0], dv[1], dv[2], 0.f);
  }
  double bsum = block_sum<256>(acc, sred);
  if (publish_partial(red, site, 1, &bsum, &am_last)) {
    double tot = final_sum<256>(red, site, 0, sred);
    if (threadIdx.x == 0) {
      *dc2 = tot;
      red.counters[site] = 0u;
    }
  }
}

__global__ void rhs_minus_kernel(const double* R, const float* y, const uint8_t* fixed, double* out,
                                 int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t fx = fixed[i];
  const float4 yv = reinterpret_cast<const float4*>(y)[i];
  const float ys[3] = {yv.x, yv.y, yv.z};
  for (int d = 0; d < 3; ++d) out[3 * i + d] = ((fx >> d) & 1) ? 0.0 : R[3 * i + d] - (double)ys[d];
}

// ───────────────────────── launchers ─────────────────────────

static inline int nblk(int n, int t) { return (n + t - 1) / t; }

// CTAs that fit on the device at once (resident per SM x SMs) for a
// persistent kernel of `threads` threads and no dynamic shared memory.
template <typename K>
static int resident_grid(K kernel, int threads) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0);
  return (sms > 0 ? sms : 1) * (per > 0 ? per : 1);
}

void launch_f4_to_d3(const float* in, double* out, int n_nodes, cudaStream_t s) {
  f4_to_d3_kernel<<<nblk(n_nodes, 256), 256, 0, s>>>(in, out, n_nodes);
}
void launch_f4_add(float* x, const float* x0, int n_nodes, cudaStream_t s) {
  f4_add_kernel<<<nblk(n_nodes, 256), 256, 0, s>>>(x, x0, n_nodes);
}
void launch_extrap(double* u, const double* u_last, const double* du_last, int n, cudaStream_t s) {
  extrap_kernel<<<nblk(n, 256), 256, 0, s>>>(u, u_last, du_last, n);
}
void launch_differ(const double* a, const double* b, int n, unsigned int* differ, cudaStream_t s) {
  differ_kernel<<<nblk(n, 256), 256, 0, s>>>(a, b, n, differ);
}
void launch_extrap_record(const double* u, const double* u_start, double* u_last, double* du_last, int n,
                          cudaStream_t s) {
  extrap_record_kernel<<<nblk(n, 256), 256, 0, s>>>(u, u_start, u_last, du_last, n);
}


// Every launch below raises its kernel's shared-memory limit to the device
// maximum first (once per kernel; also before stream capture, in
// prepare_kernels).
template <typename K>
static void allow_smem(K kernel, size_t, cudaStream_t) {
  raise_smem_limit_k(kernel);
}

static size_t slots_smem(const MeshDev& m) { return sizeof(uint32_t) * (size_t)m.max_slots; }

template <int NB, int MODEL>
static void residual_go(const ResArgs& a, cudaStream_t s) {
  const size_t smem = sizeof(double) * 12 * NB + slots_smem(a.m);
  allow_smem(residual_kernel<NB, MODEL>, smem, s);
  residual_kernel<NB, MODEL><<<a.m.n_blocks, NB, smem, s>>>(a);
}

template <int NB>
static void residual_nb(const ResArgs& a, int model, cudaStream_t s) {
  switch (model) {
    case M_LE: residual_go<NB, M_LE>(a, s); break;
    case M_NH: residual_go<NB, M_NH>(a, s); break;
    case M_MR: residual_go<NB, M_MR>(a, s); break;
    case M_J2: residual_go<NB, M_J2>(a, s); break;
    case M_TI: residual_go<NB, M_TI>(a, s); break;
    case M_FMR: residual_go<NB, M_FMR>(a, s); break;
    default: residual_go<NB, -1>(a, s); break;
  }
}

template <int MODEL>
static void res_elem(const ResArgs& a, cudaStream_t s) {
  static const int grid = resident_grid(res_elem_kernel<MODEL>, 128);
  res_elem_kernel<MODEL><<<std::min(grid, nblk(a.m.n_elems, 128)), 128, 0, s>>>(a);
}

static void residual_two_phase(const ResArgs& a, int model, cudaStream_t s) {
  switch (model) {
    case M_LE: res_elem<M_LE>(a, s); break;
    case M_NH: res_elem<M_NH>(a, s); break;
    case M_MR: res_elem<M_MR>(a, s); break;
    case M_J2: res_elem<M_J2>(a, s); break;
    case M_TI: res_elem<M_TI>(a, s); break;
    case M_FMR: res_elem<M_FMR>(a, s); break;
    default: res_elem<-1>(a, s); break;
  }
  static const int ggrid = resident_grid(res_gather_kernel<kGatherLanes>, 256);
  res_gather_kernel<kGatherLanes><<<std::min(ggrid, nblk(a.m.n_nodes, 256 / kGatherLanes)), 256, 0, s>>>(a);
}

void launch_residual(const ResArgs& a, int model, cudaStream_t s) {
  if (a.m.npe == 8) {
    launch_residual_hex(a, model, s);
    return;
  }
  if (a.stage_d) {
    residual_two_phase(a, model, s);
    return;
  }
  switch (a.m.nb) {
    case 128: residual_nb<128>(a, model, s); break;
    case 512: residual_nb<512>(a, model, s); break;
    default: residual_nb<256>(a, model, s); break;
  }
}

template <int NB, int MODEL, bool CG>
static void matvec_go(const MvArgs& a, cudaStream_t s) {
  const size_t smem = slots_smem(a.m);
  allow_smem(matvec_kernel<NB, MODEL, CG>, smem, s);
  launch_chain(matvec_kernel<NB, MODEL, CG>, a.m.n_blocks, NB, smem, s, a);
}

template <int NB, bool CG>
static void matvec_nb(const MvArgs& a, int model, cudaStream_t s) {
  switch (model) {
    case M_LE: matvec_go<NB, M_LE, CG>(a, s); break;
    case M_NH: matvec_go<NB, M_NH, CG>(a, s); break;
    case M_MR: matvec_go<NB, M_MR, CG>(a, s); break;
    case M_J2: matvec_go<NB, M_J2, CG>(a, s); break;
    case M_TI: matvec_go<NB, M_TI, CG>(a, s); break;
    case M_FMR: matvec_go<NB, M_FMR, CG>(a, s); break;
    default: matvec_go<NB, -1, CG>(a, s); break;
  }
}


template <bool CG>
static void two_phase(const MvArgs& a, int model, cudaStream_t s) {
  const int ge = nblk(a.m.n_elems, 256);
  switch (model) {
    case M_LE: launch_chain(elem_mv_kernel<M_LE, CG>, ge, 256, 0, s, a); break;
    case M_NH: launch_chain(elem_mv_kernel<M_NH, CG>, ge, 256, 0, s, a); break;
    case M_MR: launch_chain(elem_mv_kernel<M_MR, CG>, ge, 256, 0, s, a); break;
    case M_J2: launch_chain(elem_mv_kernel<M_J2, CG>, ge, 256, 0, s, a); break;
    case M_TI: launch_chain(elem_mv_kernel<M_TI, CG>, ge, 256, 0, s, a); break;
    case M_FMR: launch_chain(elem_mv_kernel<M_FMR, CG>, ge, 256, 0, s, a); break;
    default: launch_chain(elem_mv_kernel<-1, CG>, ge, 256, 0, s, a); break;
  }
  launch_chain(node_gather_kernel<CG>, nblk(a.m.n_nodes, kGatherNodes), 256, 0, s, a);
}


template <int MODEL, bool CG>
static void persist_elem(const MvArgs& a, cudaStream_t s) {
  static const int grid = resident_grid(elem_mv_persist_kernel<MODEL, CG>, 256);
  launch_chain(elem_mv_persist_kernel<MODEL, CG>, std::min(grid, nblk(a.m.n_elems, 256)), 256, 0, s, a);
}

template <bool CG>
static void two_phase_persist(const MvArgs& a, int model, cudaStream_t s) {
  switch (model) {
    case M_LE: persist_elem<M_LE, CG>(a, s); break;
    case M_NH: persist_elem<M_NH, CG>(a, s); break;
    case M_MR: persist_elem<M_MR, CG>(a, s); break;
    case M_J2: persist_elem<M_J2, CG>(a, s); break;
    case M_TI: persist_elem<M_TI, CG>(a, s); break;
    case M_FMR: persist_elem<M_FMR, CG>(a, s); break;
    default: persist_elem<-1, CG>(a, s); break;
  }
  static const int ggrid = resident_grid(node_gather_persist_kernel<CG>, 256);
  launch_chain(node_gather_persist_kernel<CG>, std::min(ggrid, nblk(a.m.n_nodes, kGatherNodes)), 256, 0, s, a);
}

template <int MODEL, bool CG>
static void wagg_elem(const MvArgs& a, cudaStream_t s) {
  static const int grid = resident_grid(elem_wagg_kernel<MODEL, CG>, 32 * kWaggWarps);
  launch_chain(elem_wagg_kernel<MODEL, CG>, std::min(grid, nblk(nblk(a.m.n_elems, 32), kWaggWarps)),
               32 * kWaggWarps, 0, s, a);
}

template <bool CG>
static void warp_agg(const MvArgs& a, int model, cudaStream_t s) {
  switch (model) {
    case M_LE: wagg_elem<M_LE, CG>(a, s); break;
    case M_NH: wagg_elem<M_NH, CG>(a, s); break;
    case M_MR: wagg_elem<M_MR, CG>(a, s); break;
    case M_J2: wagg_elem<M_J2, CG>(a, s); break;
    case M_TI: wagg_elem<M_TI, CG>(a, s); break;
    case M_FMR: wagg_elem<M_FMR, CG>(a, s); break;
    default: wagg_elem<-1, CG>(a, s); break;
  }
  // the persistent node gather over the partial rows
  MvArgs g = a;
  g.m.node_row = a.wa.prow;
  g.stage = a.wa.parts;
  static const int ggrid = resident_grid(node_gather_persist_kernel<CG>, 256);
  launch_chain(node_gather_persist_kernel<CG>, std::min(ggrid, nblk(a.m.n_nodes, kGatherNodes)), 256, 0, s, g);
}

void launch_node_gather(const MvArgs& a, cudaStream_t s) {
  if (a.cg)
    launch_chain(node_gather_kernel<true>, nblk(a.m.n_nodes, kGatherNodes), 256, 0, s, a);
  else
    launch_chain(node_gather_kernel<false>, nblk(a.m.n_nodes, kGatherNodes), 256, 0, s, a);
}

void launch_matvec(const MvArgs& a, int model, cudaStream_t s) {
  if (a.m.npe == 8) {
    launch_matvec_hex(a, model, s);
    return;
  }
  const bool cg = a.cg != nullptr;
  if (a.variant == MV_WARP_AGG && a.wa.parts != nullptr) {
    cg ? warp_agg<true>(a, model, s) : warp_agg<false>(a, model, s);
    return;
  }
  if (a.variant == MV_ELEM_BLOCK && a.eb.nodes != nullptr) {
    launch_matvec_eb(a, model, s);
    return;
  }
  if (a.variant == MV_ELEM_BLOCK || a.variant == MV_WARP_AGG) {
    // no tables (the host builds them whenever it selects the variant): the
    // two-phase pass gives the same product
    cg ? two_phase<true>(a, model, s) : two_phase<false>(a, model, s);
    return;
  }
  if (a.variant == MV_TWO_PHASE) {
    cg ? two_phase<true>(a, model, s) : two_phase<false>(a, model, s);
    return;
  }
  if (a.variant == MV_PERSIST) {
    cg ? two_phase_persist<true>(a, model, s) : two_phase_persist<false>(a, model, s);
    return;
  }
  switch (a.m.nb) {
    case 128: cg ? matvec_nb<128, true>(a, model, s) : matvec_nb<128, false>(a, model, s); break;
    case 512: cg ? matvec_nb<512, true>(a, model, s) : matvec_nb<512, false>(a, model, s); break;
    default: cg ? matvec_nb<256, true>(a, model, s) : matvec_nb<256, false>(a, model, s); break;
  }
}

template <int NB>
static void prepare_nb(int model, size_t smem) {
  (void)smem;
  auto set = [&](auto k) { raise_smem_limit_k(k); };
  switch (model) {
    case M_LE: set(matvec_kernel<NB, M_LE, true>); break;
    case M_NH: set(matvec_kernel<NB, M_NH, true>); break;
    case M_MR: set(matvec_kernel<NB, M_MR, true>); break;
    case M_J2: set(matvec_kernel<NB, M_J2, true>); break;
    case M_TI: set(matvec_kernel<NB, M_TI, true>); break;
    case M_FMR: set(matvec_kernel<NB, M_FMR, true>); break;
    default: set(matvec_kernel<NB, -1, true>); break;
  }
}

void prepare_kernels(const MeshDev& m, int model) {
  switch (m.nb) {
    case 128: prepare_nb<128>(model, slots_smem(m)); break;
    case 512: prepare_nb<512>(model, slots_smem(m)); break;
    default: prepare_nb<256>(model, slots_smem(m)); break;
  }
}

template <int NB, int MODEL>
static void diag_go(const DiagArgs& a, cudaStream_t s) {
  const size_t smem = slots_smem(a.m);
  if (a.boff) {
    allow_smem(diag_kernel<NB, MODEL, true>, smem, s);
    diag_kernel<NB, MODEL, true><<<a.m.n_blocks, NB, smem, s>>>(a);
    return;
  }
  allow_smem(diag_kernel<NB, MODEL, false>, smem, s);
  diag_kernel<NB, MODEL, false><<<a.m.n_blocks, NB, smem, s>>>(a);
}

template <int NB>
static void diag_nb(const DiagArgs& a, int model, cudaStream_t s) {
  switch (model) {
    case M_LE: diag_go<NB, M_LE>(a, s); break;
    case M_NH: diag_go<NB, M_NH>(a, s); break;
    case M_MR: diag_go<NB, M_MR>(a, s); break;
    case M_J2: diag_go<NB, M_J2>(a, s); break;
    case M_TI: diag_go<NB, M_TI>(a, s); break;
    case M_FMR: diag_go<NB, M_FMR>(a, s); break;
    default: diag_go<NB, -1>(a, s); break;
  }
}

void launch_diag(const DiagArgs& a, int model, cudaStream_t s) {
  if (a.m.npe == 8) {
    launch_diag_hex(a, model, s);
    return;
  }
  switch (a.m.nb) {
    case 128: diag_nb<128>(a, model, s); break;
    case 512: diag_nb<512>(a, model, s); break;
    default: diag_nb<256>(a, model, s); break;
  }
}

void launch_cg_init(const double* b, float* r, float* x, float* p, const float* dinv, int n_nodes,
                    CGState* cg, double rtol, int maxit, Reduce red, int site, cudaStream_t s,
                    int precond_in_update) {
  cg_init_kernel<<<nblk(n_nodes, kVecThreads), kVecThreads, 0, s>>>(b, r, x, p, dinv, n_nodes, cg,
                                                                    rtol, maxit, red, site,
                                                                    precond_in_update);
}

void launch_cg_update(float* x, float* r, const float* p, const float* y, const float* dinv,
                      int n_nodes, CGState* cg, Reduce red, int site, cudaStream_t s,
                      int precond_in_update) {
  launch_chain(cg_update_kernel, nblk(n_nodes, kVecThreads), kVecThreads, 0, s, x, r, p, y, dinv, n_nodes, cg,
               red, site, precond_in_update);
}

void launch_cg_pupdate(float* p, const float* r, const float* dinv, int n_nodes, CGState* cg,
                       cudaStream_t s) {
  launch_chain(cg_pupdate_kernel, nblk(n_nodes, kVecThreads), kVecThreads, 0, s, p, r, dinv, n_nodes,
               static_cast<const CGState*>(cg));
}

void launch_stress(const MeshDev& m, const DevMat<double>* matD, int model, const double* u,
                   const double* ep_c, const double* epe_c, const int* perm_elem, double* F_out,
                   double* sig_out, cudaStream_t s) {
  if (m.npe == 8) {
    launch_stress_hex(m, matD, model, u, ep_c, epe_c, perm_elem, F_out, sig_out, s);
    return;
  }
  const int t = 128;
  switch (model) {
    case M_LE: stress_kernel<M_LE><<<nblk(m.n_elems, t), t, 0, s>>>(m, matD, u, ep_c, epe_c, perm_elem, F_out, sig_out); break;
    case M_NH: stress_kernel<M_NH><<<nblk(m.n_elems, t), t, 0, s>>>(m, matD, u, ep_c, epe_c, perm_elem, F_out, sig_out); break;
    case M_J2: stress_kernel<M_J2><<<nblk(m.n_elems, t), t, 0, s>>>(m, matD, u, ep_c, epe_c, perm_elem, F_out, sig_out); break;
    default: stress_kernel<-1><<<nblk(m.n_elems, t), t, 0, s>>>(m, matD, u, ep_c, epe_c, perm_elem, F_out, sig_out); break;
  }
}

void launch_nodal_mises(const MeshDev& m, const int* perm_elem, const int* perm_node, const double* sig_user,
                        int average, double* out_user, cudaStream_t s) {
  nodal_mises_kernel<<<nblk(m.n_nodes, 256), 256, 0, s>>>(m, perm_elem, perm_node, sig_user, average, out_user);
}

void launch_refq(const MeshDev& m, const int* perm_elem, double* dNdX, double* vol,
                 cudaStream_t s) {
  if (m.npe == 8) {
    launch_refq_hex(m, perm_elem, dNdX, vol, s);
    return;
  }
  refq_kernel<<<nblk(m.n_elems, 128), 128, 0, s>>>(m, perm_elem, dNdX, vol);
}

void launch_gather_d(const double* in_user, double* out_int, const int* perm, int n,
                     cudaStream_t s) {
  gather3_kernel<double, double><<<nblk(n, 256), 256, 0, s>>>(in_user, out_int, perm, n);
}
void launch_scatter_d(const double* in_int, double* out_user, const int* perm, int n,
                      cudaStream_t s) {
  scatter3_kernel<double, double><<<nblk(n, 256), 256, 0, s>>>(in_int, out_user, perm, n);
}
void launch_gather_f(const float* in_user, float* out_int, const int* perm, int n,
                     cudaStream_t s) {
  gather_f4_kernel<<<nblk(n, 256), 256, 0, s>>>(in_user, out_int, perm, n);
}
void launch_scatter_f(const float* in_int, float* out_user, const int* perm, int n,
                      cudaStream_t s) {
  scatter_f4_kernel<float><<<nblk(n, 256), 256, 0, s>>>(in_int, out_user, perm, n);
}
void launch_scatter_f2d(const float* in_int, double* out_user, const int* perm, int n,
                        cudaStream_t s) {
  scatter_f4_kernel<double><<<nblk(n, 256), 256, 0, s>>>(in_int, out_user, perm, n);
}
__global__ void scale_d_kernel(const double* in, double s, double* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = s * in[i];
}

void launch_scale_d(const double* in, double s, double* out, int n, cudaStream_t st) {
  scale_d_kernel<<<nblk(n, 256), 256, 0, st>>>(in, s, out, n);
}

__global__ void cg_loop_cond_kernel(cudaGraphConditionalHandle h, CGState* cg, int iters_per_trip) {
  chain_enter();
  if (threadIdx.x != 0) return;
  const int trips = ++cg->trips;
  const int cap = cg->max_iter / iters_per_trip + 2;
  bool go = cg->done == 0;
  if (go && trips >= cap) {
    cg->done = 2;
    go = false;
  }
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

void launch_cg_loop_cond(cudaGraphConditionalHandle h, CGState* cg, int iters_per_trip, cudaStream_t s) {
  launch_chain(cg_loop_cond_kernel, 1, 32, 0, s, h, cg, iters_per_trip);
}

void launch_x32_mask(float4* X32, const uint8_t* fixed, int n, cudaStream_t s) {
  x32_mask_kernel<<<nblk(n, 256), 256, 0, s>>>(X32, fixed, n);
}
void launch_gather_mask(const uint8_t* in_user, uint8_t* out_int, const int* perm, int n,
                        cudaStream_t s) {
  gather_mask_kernel<<<nblk(n, 256), 256, 0, s>>>(in_user, out_int, perm, n);
}
void launch_apply_bc(double* u, const double* fixed_vals, const uint8_t* fixed, int n,
                     cudaStream_t s) {
  apply_bc_kernel<<<nblk(n, 256), 256, 0, s>>>(u, fixed_vals, fixed, n);
}
void launch_u_update(double* u, const double* u_base, const float* du, double alpha, int n,
                     cudaStream_t s) {
  u_update_kernel<<<nblk(n, 256), 256, 0, s>>>(u, u_base, du, alpha, n);
}
void launch_gather_d_masked(const double* in_user, double* out_int, const int* perm,
                            const uint8_t* fixed, int n, cudaStream_t s) {
  gather3_masked_kernel<<<nblk(n, 256), 256, 0, s>>>(in_user, out_int, perm, fixed, n);
}
void launch_dinv_identity(float* dinv, const uint8_t* fixed, int n, cudaStream_t s) {
  dinv_identity_kernel<<<nblk(n, 256), 256, 0, s>>>(dinv, fixed, n);
}
void launch_bc_delta(const double* u, const double* fixed_vals, const uint8_t* fixed, float* dc,
                     int n, Reduce red, int site, double* dc2, cudaStream_t s) {
  bc_delta_kernel<<<nblk(n, 256), 256, 0, s>>>(u, fixed_vals, fixed, dc, n, red, site, dc2);
}
void launch_rhs_minus(const double* R, const float* y, const uint8_t* fixed, double* out, int n,
                      cudaStream_t s) {
  rhs_minus_kernel<<<nblk(n, 256), 256, 0, s>>>(R, y, fixed, out, n);
}

}  // namespace femb200
