// Two-level preconditioner of the PCG solve: Jacobi on the mesh plus a
// Galerkin coarse correction on a regular lattice of trilinear cells,
//
//   z = D^-1 r + P Ac^-1 P^T r,   Ac = P^T K_T P   (free DOFs only).
//
// P interpolates coarse-node displacements trilinearly to the mesh nodes.
// Each mesh node lives in one lattice cell (the cell of one of its elements);
// each element is assembled in the cell of its centroid with its nodes'
// trilinear weights clamped to that cell.  On voxel meshes whose cells are
// whole multiples of the voxel, both views of P coincide and Ac is exactly
// P^T K P; elsewhere Ac is a sum of per-element Galerkin blocks, still SPD.
//
// No reference counterpart: the reference solves the assembled system with
// spsolve / ILU-CG (backend/fea/fem/solver/static_solver.py:399-462).
#include <cuda_runtime.h>

#include <algorithm>

#include "fem_internal.h"
#include "fem_lattice.cuh"
#include "fem_reduce.cuh"

namespace femb200 {

namespace {

template <int NT>
__device__ __forceinline__ float block_sum_f(float v, float* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  float r = 0.f;
  if (w == 0) {
    r = (l < NT / 32) ? sh[l] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;  // valid in thread 0
}

}  // namespace

// ───────────────────────── coarse operator assembly ─────────────────────────
// One CTA per lattice cell.  Chunks of kCellThreads elements: each thread
// writes its element's 12x12 tangent (fixed rows and columns zeroed) and the
// 4x8 trilinear weights to shared memory; then each thread owns up to five of
// the cell's 24x24 block entries and adds w_a,c1 K_ab w_b,c2 over the chunk,
// in element order (FP32 products, FP64 accumulation).
constexpr int kCellThreads = 128;
constexpr int kCellEntries = 576;  // (8 corners x 3)^2
constexpr int kCellOwned = (kCellEntries + kCellThreads - 1) / kCellThreads;
// CTAs per cell: slice s takes chunks s, s + kCellSlices, ... of the cell's
// elements; the dense kernel adds the slices in order
constexpr int kCellSlices = 8;

template <int MODEL>
__global__ void __launch_bounds__(kCellThreads) coarse_cell_kernel(const __grid_constant__ CoarseArgs a) {
  extern __shared__ __align__(16) float s_cell[];
  float* sK = s_cell;                                // [kCellThreads][144]
  float* sW = s_cell + kCellThreads * 144;           // [kCellThreads][32]
  const MeshDev& m = a.m;
  const CoarseDev& c = a.c;
  const int cell = blockIdx.x / kCellSlices, slice = blockIdx.x - cell * kCellSlices;
  const int tid = threadIdx.x;
  const int3 ijk = c.cell_ijk[cell];
  const int e0 = c.cell_elem_ptr[cell], e1 = c.cell_elem_ptr[cell + 1];
  double acc[kCellOwned];
#pragma unroll
  for (int k = 0; k < kCellOwned; ++k) acc[k] = 0.0;
  for (int c0 = e0 + slice * kCellThreads; c0 < e1; c0 += kCellSlices * kCellThreads) {
    const int idx = c0 + tid;
    float* K = sK + tid * 144;
    float* W = sW + tid * 32;
    if (idx < e1) {
      const int e = __ldg(c.cell_elems + idx);
      const int4 cn = __ldg(m.conn + e);
      const int nid[4] = {cn.x, cn.y, cn.z, cn.w};
      float xv[4][3];
      int fx[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float4 X = __ldg(m.X32 + nid[k]);
        xv[k][0] = X.x;
        xv[k][1] = X.y;
        xv[k][2] = X.z;
        fx[k] = (int)m.fixed[nid[k]];
        float t[3];
        cell_local(c, ijk, X.x, X.y, X.z, t);
#pragma unroll
        for (int q = 0; q < 8; ++q) W[k * 8 + q] = tri_weight(t[0], t[1], t[2], q);
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
      for (int b = 0; b < 4; ++b) {
#pragma unroll
        for (int d2 = 0; d2 < 3; ++d2) {
          const bool col_fixed = (fx[b] >> d2) & 1;
          float dF[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) dF[k] = 0.f;
#pragma unroll
          for (int j = 0; j < 3; ++j) dF[3 * d2 + j] = w[b][j] * g.inv_det;
          float dP[9];
          dP_any<MODEL>(mat, scale, pay, dF, dP);
#pragma unroll
          for (int aa = 0; aa < 4; ++aa)
#pragma unroll
            for (int d1 = 0; d1 < 3; ++d1) {
              const float v = g.s6 * (dP[3 * d1] * w[aa][0] + dP[3 * d1 + 1] * w[aa][1] +
                                      dP[3 * d1 + 2] * w[aa][2]);
              const bool row_fixed = (fx[aa] >> d1) & 1;
              K[(3 * aa + d1) * 12 + 3 * b + d2] = (col_fixed || row_fixed) ? 0.f : v;
            }
        }
      }
    }
    __syncthreads();
    const int nvalid = min(kCellThreads, e1 - c0);
#pragma unroll
    for (int k = 0; k < kCellOwned; ++k) {
      const int q = tid + k * kCellThreads;
      if (q < kCellEntries) {
        const int r = q / 24, col = q - 24 * r;
        const int c1 = r / 3, d1 = r - 3 * c1;
        const int c2 = col / 3, d2 = col - 3 * c2;
        for (int el = 0; el < nvalid; ++el) {
          const float* K = sK + el * 144;
          const float* W = sW + el * 32;
          float s = 0.f;
#pragma unroll
          for (int aa = 0; aa < 4; ++aa) {
            float t = 0.f;
#pragma unroll
            for (int b = 0; b < 4; ++b) t += K[(3 * aa + d1) * 12 + 3 * b + d2] * W[b * 8 + c2];
            s += W[aa * 8 + c1] * t;
          }
          acc[k] += (double)s;
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < kCellOwned; ++k) {
    const int q = tid + k * kCellThreads;
    if (q < kCellEntries) c.blocks[(size_t)blockIdx.x * kCellEntries + q] = acc[k];
  }
}

// Dense Ac (column-major, symmetric) from the cell blocks: entry (I, J) adds
// the blocks of the cells that hold both coarse nodes, in ascending cell
// order.  A DOF no free mesh DOF reaches gets a unit diagonal.
__global__ void coarse_dense_kernel(const __grid_constant__ CoarseDev c) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = c.n_dof;
  if (q >= (int64_t)n * n) return;
  const int I = (int)(q % n), J = (int)(q / n);
  const int nI = I / 3, dI = I - 3 * nI;
  const int nJ = J / 3, dJ = J - 3 * nJ;
  double acc = 0.0;
  for (int k = 0; k < 8; ++k) {
    const int ent = c.cn_cells[nI * 8 + k];
    if (ent < 0) break;
    const int cell = ent >> 3, cI = ent & 7;
    int cJ = -1;
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (c.cell_corner[cell * 8 + t] == nJ) cJ = t;
    if (cJ >= 0) {
      const size_t off = (size_t)(3 * cI + dI) * 24 + 3 * cJ + dJ;
      for (int sl = 0; sl < c.cell_slices; ++sl)
        acc += c.blocks[((size_t)cell * c.cell_slices + sl) * kCellEntries + off];
    }
  }
  if (I == J && !(acc > 0.0)) acc = 1.0;
  c.Ac[q] = acc;
}

// Symmetric FP32 copy of the inverse whose lower triangle the dense inverse wrote
// (column-major: element (lo, hi), lo >= hi, at hi * n + lo).
__global__ void coarse_sym_kernel(const __grid_constant__ CoarseDev c) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = c.n_dof;
  if (q >= (int64_t)n * n) return;
  const int row = (int)(q / n), col = (int)(q % n);
  const int lo = max(row, col), hi = min(row, col);
  c.Ainv[q] = c.Ac32 ? c.Ac32[(size_t)hi * n + lo] : (float)c.Ac[(size_t)hi * n + lo];
}

constexpr int kTile = 64;
constexpr int kTileElems = kTile * kTile;

// Block-triangle index t = I (I + 1) / 2 + J -> (I, J), J <= I.
__device__ __forceinline__ void tile_ij(int t, int& I, int& J) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  I = i;
  J = t - i * (i + 1) / 2;
}

// Packed BF16 copy: the lower block triangle of 64 x 64 tiles.
__global__ void coarse_pack16_kernel(const __grid_constant__ CoarseDev c) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nt = c.nb16 * (c.nb16 + 1) / 2;
  if (q >= (int64_t)nt * kTileElems) return;
  const int t = (int)(q / kTileElems), e = (int)(q % kTileElems);
  int I, J;
  tile_ij(t, I, J);
  const int row = I * kTile + e / kTile, col = J * kTile + e % kTile;
  const int n = c.n_dof;
  float v = 0.f;
  if (row < n && col < n) {
    const int lo = max(row, col), hi = min(row, col);
    v = c.Ac32 ? c.Ac32[(size_t)hi * n + lo] : (float)c.Ac[(size_t)hi * n + lo];
  }
  c.Ainv16[q] = __float2bfloat16_rn(v);
}

// ───────────────────────── per-iteration application ─────────────────────────

// Restriction, one warp per (cell, slice) item: slice s of a cell takes the
// cell's nodes in runs of 32, runs s, s + S, ... (S = r_slices, chosen so the
// items fill the GPU's warps); the item's 24 shares
//   cell_r[cell][s][3 corner + d] = sum over its nodes of w_corner r_d
// are completed by a reduce-scatter (lane k stores share k).  UPDATE fuses
// the CG update in front: x += alpha p, r -= alpha q on the item's nodes
// (every node belongs to exactly one cell); ||r||^2 and the convergence test
// run with r.z in tl_rz_kernel, so this kernel needs no grid reduction.
constexpr int kRestrictWarps = 8;
constexpr int kMaxRestrictSlices = 8;

__device__ __forceinline__ float warp_allsum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <bool UPDATE>
__global__ void __launch_bounds__(kRestrictWarps * 32) restrict_cells_kernel(
    const __grid_constant__ CoarseArgs a, float* r, float* x, const float* __restrict__ p,
    const float* __restrict__ q, const CGState* cg) {
  chain_enter();
  if (cg && cg->done) return;
  const CoarseDev& c = a.c;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = c.r_slices;
  const int n_items = c.n_cells * S;
  const float alpha = UPDATE ? (float)cg->alpha : 0.f;
  float4* r4 = reinterpret_cast<float4*>(r);
  float4* x4 = reinterpret_cast<float4*>(x);
  const float4* p4 = reinterpret_cast<const float4*>(p);
  const float4* q4 = reinterpret_cast<const float4*>(q);
  for (int item = blockIdx.x * kRestrictWarps + warp; item < n_items; item += gridDim.x * kRestrictWarps) {
    const int cell = item / S, sl = item - cell * S;
    const int3 ijk = c.cell_ijk[cell];
    const int n0 = c.cell_node_ptr[cell], n1 = c.cell_node_ptr[cell + 1];
    float acc[24];
#pragma unroll
    for (int k = 0; k < 24; ++k) acc[k] = 0.f;
    for (int i = n0 + 32 * sl + lane; i < n1; i += 32 * S) {
      const int node = __ldg(c.cell_nodes + i);
      const float4 X = __ldg(a.m.X32 + node);
      float4 rv = r4[node];
      if (UPDATE) {
        float4 xv = x4[node];
        const float4 pv = p4[node], qv = q4[node];
        xv.x += alpha * pv.x; xv.y += alpha * pv.y; xv.z += alpha * pv.z;
        rv.x -= alpha * qv.x; rv.y -= alpha * qv.y; rv.z -= alpha * qv.z;
        x4[node] = xv;
        r4[node] = rv;
      }
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
    // reduce-scatter of the 24 shares (padded to 32) over the warp: after
    // the step of width o each lane keeps the half whose bit o matches its
    // own; lane k ends with the full share k (31 shuffles, not 24 x 5)
    float u[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) u[k] = k < 24 ? acc[k] : 0.f;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int k = 0; k < o; ++k) {
        const float send = up ? u[k] : u[k + o];
        const float keep = up ? u[k + o] : u[k];
        u[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
    if (lane < 24) c.cell_r[(size_t)item * 24 + lane] = u[0];
  }
}

// r_c, one warp per coarse node: lane 4k + j adds the node's k-th cell share
// (cn_cells order) over slices j, j + 4, ...; a fixed butterfly combines the
// lanes (lanes 0..2 store the node's three DOFs).
__global__ void __launch_bounds__(256) coarse_rc_kernel(const __grid_constant__ CoarseDev c, const CGState* cg) {
  chain_enter();
  if (cg && cg->done) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cn = blockIdx.x * 8 + warp;
  if (cn >= c.n_cn) return;
  const int S = c.r_slices;
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
  v0 = warp_allsum(v0);
  v1 = warp_allsum(v1);
  v2 = warp_allsum(v2);
  if (lane < 3) c.rc[3 * cn + lane] = lane == 0 ? v0 : (lane == 1 ? v1 : v2);
}

// y_c = Ainv r_c with the FP32 inverse: r_c staged in shared memory, one warp
// per row.
constexpr int kCoarseMvThreads = 256;

__global__ void __launch_bounds__(kCoarseMvThreads) coarse_mv_kernel(
    const __grid_constant__ CoarseDev c, const CGState* cg) {
  chain_enter();
  if (cg && cg->done) return;
  extern __shared__ __align__(16) float s_rc[];
  const int n = c.n_dof;
  for (int I = threadIdx.x; I < n; I += kCoarseMvThreads) s_rc[I] = __ldcg(c.rc + I);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * (kCoarseMvThreads / 32) + warp;
  if (row >= n) return;
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
  if (lane == 0) c.yc[row] = s;
}

// y_c = Ainv r_c with the packed BF16 inverse, in two passes.
//
// Pass 1, one warp per stored tile (I, J), reading the tile once for both
// products it feeds: u = A_IJ r_J (row block I) and, off the diagonal,
// v = A_IJ^T r_I (row block J).  Lane l takes row quad position q = l / 8
// and the 8 columns 8 (l % 8) ...; one 16-byte load per lane covers 4 tile
// rows (512 contiguous bytes per warp), 16 loads the whole tile.  The row
// sums of u are completed across the 8 lanes of a row by a butterfly
// reduce-scatter (each lane ends with 2 rows); the column sums of v across
// the 4 lanes of a column group likewise (each lane ends with 2 columns).
// u goes to slot (I, J), v to slot (J, I): every slot (R, K) has exactly one
// writer.  The product streams the packed half of the matrix once.
//
// Pass 2: y_c[64 R + i] = sum over K of slot (R, K), K ascending: a CTA per
// (R, half of the rows), its 8 warps take K = w, w + 8, ... and the 8
// partials are added in warp order.  Both passes are deterministic.
constexpr int kTileWarps = 8;

__device__ __forceinline__ void bf16x8_to_f32(const uint4 w, float a[8]) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&w);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float2 f = __bfloat1622float2(h[k]);
    a[2 * k] = f.x;
    a[2 * k + 1] = f.y;
  }
}

__global__ void __launch_bounds__(kTileWarps * 32, 3) coarse_tile_mv_kernel(
    const __grid_constant__ CoarseDev c, const CGState* cg) {
  chain_enter();
  if (cg && cg->done) return;
  __shared__ float s_x[kTileWarps][2][kTile];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nb = c.nb16;
  const int n_tiles = nb * (nb + 1) / 2;
  const int q = lane >> 3, cg8 = lane & 7;
  for (int t = blockIdx.x * kTileWarps + warp; t < n_tiles; t += gridDim.x * kTileWarps) {
    int I, J;
    tile_ij(t, I, J);
    const bool offdiag = I != J;
    __syncwarp();
    reinterpret_cast<float2*>(s_x[warp][0])[lane] = __ldcg(reinterpret_cast<const float2*>(c.rc + J * kTile) + lane);
    reinterpret_cast<float2*>(s_x[warp][1])[lane] = __ldcg(reinterpret_cast<const float2*>(c.rc + I * kTile) + lane);
    __syncwarp();
    float xj[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) xj[k] = s_x[warp][0][8 * cg8 + k];
    const uint4* tile = reinterpret_cast<const uint4*>(c.Ainv16 + (size_t)t * kTileElems);
    float u[16], v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = 0.f;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int row = 4 * k + q;
      float a[8];
      // streamed once per product (evict-first), so the matvec's working set keeps the L2
      bf16x8_to_f32(__ldcs(tile + row * (kTile / 8) + cg8), a);
      float s = 0.f;
#pragma unroll
      for (int e = 0; e < 8; ++e) s += a[e] * xj[e];
      u[k] = s;
      const float xr = s_x[warp][1][row];
#pragma unroll
      for (int e = 0; e < 8; ++e) v[e] += a[e] * xr;
    }
    // u: reduce-scatter over the 8 lanes of a row quad position (lane bits
    // 2, 1, 0); lane keeps k = 2 cg8 + {0, 1}, i.e. rows 4 (2 cg8 + j) + q
#pragma unroll
    for (int o = 4, w = 8; o >= 1; o >>= 1, w >>= 1) {
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int k = 0; k < w; ++k) {
        const float send = up ? u[k] : u[k + w];
        const float keep = up ? u[k + w] : u[k];
        u[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
    float* slot_u = c.yslots + ((size_t)I * nb + J) * kTile;
    slot_u[4 * (2 * cg8) + q] = u[0];
    slot_u[4 * (2 * cg8 + 1) + q] = u[1];
    if (offdiag) {
      // v: reduce-scatter over the 4 lanes of a column group (lane bits 4,
      // 3); lane keeps columns 8 cg8 + 2 q + {0, 1}
#pragma unroll
      for (int o = 16, w = 4; o >= 8; o >>= 1, w >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int k = 0; k < w; ++k) {
          const float send = up ? v[k] : v[k + w];
          const float keep = up ? v[k + w] : v[k];
          v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
      }
      reinterpret_cast<float2*>(c.yslots + ((size_t)J * nb + I) * kTile + 8 * cg8 + 2 * q)[0] =
          make_float2(v[0], v[1]);
    }
  }
}

__global__ void __launch_bounds__(kTileWarps * 32) coarse_slot_sum_kernel(
    const __grid_constant__ CoarseDev c, const CGState* cg) {
  chain_enter();
  if (cg && cg->done) return;
  __shared__ float part[kTileWarps][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int R = blockIdx.x >> 1, half = blockIdx.x & 1;
  const int nb = c.nb16;
  const float* src = c.yslots + (size_t)R * nb * kTile + 32 * half + lane;
  float v = 0.f;
#pragma unroll 4
  for (int K = warp; K < nb; K += kTileWarps) v += __ldcg(src + (size_t)K * kTile);
  part[warp][lane] = v;
  __syncthreads();
  if (warp == 0) {
    float y = 0.f;
#pragma unroll
    for (int w = 0; w < kTileWarps; ++w) y += part[w][lane];
    const int row = R * kTile + 32 * half + lane;
    if (row < c.n_dof) c.yc[row] = y;
  }
}

// z = D^-1 r + P y_c (zero on fixed DOFs) and r.z.  INIT: p = z, rz set;
// otherwise also ||r||^2 of the r the update kernel just wrote: the last
// block runs the convergence test (iteration count, converged / out of
// iterations / breakdown), then beta = rz_new / rz_old (Fletcher-Reeves,
// exact for a fixed SPD preconditioner) and rz replaced.  The node's eight
// corner coarse nodes come from the per-node table (one dependent load less).
template <bool INIT>
__global__ void __launch_bounds__(256) tl_rz_kernel(const __grid_constant__ CoarseArgs a,
                                                    const float* __restrict__ r,
                                                    const float* __restrict__ dinv, float* z,
                                                    float* p, CGState* cg, Reduce red, int site) {
  chain_enter();
  if (cg->done) return;
  __shared__ double sred[8];
  __shared__ bool am_last;
  const CoarseDev& c = a.c;
  const int i = blockIdx.x * 256 + threadIdx.x;
  double rz = 0.0, rr = 0.0;
  if (i < a.m.n_nodes) {
    const float4 rv = reinterpret_cast<const float4*>(r)[i];
    const float4 dv = reinterpret_cast<const float4*>(dinv)[i];
    float t[3];
    node_lattice(c, i, t);
    const uint4 cw = __ldg(c.node_corners + i);
    const uint32_t cpk[4] = {cw.x, cw.y, cw.z, cw.w};
    float cz[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int cnode = (int)((cpk[q >> 1] >> (16 * (q & 1))) & 0xFFFFu);
      const float wq = tri_weight(t[0], t[1], t[2], q);
      cz[0] += wq * c.yc[3 * cnode];
      cz[1] += wq * c.yc[3 * cnode + 1];
      cz[2] += wq * c.yc[3 * cnode + 2];
    }
    const int fx = (int)a.m.fixed[i];
    float sm[3] = {dv.x * rv.x, dv.y * rv.y, dv.z * rv.z};
    if (a.boff) {
      // nodal block smoother: off-diagonals (01, 02, 12) of the block inverse
      const float4 ov = __ldg(reinterpret_cast<const float4*>(a.boff) + i);
      sm[0] += ov.x * rv.y + ov.y * rv.z;
      sm[1] += ov.x * rv.x + ov.z * rv.z;
      sm[2] += ov.y * rv.x + ov.z * rv.y;
    }
    float4 zv;
    zv.x = (fx & 1) ? 0.f : sm[0] + cz[0];
    zv.y = (fx & 2) ? 0.f : sm[1] + cz[1];
    zv.z = (fx & 4) ? 0.f : sm[2] + cz[2];
    zv.w = 0.f;
    reinterpret_cast<float4*>(z)[i] = zv;
    if (INIT) reinterpret_cast<float4*>(p)[i] = zv;
    rz = (double)rv.x * zv.x + (double)rv.y * zv.y + (double)rv.z * zv.z;
    rr = (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z;
  }
  chain_release();
  double v[2];
  v[0] = block_sum<256>(rz, sred);
  v[1] = INIT ? 0.0 : block_sum<256>(rr, sred);
  if (publish_partial(red, site, INIT ? 1 : 2, v, &am_last)) {
    const double trz = final_sum<256>(red, site, 0, sred);
    const double trr = INIT ? 0.0 : final_sum<256>(red, site, 1, sred);
    if (threadIdx.x == 0) {
      if (INIT) {
        cg->beta = 0.0;
      } else {
        cg->beta = trz / cg->rz;
        cg->rr = trr;
        cg->iter += 1;
      }
      cg->rz = trz;
      if (!INIT && !isfinite(trr)) {
        cg->done = 3;
        cg->status = 3;
      } else if (!INIT && trr <= cg->tol2) {
        cg->done = 1;
      } else if (!INIT && cg->iter >= cg->max_iter) {
        cg->done = 2;
      } else if (!isfinite(trz) || !(trz > 0.0)) {
        cg->done = 3;
        cg->status = 3;
      }
      red.counters[site] = 0u;
    }
  }
}

// p = z + beta p
__global__ void __launch_bounds__(256) tl_pupdate_kernel(float* p, const float* __restrict__ z,
                                                         int n_nodes, const CGState* cg) {
  chain_enter();
  if (cg->done) return;
  const float beta = (float)cg->beta;
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= n_nodes) return;
  float4 pv = reinterpret_cast<float4*>(p)[i];
  const float4 zv = reinterpret_cast<const float4*>(z)[i];
  pv.x = zv.x + beta * pv.x;
  pv.y = zv.y + beta * pv.y;
  pv.z = zv.z + beta * pv.z;
  reinterpret_cast<float4*>(p)[i] = pv;
}

// Flexible PCG step around the learned preconditioner.  z holds the
// network's output (which already contains D^-1 r); the kernel adds the coarse
// part P yc when COARSE, forms the Jacobi (+ coarse) alternative in zalt, and
// reduces r.z, z.q for both.  The last block keeps the network's direction
// unless it is not a descent direction relative to the alternative
// (r.z_net <= kSafe r.z_alt, or not finite); then the alternative is used for
// this iteration (cg->zsel = 1); after kLock such steps the network is
// switched off for the rest of the solve (cg->locked; its kernels then exit at
// entry) and the recursion restarts with beta = 0, so a network that does not
// help costs a few steps, not a slower solve.  INIT: p = chosen z.  Otherwise
// Polak-Ribiere beta = z.(r_new - r_old) / rz_old = -alpha z.q / rz_old,
// r_new - r_old = -alpha q.
constexpr double kSafe = 0.25;
constexpr int kLock = 3;

template <bool INIT, bool COARSE>
__global__ void __launch_bounds__(256) fpcg_dots_kernel(const __grid_constant__ CoarseArgs a,
                                                        const float* __restrict__ r,
                                                        const float* __restrict__ q,
                                                        const float* __restrict__ dinv, float* z, float* zalt,
                                                        float* p, CGState* cg, Reduce red, int site,
                                                        int site2) {
  if (cg->done) return;
  __shared__ double sred[8];
  __shared__ bool am_last;
  const int i = blockIdx.x * 256 + threadIdx.x;
  double rz = 0.0, zq = 0.0, rza = 0.0, zqa = 0.0;
  if (i < a.m.n_nodes) {
    const float4 rv = reinterpret_cast<const float4*>(r)[i];
    const float4 dv = reinterpret_cast<const float4*>(dinv)[i];
    float4 zv = reinterpret_cast<const float4*>(z)[i];
    float4 av = make_float4(dv.x * rv.x, dv.y * rv.y, dv.z * rv.z, 0.f);
    if (COARSE) {
      const CoarseDev& c = a.c;
      float t[3];
      const int cell = node_lattice(c, i, t);
      float cz[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int cnode = __ldg(c.cell_corner + cell * 8 + k);
        const float wk = tri_weight(t[0], t[1], t[2], k);
        cz[0] += wk * c.yc[3 * cnode];
        cz[1] += wk * c.yc[3 * cnode + 1];
        cz[2] += wk * c.yc[3 * cnode + 2];
      }
      const int fx = (int)a.m.fixed[i];
      zv.x = (fx & 1) ? 0.f : zv.x + cz[0];
      zv.y = (fx & 2) ? 0.f : zv.y + cz[1];
      zv.z = (fx & 4) ? 0.f : zv.z + cz[2];
      av.x = (fx & 1) ? 0.f : av.x + cz[0];
      av.y = (fx & 2) ? 0.f : av.y + cz[1];
      av.z = (fx & 4) ? 0.f : av.z + cz[2];
    }
    zv.w = 0.f;
    reinterpret_cast<float4*>(z)[i] = zv;
    reinterpret_cast<float4*>(zalt)[i] = av;
    rz = (double)rv.x * zv.x + (double)rv.y * zv.y + (double)rv.z * zv.z;
    rza = (double)rv.x * av.x + (double)rv.y * av.y + (double)rv.z * av.z;
    if (!INIT) {
      const float4 qv = reinterpret_cast<const float4*>(q)[i];
      zq = (double)zv.x * qv.x + (double)zv.y * qv.y + (double)zv.z * qv.z;
      zqa = (double)av.x * qv.x + (double)av.y * qv.y + (double)av.z * qv.z;
    }
  }
  double v[2], v2[2];
  v[0] = block_sum<256>(rz, sred);
  v[1] = block_sum<256>(zq, sred);
  v2[0] = block_sum<256>(rza, sred);
  v2[1] = block_sum<256>(zqa, sred);
  if (threadIdx.x == 0) {
    red.partials[(size_t)(site2 * 2) * red.max_blocks + blockIdx.x] = v2[0];
    red.partials[(size_t)(site2 * 2 + 1) * red.max_blocks + blockIdx.x] = v2[1];
  }
  if (publish_partial(red, site, 2, v, &am_last)) {
    const double trz = final_sum<256>(red, site, 0, sred);
    const double tzq = final_sum<256>(red, site, 1, sred);
    const double arz = final_sum<256>(red, site2, 0, sred);
    const double azq = final_sum<256>(red, site2, 1, sred);
    if (threadIdx.x == 0) {
      const bool was_locked = cg->locked != 0;
      const bool net_ok = !was_locked && isfinite(trz) && isfinite(tzq) && trz > kSafe * arz;
      const double rzc = net_ok ? trz : arz;
      const double zqc = net_ok ? tzq : azq;
      cg->zsel = net_ok ? 0 : 1;
      bool restart = false;
      if (!net_ok) {
        cg->n_alt += 1;
        if (!was_locked && cg->n_alt >= kLock) {
          // the network is switched off: hand the rest of the solve, from the
          // current iterate, to the plain preconditioned CG (status 4)
          cg->locked = 1;
          cg->done = 4;
          cg->status = 4;
          restart = true;
        }
      }
      cg->beta = (INIT || restart) ? 0.0 : -cg->alpha * zqc / cg->rz;
      cg->rz = rzc;
      if (!isfinite(rzc) || !(rzc > 0.0) || !isfinite(cg->beta)) {
        cg->done = 3;
        cg->status = 3;
      }
      red.counters[site] = 0u;
    }
  }
}

// p = z_sel + beta p (INIT: p = z_sel), z_sel the direction fpcg_dots kept
__global__ void __launch_bounds__(256) fpcg_pupdate_kernel(float* p, const float* __restrict__ z,
                                                           const float* __restrict__ zalt, int n_nodes,
                                                           const CGState* cg, int init) {
  if (cg->done) return;
  const float beta = init ? 0.f : (float)cg->beta;
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= n_nodes) return;
  const float4 zv = reinterpret_cast<const float4*>(cg->zsel ? zalt : z)[i];
  float4 pv = init ? make_float4(0.f, 0.f, 0.f, 0.f) : reinterpret_cast<float4*>(p)[i];
  pv.x = zv.x + beta * pv.x;
  pv.y = zv.y + beta * pv.y;
  pv.z = zv.z + beta * pv.z;
  pv.w = 0.f;
  reinterpret_cast<float4*>(p)[i] = pv;
}

// z += P yc on free DOFs (the coarse part of a composite preconditioner)
__global__ void __launch_bounds__(256) coarse_add_kernel(const __grid_constant__ CoarseArgs a, float* z) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= a.m.n_nodes) return;
  const CoarseDev& c = a.c;
  float t[3];
  const int cell = node_lattice(c, i, t);
  float cz[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int cnode = __ldg(c.cell_corner + cell * 8 + k);
    const float wk = tri_weight(t[0], t[1], t[2], k);
    cz[0] += wk * c.yc[3 * cnode];
    cz[1] += wk * c.yc[3 * cnode + 1];
    cz[2] += wk * c.yc[3 * cnode + 2];
  }
  const int fx = (int)a.m.fixed[i];
  float4 zv = reinterpret_cast<float4*>(z)[i];
  zv.x = (fx & 1) ? 0.f : zv.x + cz[0];
  zv.y = (fx & 2) ? 0.f : zv.y + cz[1];
  zv.z = (fx & 4) ? 0.f : zv.z + cz[2];
  reinterpret_cast<float4*>(z)[i] = zv;
}

// Energy loss of one training pair (r, e) with A e = r:
//   L = (z.Az - 2 z.r + e.r) / e.r = ||z - e||_A^2 / ||e||_A^2
// out[0] += L; out[1] = 2 / e.r (scale of dL/dz = 2 (Az - r) / e.r)
__global__ void __launch_bounds__(256) train_loss_kernel(const float* __restrict__ z, const float* __restrict__ q,
                                                         const float* __restrict__ r, const float* __restrict__ e,
                                                         int n, double* out, Reduce red, int site) {
  __shared__ double sred[8];
  __shared__ bool am_last;
  const int i = blockIdx.x * 256 + threadIdx.x;
  double zq = 0.0, zr = 0.0, er = 0.0;
  if (i < n) {
    const float4 zv = reinterpret_cast<const float4*>(z)[i];
    const float4 qv = reinterpret_cast<const float4*>(q)[i];
    const float4 rv = reinterpret_cast<const float4*>(r)[i];
    const float4 ev = reinterpret_cast<const float4*>(e)[i];
    zq = (double)zv.x * qv.x + (double)zv.y * qv.y + (double)zv.z * qv.z;
    zr = (double)zv.x * rv.x + (double)zv.y * rv.y + (double)zv.z * rv.z;
    er = (double)ev.x * rv.x + (double)ev.y * rv.y + (double)ev.z * rv.z;
  }
  double v[2];
  v[0] = block_sum<256>(zq - 2.0 * zr, sred);
  v[1] = block_sum<256>(er, sred);
  if (publish_partial(red, site, 2, v, &am_last)) {
    const double a = final_sum<256>(red, site, 0, sred);
    const double b = final_sum<256>(red, site, 1, sred);
    if (threadIdx.x == 0) {
      const bool good = b > 0.0 && isfinite(a) && isfinite(b);
      out[0] += good ? (a + b) / b : 0.0;
      out[1] = good ? 2.0 / b : 0.0;
      red.counters[site] = 0u;
    }
  }
}

// gz = scale (q - r) on free DOFs
__global__ void __launch_bounds__(256) train_grad_z_kernel(const float* __restrict__ q, const float* __restrict__ r,
                                                           const uint8_t* __restrict__ fixed, const double* scale,
                                                           float* gz, int n) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  const float sc = (float)scale[1];
  const float4 qv = reinterpret_cast<const float4*>(q)[i];
  const float4 rv = reinterpret_cast<const float4*>(r)[i];
  const int fx = (int)fixed[i];
  float4 g;
  g.x = (fx & 1) ? 0.f : sc * (qv.x - rv.x);
  g.y = (fx & 2) ? 0.f : sc * (qv.y - rv.y);
  g.z = (fx & 4) ? 0.f : sc * (qv.z - rv.z);
  g.w = 0.f;
  reinterpret_cast<float4*>(gz)[i] = g;
}

// z = D^-1 r (the network's output with a zero decoder)
__global__ void jacobi_apply_kernel(const float* __restrict__ r, const float* __restrict__ dinv, float* z, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 rv = reinterpret_cast<const float4*>(r)[i];
  const float4 dv = reinterpret_cast<const float4*>(dinv)[i];
  reinterpret_cast<float4*>(z)[i] = make_float4(dv.x * rv.x, dv.y * rv.y, dv.z * rv.z, 0.f);
}

// ───────────────────────── launchers ─────────────────────────

static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

size_t coarse_cell_smem() { return sizeof(float) * kCellThreads * (144 + 32); }
int coarse_cell_slices(int npe) { return npe == 8 ? kCellSlices * 4 : kCellSlices; }
int coarse_restrict_slices(int n_cells) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int warps = std::max(sms, 1) * 32;
  return std::max(1, std::min(kMaxRestrictSlices, (warps + std::max(n_cells, 1) - 1) / std::max(n_cells, 1)));
}

void prepare_coarse_kernels(int model, int n_dof) {
  (void)n_dof;
  switch (model) {
    case M_LE: raise_smem_limit_k(coarse_cell_kernel<M_LE>); break;
    case M_NH: raise_smem_limit_k(coarse_cell_kernel<M_NH>); break;
    case M_MR: raise_smem_limit_k(coarse_cell_kernel<M_MR>); break;
    case M_J2: raise_smem_limit_k(coarse_cell_kernel<M_J2>); break;
    case M_TI: raise_smem_limit_k(coarse_cell_kernel<M_TI>); break;
    case M_FMR: raise_smem_limit_k(coarse_cell_kernel<M_FMR>); break;
    default: raise_smem_limit_k(coarse_cell_kernel<-1>); break;
  }
  raise_smem_limit_k(coarse_mv_kernel);
}

void launch_coarse_assemble(const CoarseArgs& a, int model, cudaStream_t s) {
  const size_t smem = coarse_cell_smem();
  const int g = a.c.n_cells * kCellSlices;
  if (a.m.npe == 8) launch_coarse_cells_hex(a, model, s);
  else switch (model) {
    case M_LE: coarse_cell_kernel<M_LE><<<g, kCellThreads, smem, s>>>(a); break;
    case M_NH: coarse_cell_kernel<M_NH><<<g, kCellThreads, smem, s>>>(a); break;
    case M_MR: coarse_cell_kernel<M_MR><<<g, kCellThreads, smem, s>>>(a); break;
    case M_J2: coarse_cell_kernel<M_J2><<<g, kCellThreads, smem, s>>>(a); break;
    case M_TI: coarse_cell_kernel<M_TI><<<g, kCellThreads, smem, s>>>(a); break;
    case M_FMR: coarse_cell_kernel<M_FMR><<<g, kCellThreads, smem, s>>>(a); break;
    default: coarse_cell_kernel<-1><<<g, kCellThreads, smem, s>>>(a); break;
  }
  const int64_t nn = (int64_t)a.c.n_dof * a.c.n_dof;
  coarse_dense_kernel<<<nblk(nn, 256), 256, 0, s>>>(a.c);
}

void launch_coarse_symmetrize(const CoarseDev& c, cudaStream_t s) {
  if (c.Ainv16) {
    const int64_t ne = (int64_t)c.nb16 * (c.nb16 + 1) / 2 * kTileElems;
    coarse_pack16_kernel<<<nblk(ne, 256), 256, 0, s>>>(c);
    return;
  }
  const int64_t nn = (int64_t)c.n_dof * c.n_dof;
  coarse_sym_kernel<<<nblk(nn, 256), 256, 0, s>>>(c);
}

__global__ void coarse_node_lat_kernel(const __grid_constant__ MeshDev m, const __grid_constant__ CoarseDev c,
                                       float4* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.n_nodes) return;
  const float4 X = __ldg(m.X32 + i);
  const int cell = c.node_cell[i];
  float t[3];
  cell_local(c, c.cell_ijk[cell], X.x, X.y, X.z, t);
  out[i] = make_float4(t[0], t[1], t[2], __int_as_float(cell));
}

void launch_coarse_node_lat(const MeshDev& m, const CoarseDev& c, float4* out, cudaStream_t s) {
  coarse_node_lat_kernel<<<nblk(m.n_nodes, 256), 256, 0, s>>>(m, c, out);
}

// node_corners[i] = the eight corner coarse nodes of node i's cell, 16 bits each
__global__ void coarse_node_corners_kernel(const __grid_constant__ MeshDev m, const __grid_constant__ CoarseDev c,
                                           uint4* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.n_nodes) return;
  const int cell = c.node_cell[i];
  uint32_t w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    w[k] = ((uint32_t)c.cell_corner[cell * 8 + 2 * k] & 0xFFFFu) |
           (((uint32_t)c.cell_corner[cell * 8 + 2 * k + 1] & 0xFFFFu) << 16);
  out[i] = make_uint4(w[0], w[1], w[2], w[3]);
}

void launch_coarse_node_corners(const MeshDev& m, const CoarseDev& c, uint4* out, cudaStream_t s) {
  coarse_node_corners_kernel<<<nblk(m.n_nodes, 256), 256, 0, s>>>(m, c, out);
}

int coarse_product_kernels(const CoarseDev& c) { return c.Ainv16 ? 2 : 1; }

// Resident CTAs of the tile product on this device (one wave, tiles looped).
int tile_mv_grid() {
  static int grid = 0;
  if (grid == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, coarse_tile_mv_kernel, kTileWarps * 32, 0);
    grid = std::max(1, sms * std::max(per_sm, 1));
  }
  return grid;
}

void launch_coarse_apply(const CoarseArgs& a, const float* r, const CGState* cg, cudaStream_t s) {
  restrict_cells_kernel<false><<<nblk((int64_t)a.c.n_cells * a.c.r_slices, kRestrictWarps), kRestrictWarps * 32, 0,
                                  s>>>(a, const_cast<float*>(r), nullptr, nullptr, nullptr, cg);
  launch_coarse_solve(a, cg, s);
}

void launch_update_restrict(const CoarseArgs& a, float* x, float* r, const float* p, const float* q, CGState* cg,
                            cudaStream_t s) {
  launch_chain(restrict_cells_kernel<true>, nblk((int64_t)a.c.n_cells * a.c.r_slices, kRestrictWarps),
               kRestrictWarps * 32, 0, s, a, r, x, p, q, static_cast<const CGState*>(cg));
}

void launch_coarse_solve(const CoarseArgs& a, const CGState* cg, cudaStream_t s) {
  launch_chain(coarse_rc_kernel, nblk(a.c.n_cn, 8), 256, 0, s, a.c, cg);
  if (a.c.Ainv16) {
    const int nt = a.c.nb16 * (a.c.nb16 + 1) / 2;
    launch_chain(coarse_tile_mv_kernel, std::min(nblk(nt, kTileWarps), tile_mv_grid()), kTileWarps * 32, 0, s, a.c,
                 cg);
    launch_chain(coarse_slot_sum_kernel, 2 * a.c.nb16, kTileWarps * 32, 0, s, a.c, cg);
    return;
  }
  const int rows_per_cta = kCoarseMvThreads / 32;
  launch_chain(coarse_mv_kernel, nblk(a.c.n_dof, rows_per_cta), kCoarseMvThreads, sizeof(float) * (size_t)a.c.n_dof,
               s, a.c, cg);
}

void launch_tl_rz(const CoarseArgs& a, bool init, const float* r, const float* dinv, float* z, float* p,
                  CGState* cg, Reduce red, int site, cudaStream_t s) {
  const int g = nblk(a.m.n_nodes, 256);
  if (init)
    tl_rz_kernel<true><<<g, 256, 0, s>>>(a, r, dinv, z, p, cg, red, site);
  else
    launch_chain(tl_rz_kernel<false>, g, 256, 0, s, a, r, dinv, z, p, cg, red, site);
}

void launch_fpcg_dots(const CoarseArgs& a, bool init, bool coarse, const float* r, const float* q,
                      const float* dinv, float* z, float* zalt, float* p, CGState* cg, Reduce red, int site,
                      int site2, cudaStream_t s) {
  const int g = nblk(a.m.n_nodes, 256);
  if (init) {
    if (coarse)
      fpcg_dots_kernel<true, true><<<g, 256, 0, s>>>(a, r, q, dinv, z, zalt, p, cg, red, site, site2);
    else
      fpcg_dots_kernel<true, false><<<g, 256, 0, s>>>(a, r, q, dinv, z, zalt, p, cg, red, site, site2);
  } else {
    if (coarse)
      fpcg_dots_kernel<false, true><<<g, 256, 0, s>>>(a, r, q, dinv, z, zalt, p, cg, red, site, site2);
    else
      fpcg_dots_kernel<false, false><<<g, 256, 0, s>>>(a, r, q, dinv, z, zalt, p, cg, red, site, site2);
  }
}

void launch_fpcg_pupdate(float* p, const float* z, const float* zalt, int n_nodes, const CGState* cg, bool init,
                         cudaStream_t s) {
  fpcg_pupdate_kernel<<<nblk(n_nodes, 256), 256, 0, s>>>(p, z, zalt, n_nodes, cg, init ? 1 : 0);
}

void launch_tl_pupdate(float* p, const float* z, int n_nodes, const CGState* cg, cudaStream_t s) {
  launch_chain(tl_pupdate_kernel, nblk(n_nodes, 256), 256, 0, s, p, z, n_nodes, cg);
}

void launch_coarse_add(const CoarseArgs& a, float* z, cudaStream_t s) {
  coarse_add_kernel<<<nblk(a.m.n_nodes, 256), 256, 0, s>>>(a, z);
}

void launch_train_loss(const float* z, const float* q, const float* r, const float* e, int n, double* out,
                       Reduce red, int site, cudaStream_t s) {
  train_loss_kernel<<<nblk(n, 256), 256, 0, s>>>(z, q, r, e, n, out, red, site);
}

void launch_train_grad_z(const float* q, const float* r, const uint8_t* fixed, const double* scale, float* gz,
                         int n, cudaStream_t s) {
  train_grad_z_kernel<<<nblk(n, 256), 256, 0, s>>>(q, r, fixed, scale, gz, n);
}

void launch_jacobi_apply(const float* r, const float* dinv, float* z, int n, cudaStream_t s) {
  jacobi_apply_kernel<<<nblk(n, 256), 256, 0, s>>>(r, dinv, z, n);
}

}  // namespace femb200
