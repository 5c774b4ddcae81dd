// Learned preconditioner: a message-passing network over mesh nodes applied
// as z = M(r) inside flexible PCG.  Per node i (N(i): nodes sharing an
// element with i; d = sqrt(D^-1), D = diag K_T on free DOFs):
//
//   s   = RMS_i |d_i r_i|                      (FP64 reduction)
//   f_i = [d_i r_i / s, fixed bits, c_i, 0...]  (16, BF16)
//   h_i = relu(W_e f_i + b_e)                  (64, BF16 storage)
//   4x: m_i = mean_{j in N(i)} h_j;  h_i += relu(W_l [h_i, m_i] + b_l)
//   z_i = D^-1 r_i + s d_i (W_d h_i + b_d)
//
// The dense layers run on the 5th-generation tensor cores: one CTA per tile
// of 128 nodes stages the BF16 operand tile in shared memory, one thread
// issues tcgen05.mma into a TMEM accumulator, and the epilogue reads it back
// with tcgen05.ld.  The aggregation over N(i) is a fixed-order gather.
// No reference counterpart (the reference factorises the assembled tangent,
// backend/fea/fem/solver/static_solver.py:399-462).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "fem_internal.h"
#include "fem_reduce.cuh"
#include "fem_umma.cuh"

namespace femb200 {

namespace {

constexpr int kTile = 128;
constexpr int kHid = kMpnnHidden;   // 64
constexpr int kIn = kMpnnIn;        // 16
constexpr int kPolls = 1 << 22;     // mbarrier polls before a layer reports a stalled MMA

__device__ __forceinline__ void unpack8(const uint4 v, float f[8]) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float2 t = __bfloat1622float2(h[i]);
    f[2 * i] = t.x;
    f[2 * i + 1] = t.y;
  }
}

__device__ __forceinline__ uint4 pack8(const float f[8]) {
  uint4 v;
  __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
  for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
  return v;
}

}  // namespace

// ───────────────────────── weights ─────────────────────────

// FP32 master parameters -> BF16 tensor-core operand tiles (canonical K-major):
// W_e as [64 out x 16 in], W_l as [64 out x 128 in], W_l^T as [128 in x 64 out].
__global__ void mpnn_pack_kernel(const float* __restrict__ w, __nv_bfloat16* We_p, __nv_bfloat16* Wl_p,
                                 __nv_bfloat16* WlT_p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < kHid * kIn) {
    const int n = t / kIn, k = t - n * kIn;
    We_p[umma::kmajor_off(n, k, kIn) / 2] = __float2bfloat16_rn(w[kMpnnOffWe + t]);
  }
  const int per = kHid * 2 * kHid;
  if (t < kMpnnLayers * per) {
    const int l = t / per, q = t - l * per;
    const int n = q / (2 * kHid), k = q - n * 2 * kHid;
    const __nv_bfloat16 v = __float2bfloat16_rn(w[kMpnnOffW(l) + q]);
    Wl_p[(size_t)l * per + umma::kmajor_off(n, k, 2 * kHid) / 2] = v;
    WlT_p[(size_t)l * per + umma::kmajor_off(k, n, kHid) / 2] = v;
  }
}

// ───────────────────────── forward ─────────────────────────

// s = sqrt(sum |d r|^2 / Nn) into m.scal[0]
__global__ void __launch_bounds__(256) mpnn_scale_kernel(const __grid_constant__ MpnnDev m,
                                                         const float* __restrict__ r,
                                                         const float* __restrict__ dinv, const CGState* cg,
                                                         Reduce red, int site) {
  if (cg && (cg->done || cg->locked)) return;
  __shared__ double sred[8];
  __shared__ bool am_last;
  const int i = blockIdx.x * 256 + threadIdx.x;
  double acc = 0.0;
  if (i < m.n_nodes) {
    const float4 rv = reinterpret_cast<const float4*>(r)[i];
    const float4 dv = reinterpret_cast<const float4*>(dinv)[i];
    acc = (double)dv.x * rv.x * rv.x + (double)dv.y * rv.y * rv.y + (double)dv.z * rv.z * rv.z;
  }
  double v = block_sum<256>(acc, sred);
  if (publish_partial(red, site, 1, &v, &am_last)) {
    const double tot = final_sum<256>(red, site, 0, sred);
    if (threadIdx.x == 0) {
      m.scal[0] = sqrt(tot / (double)m.n_nodes);
      red.counters[site] = 0u;
    }
  }
}

// h0 = relu(W_e f + b_e), one tile of 128 nodes per CTA
__global__ void __launch_bounds__(kTile) mpnn_encode_kernel(const __grid_constant__ MpnnDev m,
                                                            const float* __restrict__ r,
                                                            const float* __restrict__ dinv, const CGState* cg) {
  if (cg && (cg->done || cg->locked)) return;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  unsigned char* sA = smem;              // 128 x 16 BF16 = 4 KB
  unsigned char* sB = smem + 4096;       // 64 x 16 BF16 = 2 KB
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int node = blockIdx.x * kTile + tid;
  if (warp == 0) umma::tmem_alloc(&tmem_base, 64);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  {
    float f[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = 0.f;
    if (node < m.n_nodes) {
      const double s = m.scal[0];
      const float inv_s = s > 0.0 ? (float)(1.0 / s) : 0.f;
      const float4 rv = reinterpret_cast<const float4*>(r)[node];
      const float4 dv = reinterpret_cast<const float4*>(dinv)[node];
      f[0] = sqrtf(dv.x) * rv.x * inv_s;
      f[1] = sqrtf(dv.y) * rv.y * inv_s;
      f[2] = sqrtf(dv.z) * rv.z * inv_s;
      const int fx = (int)m.fixed[node];
      f[3] = (float)(fx & 1);
      f[4] = (float)((fx >> 1) & 1);
      f[5] = (float)((fx >> 2) & 1);
      f[6] = m.cfeat[node];
    }
    *reinterpret_cast<uint4*>(sA + umma::kmajor_off(tid, 0, kIn)) = pack8(f);
    *reinterpret_cast<uint4*>(sA + umma::kmajor_off(tid, 8, kIn)) = pack8(f + 8);
    reinterpret_cast<uint4*>(sB)[tid] = reinterpret_cast<const uint4*>(m.We_p)[tid];
  }
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (tid == 0) {
    umma::mma_bf16(tbase, umma::smem_desc(umma::smem_u32(sA), kIn), umma::smem_desc(umma::smem_u32(sB), kIn),
                   umma::idesc_bf16(kTile, kHid), 0u);
    umma::commit(&mbar);
  }
  __syncwarp();
  const bool ok = umma::mbar_wait(&mbar, 0, kPolls);
  umma::fence_after_sync();
  if (ok) {
    const float* b = m.w + kMpnnOffBe;
#pragma unroll
    for (int c0 = 0; c0 < kHid; c0 += 16) {
      float v[16];
      umma::tmem_ld16(umma::taddr(tbase, 32 * warp, c0), v);
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j] + __ldg(b + c0 + j), 0.f);
      if (node < m.n_nodes) {
        uint4* dst = reinterpret_cast<uint4*>(m.H[0] + (size_t)node * kHid + c0);
        dst[0] = pack8(v);
        dst[1] = pack8(v + 8);
      }
    }
  } else if (lane == 0) {
    atomicExch(m.err, 1);
  }
  umma::drain_mma(&mbar, 0, ok, kPolls);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, 64);
}

// One message-passing layer over a tile of 128 nodes, 256 threads: thread t
// gathers channel half t >> 7 of node t & 127.  LAST: the decoder and the
// preconditioned vector z are fused into the epilogue.
template <bool LAST>
__global__ void __launch_bounds__(2 * kTile) mpnn_layer_kernel(const __grid_constant__ MpnnDev m, int layer,
                                                               const float* __restrict__ r,
                                                               const float* __restrict__ dinv, float* z,
                                                               const CGState* cg) {
  if (cg && (cg->done || cg->locked)) return;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ float sO[kTile][4];
  unsigned char* sA = smem;                          // 128 x 128 BF16 = 32 KB
  unsigned char* sB = smem + kTile * 2 * kHid * 2;   // 64 x 128 BF16 = 16 KB
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nl = tid & (kTile - 1), half = tid >> 7;
  const int node = blockIdx.x * kTile + nl;
  const __nv_bfloat16* Hin = m.H[layer];
  if (warp == 0) umma::tmem_alloc(&tmem_base, 64);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  {
    const uint4* wsrc = reinterpret_cast<const uint4*>(m.Wl_p + (size_t)layer * kHid * 2 * kHid);
#pragma unroll
    for (int q = 0; q < 4; ++q) reinterpret_cast<uint4*>(sB)[tid + q * 2 * kTile] = __ldg(wsrc + tid + q * 2 * kTile);
  }
  {
    float acc[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) acc[k] = 0.f;
    uint4 own[4] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
    float dinv_deg = 0.f;
    if (node < m.n_nodes) {
      const uint4* hs = reinterpret_cast<const uint4*>(Hin + (size_t)node * kHid + 32 * half);
#pragma unroll
      for (int c = 0; c < 4; ++c) own[c] = hs[c];
      const int j0 = __ldg(m.adj_ptr + node), j1 = __ldg(m.adj_ptr + node + 1);
      dinv_deg = __ldg(m.deg_inv + node);
      for (int j = j0; j < j1; ++j) {
        const int nb = __ldg(m.adj_idx + j);
        const uint4* hn = reinterpret_cast<const uint4*>(Hin + (size_t)nb * kHid + 32 * half);
        uint4 v[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) v[c] = hn[c];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          float f[8];
          unpack8(v[c], f);
#pragma unroll
          for (int q = 0; q < 8; ++q) acc[8 * c + q] += f[q];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float f[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) f[q] = acc[8 * c + q] * dinv_deg;
      *reinterpret_cast<uint4*>(sA + umma::kmajor_off(nl, 32 * half + 8 * c, 2 * kHid)) = own[c];
      *reinterpret_cast<uint4*>(sA + umma::kmajor_off(nl, kHid + 32 * half + 8 * c, 2 * kHid)) = pack8(f);
    }
  }
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (tid == 0) {
    const uint32_t a0 = umma::smem_u32(sA), b0 = umma::smem_u32(sB);
    const uint32_t idesc = umma::idesc_bf16(kTile, kHid);
#pragma unroll
    for (int s = 0; s < 2 * kHid / 16; ++s)
      umma::mma_bf16(tbase, umma::smem_desc(a0 + 256 * s, 2 * kHid), umma::smem_desc(b0 + 256 * s, 2 * kHid), idesc,
                     s > 0 ? 1u : 0u);
    umma::commit(&mbar);
  }
  __syncwarp();
  const bool ok = umma::mbar_wait(&mbar, 0, kPolls);
  umma::fence_after_sync();
  // epilogue: warp w reads TMEM lanes 32 (w % 4).., columns of half w / 4
  const int row = 32 * (warp & 3) + lane;
  const int ehalf = warp >> 2;
  const int enode = blockIdx.x * kTile + row;
  float o[3] = {0.f, 0.f, 0.f};
  if (ok) {
    const float* b = m.w + kMpnnOffB(layer);
    uint32_t bits = 0;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
      const int c0 = 32 * ehalf + 16 * cc;
      float v[16];
      umma::tmem_ld16(umma::taddr(tbase, 32 * (warp & 3), c0), v);
      float hin[16];
      unpack8(*reinterpret_cast<const uint4*>(sA + umma::kmajor_off(row, c0, 2 * kHid)), hin);
      unpack8(*reinterpret_cast<const uint4*>(sA + umma::kmajor_off(row, c0 + 8, 2 * kHid)), hin + 8);
      float hout[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float pre = v[j] + __ldg(b + c0 + j);
        if (pre > 0.f) bits |= 1u << (16 * cc + j);
        hout[j] = hin[j] + fmaxf(pre, 0.f);
      }
      const uint4 p0 = pack8(hout), p1 = pack8(hout + 8);
      if (enode < m.n_nodes) {
        uint4* dst = reinterpret_cast<uint4*>(m.H[layer + 1] + (size_t)enode * kHid + c0);
        dst[0] = p0;
        dst[1] = p1;
      }
      if (LAST) {
        float hr[16];
        unpack8(p0, hr);
        unpack8(p1, hr + 8);
        const float* Wd = m.w + kMpnnOffWd;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          o[0] += __ldg(Wd + c0 + j) * hr[j];
          o[1] += __ldg(Wd + kHid + c0 + j) * hr[j];
          o[2] += __ldg(Wd + 2 * kHid + c0 + j) * hr[j];
        }
      }
    }
    if (enode < m.n_nodes) reinterpret_cast<uint32_t*>(m.mask[layer])[2 * (size_t)enode + ehalf] = bits;
  } else if (lane == 0) {
    atomicExch(m.err, 1);
  }
  if (LAST) {
    if (ehalf == 1) {
      sO[row][0] = o[0];
      sO[row][1] = o[1];
      sO[row][2] = o[2];
    }
  }
  umma::drain_mma(&mbar, 0, ok, kPolls);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, 64);
  if (LAST && ehalf == 0 && enode < m.n_nodes) {
    const float* bd = m.w + kMpnnOffBd;
    const float s = (float)m.scal[0];
    const float4 rv = reinterpret_cast<const float4*>(r)[enode];
    const float4 dv = reinterpret_cast<const float4*>(dinv)[enode];
    float4 zv;
    zv.x = dv.x * rv.x + s * sqrtf(dv.x) * (o[0] + sO[row][0] + bd[0]);
    zv.y = dv.y * rv.y + s * sqrtf(dv.y) * (o[1] + sO[row][1] + bd[1]);
    zv.z = dv.z * rv.z + s * sqrtf(dv.z) * (o[2] + sO[row][2] + bd[2]);
    zv.w = 0.f;
    reinterpret_cast<float4*>(z)[enode] = zv;
  }
}

// ───────────────────────── backward (training) ─────────────────────────
// Gradient of <gz, z> with respect to the parameters.  Every kernel writes
// its tile's share of the gradient into gpart[tile][param]; a final kernel
// sums the tiles in index order, so gradients are bitwise reproducible.

// decoder: go = s d gz; GH = W_d^T go; dW_d, db_d from this tile's nodes
__global__ void __launch_bounds__(kTile) mpnn_dec_bwd_kernel(const __grid_constant__ MpnnTrain t,
                                                             const float* __restrict__ dinv,
                                                             const float* __restrict__ gz) {
  const MpnnDev& m = t.m;
  __shared__ float sGo[kTile][3];
  __shared__ float sH[kTile][kHid + 1];
  const int tid = threadIdx.x;
  const int node = blockIdx.x * kTile + tid;
  const float s = (float)m.scal[0];
  float go[3] = {0.f, 0.f, 0.f};
  float h[kHid];
#pragma unroll
  for (int c = 0; c < kHid; ++c) h[c] = 0.f;
  if (node < m.n_nodes) {
    const float4 g = reinterpret_cast<const float4*>(gz)[node];
    const float4 dv = reinterpret_cast<const float4*>(dinv)[node];
    go[0] = s * sqrtf(dv.x) * g.x;
    go[1] = s * sqrtf(dv.y) * g.y;
    go[2] = s * sqrtf(dv.z) * g.z;
    const uint4* hp = reinterpret_cast<const uint4*>(m.H[kMpnnLayers] + (size_t)node * kHid);
#pragma unroll
    for (int c = 0; c < kHid / 8; ++c) unpack8(hp[c], h + 8 * c);
    const float* Wd = m.w + kMpnnOffWd;
    float* gh = t.GH + (size_t)node * kHid;
#pragma unroll 8
    for (int c = 0; c < kHid; ++c)
      gh[c] = __ldg(Wd + c) * go[0] + __ldg(Wd + kHid + c) * go[1] + __ldg(Wd + 2 * kHid + c) * go[2];
  }
  sGo[tid][0] = go[0];
  sGo[tid][1] = go[1];
  sGo[tid][2] = go[2];
#pragma unroll
  for (int c = 0; c < kHid; ++c) sH[tid][c] = h[c];
  __syncthreads();
  float* part = t.gpart + (size_t)blockIdx.x * kMpnnParams;
  for (int q = tid; q < 3 * kHid + 3; q += kTile) {
    float acc = 0.f;
    if (q < 3 * kHid) {
      const int k = q / kHid, c = q - k * kHid;
      for (int i = 0; i < kTile; ++i) acc += sGo[i][k] * sH[i][c];
      part[kMpnnOffWd + q] = acc;
    } else {
      const int k = q - 3 * kHid;
      for (int i = 0; i < kTile; ++i) acc += sGo[i][k];
      part[kMpnnOffBd + k] = acc;
    }
  }
}

// One layer backward over a tile: gpre = GH * relu mask; two tcgen05 products
//   g_a[node][in]   = sum_out gpre[node][out] W[out][in]      (M 128 nodes, N 128, K 64)
//   dW^T[in][out]   = sum_node a[node][in] gpre[node][out]    (M 128 features, N 64, K 128 nodes)
// Epilogue: GHn = GH + g_a[:, :64]; Q = g_a[:, 64:] / deg; dW, db into gpart.
constexpr size_t kBwdSmem = 32768 /*sAT*/ + 16384 /*sG1*/ + 16384 /*sG2*/ + 16384 /*sWT*/ + kTile * kHid * 4;

__global__ void __launch_bounds__(2 * kTile) mpnn_layer_bwd_kernel(const __grid_constant__ MpnnTrain t, int layer) {
  const MpnnDev& m = t.m;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  unsigned char* sAT = smem;             // a^T: 128 features x 128 nodes (K-major over nodes)
  unsigned char* sG1 = smem + 32768;     // gpre: 128 nodes x 64 outs
  unsigned char* sG2 = smem + 49152;     // gpre^T: 64 outs x 128 nodes
  unsigned char* sWT = smem + 65536;     // W^T: 128 in x 64 out
  float* sGf = reinterpret_cast<float*>(smem + 81920);  // gpre FP32 [128][64]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nl = tid & (kTile - 1), half = tid >> 7;
  const int node = blockIdx.x * kTile + nl;
  const __nv_bfloat16* Hin = m.H[layer];
  if (warp == 0) umma::tmem_alloc(&tmem_base, 256);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  {
    const uint4* wsrc = reinterpret_cast<const uint4*>(m.WlT_p + (size_t)layer * kHid * 2 * kHid);
#pragma unroll
    for (int q = 0; q < 4; ++q) reinterpret_cast<uint4*>(sWT)[tid + q * 2 * kTile] = __ldg(wsrc + tid + q * 2 * kTile);
  }
  {
    // a = [h_in, mean of neighbours] for this thread's 32 channels, as a^T
    float acc[32];
    float own[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) acc[k] = own[k] = 0.f;
    if (node < m.n_nodes) {
      const uint4* hs = reinterpret_cast<const uint4*>(Hin + (size_t)node * kHid + 32 * half);
#pragma unroll
      for (int c = 0; c < 4; ++c) unpack8(hs[c], own + 8 * c);
      const int j0 = __ldg(m.adj_ptr + node), j1 = __ldg(m.adj_ptr + node + 1);
      for (int j = j0; j < j1; ++j) {
        const int nb = __ldg(m.adj_idx + j);
        const uint4* hn = reinterpret_cast<const uint4*>(Hin + (size_t)nb * kHid + 32 * half);
        uint4 v[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) v[c] = hn[c];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          float f[8];
          unpack8(v[c], f);
#pragma unroll
          for (int q = 0; q < 8; ++q) acc[8 * c + q] += f[q];
        }
      }
      const float dd = __ldg(m.deg_inv + node);
#pragma unroll
      for (int k = 0; k < 32; ++k) acc[k] *= dd;
    }
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      *reinterpret_cast<__nv_bfloat16*>(sAT + umma::kmajor_off(32 * half + k, nl, kTile)) =
          __float2bfloat16_rn(own[k]);
      *reinterpret_cast<__nv_bfloat16*>(sAT + umma::kmajor_off(kHid + 32 * half + k, nl, kTile)) =
          __float2bfloat16_rn(acc[k]);
    }
    // gpre for this thread's 32 output channels
    float g[32];
    uint32_t bits = 0;
    if (node < m.n_nodes) bits = reinterpret_cast<const uint32_t*>(m.mask[layer])[2 * (size_t)node + half];
#pragma unroll
    for (int k = 0; k < 32; ++k) g[k] = 0.f;
    if (node < m.n_nodes) {
      const float4* gp = reinterpret_cast<const float4*>(t.GH + (size_t)node * kHid + 32 * half);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const float4 v = gp[c];
        g[4 * c] = v.x;
        g[4 * c + 1] = v.y;
        g[4 * c + 2] = v.z;
        g[4 * c + 3] = v.w;
      }
#pragma unroll
      for (int k = 0; k < 32; ++k)
        if (!((bits >> k) & 1u)) g[k] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      sGf[nl * kHid + 32 * half + k] = g[k];
      *reinterpret_cast<__nv_bfloat16*>(sG2 + umma::kmajor_off(32 * half + k, nl, kTile)) = __float2bfloat16_rn(g[k]);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
      *reinterpret_cast<uint4*>(sG1 + umma::kmajor_off(nl, 32 * half + 8 * c, kHid)) = pack8(g + 8 * c);
  }
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (tid == 0) {
    const uint32_t g1 = umma::smem_u32(sG1), wt = umma::smem_u32(sWT);
    const uint32_t at = umma::smem_u32(sAT), g2 = umma::smem_u32(sG2);
    const uint32_t id1 = umma::idesc_bf16(kTile, 2 * kHid), id2 = umma::idesc_bf16(kTile, kHid);
#pragma unroll
    for (int q = 0; q < kHid / 16; ++q)
      umma::mma_bf16(tbase, umma::smem_desc(g1 + 256 * q, kHid), umma::smem_desc(wt + 256 * q, kHid), id1,
                     q > 0 ? 1u : 0u);
#pragma unroll
    for (int q = 0; q < kTile / 16; ++q)
      umma::mma_bf16(tbase + 2 * kHid, umma::smem_desc(at + 256 * q, kTile), umma::smem_desc(g2 + 256 * q, kTile),
                     id2, q > 0 ? 1u : 0u);
    umma::commit(&mbar);
  }
  __syncwarp();
  const bool ok = umma::mbar_wait(&mbar, 0, kPolls);
  umma::fence_after_sync();
  const int row = 32 * (warp & 3) + lane;
  const int ehalf = warp >> 2;
  float* part = t.gpart + (size_t)blockIdx.x * kMpnnParams;
  if (ok) {
    // g_a: lane = node; half 0 -> self path, half 1 -> aggregation path
    const int enode = blockIdx.x * kTile + row;
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
      float v[16];
      umma::tmem_ld16(umma::taddr(tbase, 32 * (warp & 3), kHid * ehalf + 16 * cc), v);
      if (enode < m.n_nodes) {
        if (ehalf == 0) {
          const float* gh = t.GH + (size_t)enode * kHid + 16 * cc;
          float* dst = t.GHn + (size_t)enode * kHid + 16 * cc;
#pragma unroll
          for (int j = 0; j < 16; ++j) dst[j] = gh[j] + v[j];
        } else {
          const float dd = __ldg(m.deg_inv + enode);
          float* dst = t.Q + (size_t)enode * kHid + 16 * cc;
#pragma unroll
          for (int j = 0; j < 16; ++j) dst[j] = v[j] * dd;
        }
      }
    }
    // dW^T: lane = input feature, columns 128 + out
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
      const int o0 = 32 * ehalf + 16 * cc;
      float v[16];
      umma::tmem_ld16(umma::taddr(tbase, 32 * (warp & 3), 2 * kHid + o0), v);
#pragma unroll
      for (int j = 0; j < 16; ++j) part[kMpnnOffW(layer) + (o0 + j) * 2 * kHid + row] = v[j];
    }
  } else if (lane == 0) {
    atomicExch(m.err, 1);
  }
  if (tid < kHid) {
    float acc = 0.f;
    for (int i = 0; i < kTile; ++i) acc += sGf[i * kHid + tid];
    part[kMpnnOffB(layer) + tid] = acc;
  }
  umma::drain_mma(&mbar, 0, ok, kPolls);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, 256);
}

// GH[j] = GHn[j] + sum_{i in N(j)} Q[i]  (transpose of the mean aggregation)
__global__ void __launch_bounds__(256) mpnn_scatter_bwd_kernel(const __grid_constant__ MpnnTrain t) {
  const MpnnDev& m = t.m;
  const int gid = blockIdx.x * 256 + threadIdx.x;
  const int node = gid >> 1, half = gid & 1;
  if (node >= m.n_nodes) return;
  float acc[32];
  const float4* self = reinterpret_cast<const float4*>(t.GHn + (size_t)node * kHid + 32 * half);
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const float4 v = self[c];
    acc[4 * c] = v.x;
    acc[4 * c + 1] = v.y;
    acc[4 * c + 2] = v.z;
    acc[4 * c + 3] = v.w;
  }
  const int j0 = __ldg(m.adj_ptr + node), j1 = __ldg(m.adj_ptr + node + 1);
  for (int j = j0; j < j1; ++j) {
    const int nb = __ldg(m.adj_idx + j);
    const float4* q = reinterpret_cast<const float4*>(t.Q + (size_t)nb * kHid + 32 * half);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const float4 v = q[c];
      acc[4 * c] += v.x;
      acc[4 * c + 1] += v.y;
      acc[4 * c + 2] += v.z;
      acc[4 * c + 3] += v.w;
    }
  }
  float4* dst = reinterpret_cast<float4*>(t.GH + (size_t)node * kHid + 32 * half);
#pragma unroll
  for (int c = 0; c < 8; ++c) dst[c] = make_float4(acc[4 * c], acc[4 * c + 1], acc[4 * c + 2], acc[4 * c + 3]);
}

// encoder: gpre0 = GH * (h0 > 0); dW_e = sum gpre0 f^T, db_e = sum gpre0
__global__ void __launch_bounds__(kTile) mpnn_enc_bwd_kernel(const __grid_constant__ MpnnTrain t,
                                                             const float* __restrict__ r,
                                                             const float* __restrict__ dinv) {
  const MpnnDev& m = t.m;
  __shared__ float sG[kTile][kHid + 1];
  __shared__ float sF[kTile][kIn];
  const int tid = threadIdx.x;
  const int node = blockIdx.x * kTile + tid;
  float f[kIn];
#pragma unroll
  for (int k = 0; k < kIn; ++k) f[k] = 0.f;
  if (node < m.n_nodes) {
    const double s = m.scal[0];
    const float inv_s = s > 0.0 ? (float)(1.0 / s) : 0.f;
    const float4 rv = reinterpret_cast<const float4*>(r)[node];
    const float4 dv = reinterpret_cast<const float4*>(dinv)[node];
    f[0] = sqrtf(dv.x) * rv.x * inv_s;
    f[1] = sqrtf(dv.y) * rv.y * inv_s;
    f[2] = sqrtf(dv.z) * rv.z * inv_s;
    const int fx = (int)m.fixed[node];
    f[3] = (float)(fx & 1);
    f[4] = (float)((fx >> 1) & 1);
    f[5] = (float)((fx >> 2) & 1);
    f[6] = m.cfeat[node];
#pragma unroll
    for (int k = 0; k < kIn; ++k) f[k] = __bfloat162float(__float2bfloat16_rn(f[k]));
    const uint4* hp = reinterpret_cast<const uint4*>(m.H[0] + (size_t)node * kHid);
    const float* gh = t.GH + (size_t)node * kHid;
#pragma unroll
    for (int c = 0; c < kHid / 8; ++c) {
      float h[8];
      unpack8(hp[c], h);
#pragma unroll
      for (int q = 0; q < 8; ++q) sG[tid][8 * c + q] = h[q] > 0.f ? gh[8 * c + q] : 0.f;
    }
  } else {
#pragma unroll
    for (int c = 0; c < kHid; ++c) sG[tid][c] = 0.f;
  }
#pragma unroll
  for (int k = 0; k < kIn; ++k) sF[tid][k] = f[k];
  __syncthreads();
  float* part = t.gpart + (size_t)blockIdx.x * kMpnnParams;
  for (int q = tid; q < kHid * kIn + kHid; q += kTile) {
    float acc = 0.f;
    if (q < kHid * kIn) {
      const int o = q / kIn, k = q - o * kIn;
      for (int i = 0; i < kTile; ++i) acc += sG[i][o] * sF[i][k];
      part[kMpnnOffWe + q] = acc;
    } else {
      const int o = q - kHid * kIn;
      for (int i = 0; i < kTile; ++i) acc += sG[i][o];
      part[kMpnnOffBe + o] = acc;
    }
  }
}

// grad[p] (+)= sum over tiles of gpart[tile][p], tiles in index order
__global__ void mpnn_grad_reduce_kernel(const float* __restrict__ gpart, int tiles, float* grad, int accumulate) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMpnnParams) return;
  float acc = 0.f;
  for (int k = 0; k < tiles; ++k) acc += __ldg(gpart + (size_t)k * kMpnnParams + p);
  grad[p] = accumulate ? grad[p] + acc : acc;
}

// Adam with bias correction (oracle/mpnn_oracle.py adam_step); grad scaled by gscale
__global__ void mpnn_adam_kernel(float* w, float* mom, float* var, const float* grad, float gscale, float lr,
                                 float b1, float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMpnnParams) return;
  const float g = grad[p] * gscale;
  const float mo = b1 * mom[p] + (1.f - b1) * g;
  const float va = b2 * var[p] + (1.f - b2) * g * g;
  mom[p] = mo;
  var[p] = va;
  w[p] -= lr * (mo / c1) / (sqrtf(va / c2) + eps);
}

// ───────────────────────── launchers ─────────────────────────

static inline int nblk(int n, int t) { return (n + t - 1) / t; }

// The encoder's shared memory is padded to 32 KB so at most 7 CTAs share an
// SM: 7 x 64 TMEM columns stay within the SM's 512.
constexpr size_t kEncSmem = 32 * 1024;
constexpr size_t kLayerSmem = kTile * 2 * kHid * 2 + kHid * 2 * kHid * 2;  // 48 KB: <= 4 CTAs per SM

void prepare_mpnn_kernels() {
  raise_smem_limit_k(mpnn_layer_bwd_kernel);
  raise_smem_limit_k(mpnn_encode_kernel);
  raise_smem_limit_k(mpnn_layer_kernel<false>);
  raise_smem_limit_k(mpnn_layer_kernel<true>);
}

void launch_mpnn_pack(const float* w, __nv_bfloat16* We_p, __nv_bfloat16* Wl_p, __nv_bfloat16* WlT_p,
                      cudaStream_t s) {
  const int n = kMpnnLayers * kHid * 2 * kHid;
  mpnn_pack_kernel<<<nblk(n, 256), 256, 0, s>>>(w, We_p, Wl_p, WlT_p);
}

void launch_mpnn_backward(const MpnnTrain& t, const float* r, const float* dinv, const float* gz, float* grad,
                          int accumulate, cudaStream_t s) {
  const int tiles = nblk(t.m.n_nodes, kTile);
  mpnn_dec_bwd_kernel<<<tiles, kTile, 0, s>>>(t, dinv, gz);
  for (int l = kMpnnLayers - 1; l >= 0; --l) {
    mpnn_layer_bwd_kernel<<<tiles, 2 * kTile, kBwdSmem, s>>>(t, l);
    mpnn_scatter_bwd_kernel<<<nblk(2 * t.m.n_nodes, 256), 256, 0, s>>>(t);
  }
  mpnn_enc_bwd_kernel<<<tiles, kTile, 0, s>>>(t, r, dinv);
  mpnn_grad_reduce_kernel<<<nblk(kMpnnParams, 256), 256, 0, s>>>(t.gpart, tiles, grad, accumulate);
}

void launch_mpnn_adam(float* w, float* mom, float* var, const float* grad, float gscale, float lr, int step,
                      cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  mpnn_adam_kernel<<<nblk(kMpnnParams, 256), 256, 0, s>>>(w, mom, var, grad, gscale, lr, b1, b2, 1e-8f, c1, c2);
}

void launch_mpnn_forward(const MpnnDev& m, const float* r, const float* dinv, float* z, const CGState* cg,
                         Reduce red, int site, cudaStream_t s) {
  mpnn_scale_kernel<<<nblk(m.n_nodes, 256), 256, 0, s>>>(m, r, dinv, cg, red, site);
  const int tiles = nblk(m.n_nodes, kTile);
  mpnn_encode_kernel<<<tiles, kTile, kEncSmem, s>>>(m, r, dinv, cg);
  for (int l = 0; l < kMpnnLayers - 1; ++l)
    mpnn_layer_kernel<false><<<tiles, 2 * kTile, kLayerSmem, s>>>(m, l, r, dinv, z, cg);
  mpnn_layer_kernel<true><<<tiles, 2 * kTile, kLayerSmem, s>>>(m, kMpnnLayers - 1, r, dinv, z, cg);
}

}  // namespace femb200
