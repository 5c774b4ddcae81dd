// Dense SPD inverse of the two-level preconditioner's coarse operator:
// Cholesky A = L L^T, W = L^-1, A^-1 = W^T W (lower triangle), blocked in
// B x B tiles (FP32: B = 128, FP64: B = 64) on a padded copy of A whose size
// is a whole number of tiles (the padding is the identity, so L and W are
// block diagonal there and no kernel handles a ragged edge).
//
//   factor, for k = 0 .. nt - 1 (main stream):
//     dense_diag_kernel    one CTA: L_kk = chol(A_kk) in shared memory and its
//                          inverse W_kk = L_kk^-1 (a pivot <= 0 records its
//                          column in *info and the factorisation continues
//                          with a unit pivot, so every launch completes)
//     dense_panel_kernel   L_ik = A_ik W_kk^T, i > k
//     dense_update_kernel  A_ij -= L_ik L_jk^T, k < j <= i (column k + 1 here,
//                          the columns > k + 1 on a third stream, so the next
//                          diagonal and panel kernels overlap them)
//   invert, right-looking, step k on a second stream once panel k is done:
//     dense_wfin_kernel    W_kj = W_kk R_kj, j < k (R: the accumulated row)
//     dense_wupd_kernel    R_ij -= L_ik W_kj, i > k, j <= k
//   product (after both streams):
//     dense_syrk_kernel    (A^-1)_ij = sum_{l>=i} W_li^T W_lj, i >= j, or
//     dense_syrk_tc_kernel the same on TF32 tensor cores (tcgen05)
//
// The SIMT tile products run on a micro-kernel: 256 threads, each an
// (B/16) x (B/16) block of the output tile, operands staged in shared memory
// in chunks of kKC of the inner dimension.  These replace the cuSOLVER
// potrf / potri and cuBLAS trsm / syrk calls the coarse set-up made before.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/femb200.h"
#include "fem_internal.h"
#include "fem_umma.cuh"

namespace femb200 {

template <typename T>
struct DenseCfg;
template <>
struct DenseCfg<float> {
  static constexpr int B = 128, TM = 8;
};
template <>
struct DenseCfg<double> {
  static constexpr int B = 64, TM = 4;
};
constexpr int kDenseThreads = 256;
constexpr int kKC = 16;  // inner-dimension chunk staged in shared memory

// Four consecutive FP32 (or two FP64) values moved as one 16-byte access.
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using V = float4;
  static constexpr int W = 4;
  __device__ static void unpack(const V& v, float* o) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
  __device__ static V pack(const float* o) { return make_float4(o[0], o[1], o[2], o[3]); }
};
template <>
struct Vec16<double> {
  using V = double2;
  static constexpr int W = 2;
  __device__ static void unpack(const V& v, double* o) { o[0] = v.x; o[1] = v.y; }
  __device__ static V pack(const double* o) { return make_double2(o[0], o[1]); }
};

template <typename T>
constexpr int dense_ld() {  // shared row stride of a staged operand chunk
  return DenseCfg<T>::B + 4;
}

// Stages rows k0 .. k0 + kKC - 1 of the inner dimension of one B-row
// operand into s[k][m]: element (m, k) is p[k * ld + m] (m contiguous, a
// column-major tile) or, with KC, p[m * ld + k] (k contiguous).  16-byte
// global loads along the contiguous index (all operand tiles start on a
// multiple of B elements and ld is a multiple of B, so they are aligned).
template <typename T, bool KC>
__device__ __forceinline__ void dense_stage(const T* __restrict__ p, int ld, int k0, T* s) {
  using VT = Vec16<T>;
  constexpr int B = DenseCfg<T>::B, W = VT::W;
  constexpr int LD = dense_ld<T>();
  constexpr int NV = B * kKC / W;  // vectors per chunk
#pragma unroll
  for (int q = threadIdx.x; q < NV; q += kDenseThreads) {
    T v[W];
    if (KC) {
      const int m = q / (kKC / W), k = (q % (kKC / W)) * W;
      VT::unpack(__ldcg(reinterpret_cast<const typename VT::V*>(p + (size_t)m * ld + k0 + k)), v);
#pragma unroll
      for (int w = 0; w < W; ++w) s[(k + w) * LD + m] = v[w];
    } else {
      const int k = q / (B / W), m = (q % (B / W)) * W;
      *reinterpret_cast<typename VT::V*>(s + k * LD + m) =
          __ldcg(reinterpret_cast<const typename VT::V*>(p + (size_t)(k0 + k) * ld + m));
    }
  }
}

// acc(r, c) += sum_k A(r, k) Bt(c, k) over one tile of the inner dimension
// (k < B); A and Bt are B-row operands (see dense_stage).  Thread t owns the
// rows ty * H + [0, H) and B/2 + ty * H + [0, H), ty = t % 16, and the same
// columns with tx = t / 16 (H = TM / 2), so the lanes of a warp cover
// consecutive rows: coalesced stores of a column-major tile.
template <typename T, bool AK, bool BK>
__device__ __forceinline__ void dense_mma(T (&acc)[DenseCfg<T>::TM][DenseCfg<T>::TM], const T* A, int lda,
                                          const T* Bt, int ldb, T* sA, T* sB) {
  using VT = Vec16<T>;
  constexpr int B = DenseCfg<T>::B, TM = DenseCfg<T>::TM, H = TM / 2, LD = dense_ld<T>();
  static_assert(H == VT::W, "a thread's half-row block is one 16-byte vector");
  const int ty = threadIdx.x & 15, tx = threadIdx.x >> 4;
  for (int k0 = 0; k0 < B; k0 += kKC) {
    __syncthreads();
    dense_stage<T, AK>(A, lda, k0, sA);
    dense_stage<T, BK>(Bt, ldb, k0, sB);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kKC; ++k) {
      T a[TM], b[TM];
      VT::unpack(*reinterpret_cast<const typename VT::V*>(sA + k * LD + ty * H), a);
      VT::unpack(*reinterpret_cast<const typename VT::V*>(sA + k * LD + B / 2 + ty * H), a + H);
      VT::unpack(*reinterpret_cast<const typename VT::V*>(sB + k * LD + tx * H), b);
      VT::unpack(*reinterpret_cast<const typename VT::V*>(sB + k * LD + B / 2 + tx * H), b + H);
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TM; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
  }
}

// tile-local row / column of accumulator entry i
template <typename T>
__device__ __forceinline__ int dense_rc(int t16, int i) {
  constexpr int B = DenseCfg<T>::B, H = DenseCfg<T>::TM / 2;
  return i < H ? t16 * H + i : B / 2 + t16 * H + (i - H);
}

// Writes the thread's accumulator block to a column-major tile (ld), one
// 16-byte store per half column: OP 0 stores acc, 1 subtracts it from the
// tile, 2 stores -acc.
template <typename T, int OP>
__device__ __forceinline__ void dense_store(T* tile, int ld, const T (&acc)[DenseCfg<T>::TM][DenseCfg<T>::TM]) {
  using VT = Vec16<T>;
  constexpr int B = DenseCfg<T>::B, TM = DenseCfg<T>::TM, H = TM / 2;
  const int ty = threadIdx.x & 15, tx = threadIdx.x >> 4;
#pragma unroll
  for (int b = 0; b < TM; ++b) {
    const int col = b < H ? tx * H + b : B / 2 + tx * H + (b - H);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      typename VT::V* q = reinterpret_cast<typename VT::V*>(tile + (size_t)col * ld + half * (B / 2) + ty * H);
      T v[H];
#pragma unroll
      for (int i = 0; i < H; ++i) v[i] = acc[half * H + i][b];
      if (OP == 1) {
        T o[H];
        VT::unpack(*q, o);
#pragma unroll
        for (int i = 0; i < H; ++i) v[i] = o[i] - v[i];
      } else if (OP == 2) {
#pragma unroll
        for (int i = 0; i < H; ++i) v[i] = -v[i];
      }
      *q = VT::pack(v);
    }
  }
}

template <typename T>
__device__ __forceinline__ void dense_zero(T (&acc)[DenseCfg<T>::TM][DenseCfg<T>::TM]) {
#pragma unroll
  for (int i = 0; i < DenseCfg<T>::TM; ++i)
#pragma unroll
    for (int j = 0; j < DenseCfg<T>::TM; ++j) acc[i][j] = T(0);
}

// Lower-triangle tile t -> (I, J), J <= I, in row order.
__device__ __forceinline__ void dense_tri(int t, int& I, int& J) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  I = i;
  J = t - i * (i + 1) / 2;
}

// A = the padded copy of src's lower triangle (identity beyond n); W = 0
template <typename T>
__global__ void __launch_bounds__(256) dense_pad_kernel(const double* __restrict__ src, int n, T* A, T* W, int N) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (size_t)N * N) return;
  const int c = (int)(q / N), r = (int)(q % N);
  T v = T(0);
  if (r < n && c < n) {
    if (r >= c) v = (T)src[(size_t)c * n + r];
  } else if (r == c) {
    v = T(1);
  }
  A[q] = v;
  W[q] = T(0);
}

// Correctly rounded 1 / sqrt(x) (FP32) or CUDA's rsqrt (FP64): one per pivot,
// multiplied through the column instead of a division per entry.
__device__ __forceinline__ float dense_rsqrt(float x) { return __frsqrt_rn(x); }
__device__ __forceinline__ double dense_rsqrt(double x) { return rsqrt(x); }

// Diagonal tile k: L_kk = chol(A_kk) and X = L_kk^-1 in shared memory
// (L[c * S + r] = L(r, c)), both blocked in 32-wide panels so the sequential
// parts run inside one warp, in registers, and the CTA synchronises a few
// times per panel:
//   Cholesky, panel p (columns j0 .. j0 + 31):
//     warp 0 factors the 32 x 32 diagonal block in registers (lane = row,
//     the pivot column passed by shuffles) and inverts it (lane = column,
//     the factor read back as shared-memory broadcasts),
//     the rows below are L_ip = A_ip X_pp^T (16 columns per thread),
//     the rank-32 update of the trailing lower triangle runs on 4 x 4
//     register tiles;
//   then block row k is finished (X_kq = X_kk R_kq, q < k) and subtracted
//   from the rows below (R_iq -= L_ik X_kq), for k = 0, 1, ...
template <typename T>
__global__ void __launch_bounds__(kDenseThreads) dense_diag_kernel(T* A, T* W, int N, int k, int* info) {
  constexpr int B = DenseCfg<T>::B, S = B + 1, P = 32, NP = B / P;
  constexpr unsigned kFull = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char s_raw[];
  T* L = reinterpret_cast<T*>(s_raw);  // L[c * S + r]
  T* X = L + B * S;                     // X[c * S + r] = (L^-1)(r, c)
  T* Xt = X + B * S;                    // Xt[l * P + j] = (L_pp^-1)(j, l), current panel
  __shared__ T s_rinv[32];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t off = (size_t)k * B * N + (size_t)k * B;
#pragma unroll 8
  for (int it = 0; it < B * B / kDenseThreads; ++it) {
    const int q = tid + it * kDenseThreads, c = q / B, r = q % B;
    const T v = A[off + (size_t)c * N + r];
    L[c * S + r] = r >= c ? v : T(0);
    X[c * S + r] = T(0);
  }
  __syncthreads();
  for (int p = 0; p < NP; ++p) {
    const int j0 = p * P;
    if (warp == 0) {
      T a[P];  // row j0 + lane of the diagonal block
      T rinv = T(0);  // lane r: 1 / L(j0 + r, j0 + r)
#pragma unroll
      for (int c = 0; c < P; ++c) a[c] = c <= lane ? L[(j0 + c) * S + j0 + lane] : T(0);
#pragma unroll
      for (int j = 0; j < P; ++j) {
        T d = __shfl_sync(kFull, a[j], j);
        if (!(d > T(0))) {
          if (lane == 0) atomicCAS(info, 0, k * B + j0 + j + 1);
          d = T(1);
        }
        const T rs = dense_rsqrt(d);  // 1 / L(j, j)
        if (lane == j) {
          a[j] = d * rs;
          rinv = rs;
        }
        if (lane > j) a[j] *= rs;
#pragma unroll
        for (int c = 1; c < P; ++c) {  // c > j: constant trip counts unroll fully
          if (c > j) {
            const T lc = __shfl_sync(kFull, a[j], c);
            if (lane >= c) a[c] -= a[j] * lc;
          }
        }
      }
#pragma unroll
      for (int c = 0; c < P; ++c)
        if (c <= lane) L[(j0 + c) * S + j0 + lane] = a[c];
      s_rinv[lane] = rinv;
      __syncwarp();
      // column lane of L_pp^-1: x[r] = (delta(r, lane) - sum_{l < r} L(r, l) x[l]) / L(r, r)
      T x[P];
#pragma unroll
      for (int r = 0; r < P; ++r) {
        T acc = r == lane ? T(1) : T(0);
#pragma unroll
        for (int l = 0; l < P - 1; ++l)
          if (l < r) acc -= L[(j0 + l) * S + j0 + r] * x[l];
        x[r] = acc * s_rinv[r];
      }
#pragma unroll
      for (int r = 0; r < P; ++r) {
        X[(j0 + lane) * S + j0 + r] = x[r];
        Xt[lane * P + r] = x[r];
      }
    }
    __syncthreads();
    const int rows = B - j0 - P;  // rows below the diagonal block
    if (rows == 0) break;
    {
      // L(r, j0 + j) = sum_{l <= j} A(r, j0 + l) Xt[l * P + j], columns 16 cg .. 16 cg + 15
      constexpr int CG = 16;
      using VT = Vec16<T>;
      constexpr int W = VT::W;
      const bool act = tid < rows * (P / CG);
      const int r = j0 + P + (act ? tid % rows : 0), cg = act ? tid / rows : 0;
      T acc[CG];
#pragma unroll
      for (int j = 0; j < CG; ++j) acc[j] = T(0);
      if (act) {
        const int lend = cg * CG + CG;
        for (int l = 0; l < lend; ++l) {
          const T av = L[(j0 + l) * S + r];
          const typename VT::V* xt = reinterpret_cast<const typename VT::V*>(Xt + l * P + cg * CG);
#pragma unroll
          for (int v = 0; v < CG / W; ++v) {
            T xv[W];
            VT::unpack(xt[v], xv);
#pragma unroll
            for (int w = 0; w < W; ++w) acc[v * W + w] += av * xv[w];
          }
        }
      }
      __syncthreads();
      if (act) {
#pragma unroll
        for (int j = 0; j < CG; ++j) L[(j0 + cg * CG + j) * S + r] = acc[j];
      }
      __syncthreads();
    }
    {
      // trailing lower triangle on 4 x 4 tiles: L(r, c) -= sum_l L(r, j0 + l) L(c, j0 + l)
      const int nt4 = rows / 4, ntri = nt4 * (nt4 + 1) / 2, base = j0 + P;
      for (int q = tid; q < ntri; q += kDenseThreads) {
        int ti, tj;  // tj <= ti
        dense_tri(q, ti, tj);
        const int r0 = base + 4 * ti, c0 = base + 4 * tj;
        T acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
#pragma unroll 4
        for (int l = j0; l < j0 + P; ++l) {
          T lr[4], lc[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            lr[i] = L[l * S + r0 + i];
            lc[i] = L[l * S + c0 + i];
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] += lr[i] * lc[j];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (r0 + i >= c0 + j) L[(c0 + j) * S + r0 + i] -= acc[i][j];
      }
    }
    __syncthreads();
  }
  // block rows of X: finish row block kb (X_kq = X_kk R_kq, q < kb; R
  // accumulated in place), then R_iq -= L_ik X_kq for the row blocks below,
  // for kb = 0, 1, ...: register-tiled, lane = row, the other operand
  // broadcast from shared memory
  constexpr int NW = kDenseThreads / 32;
  for (int kb = 0; kb < NP; ++kb) {
    const int k0 = kb * P;
    if (kb > 0) {
      // X(k0 + lane, c) for the columns c = warp + NW t < k0
      constexpr int NV = (NP - 1) * P / NW;
      const int nc = k0 / NW;
      T v[NV];
#pragma unroll
      for (int t = 0; t < NV; ++t) v[t] = T(0);
      for (int l = 0; l < P; ++l) {
        const T xl = X[(k0 + l) * S + k0 + lane];
#pragma unroll
        for (int t = 0; t < NV; ++t)
          if (t < nc) v[t] += xl * X[(warp + NW * t) * S + k0 + l];
      }
      __syncthreads();
#pragma unroll
      for (int t = 0; t < NV; ++t)
        if (t < nc) X[(warp + NW * t) * S + k0 + lane] = v[t];
      __syncthreads();
    }
    // rows below block kb, columns up to the end of block kb: items of 32
    // rows x CW columns, one per warp in turn
    const int rows = B - k0 - P, cols = k0 + P;
    if (rows > 0) {
      constexpr int CW = 8;
      const int rw32 = rows / 32, items = rw32 * (cols / CW);
      for (int it = warp; it < items; it += NW) {
        const int r = k0 + P + (it % rw32) * 32 + lane, c0 = (it / rw32) * CW;
        T acc[CW];
#pragma unroll
        for (int w = 0; w < CW; ++w) acc[w] = T(0);
        for (int l = 0; l < P; ++l) {
          const T lv = L[(k0 + l) * S + r];
#pragma unroll
          for (int w = 0; w < CW; ++w) acc[w] += lv * X[(c0 + w) * S + k0 + l];
        }
#pragma unroll
        for (int w = 0; w < CW; ++w) X[(c0 + w) * S + r] -= acc[w];
      }
      __syncthreads();
    }
  }
  for (int q = tid; q < B * B; q += kDenseThreads) {
    const int c = q / B, r = q % B;
    A[off + (size_t)c * N + r] = L[c * S + r];
    W[off + (size_t)c * N + r] = X[c * S + r];
  }
}

// L_ik = A_ik W_kk^T for i = k + 1 + blockIdx.x
template <typename T>
__global__ void __launch_bounds__(kDenseThreads) dense_panel_kernel(T* A, const T* W, int N, int k) {
  constexpr int B = DenseCfg<T>::B, TM = DenseCfg<T>::TM;
  __shared__ __align__(16) T sA[kKC * dense_ld<T>()];
  __shared__ __align__(16) T sB[kKC * dense_ld<T>()];
  const int i = k + 1 + (int)blockIdx.x;
  T* Aik = A + (size_t)k * B * N + (size_t)i * B;
  const T* Wkk = W + (size_t)k * B * N + (size_t)k * B;
  T acc[TM][TM];
  dense_zero<T>(acc);
  // (A_ik W_kk^T)(r, c) = sum_q A_ik(r, q) W_kk(c, q): both operands m-contiguous
  dense_mma<T, false, false>(acc, Aik, N, Wkk, N, sA, sB);
  __syncthreads();
  dense_store<T, 0>(Aik, N, acc);
}

// A_ij -= L_ik L_jk^T over lower tiles j <= i: with COL the column j = k + 1
// (i = k + 1 + blockIdx.x), else the triangle j >= k + 1 + j_ofs (blockIdx.x
// in row order).
template <typename T, bool COL>
__global__ void __launch_bounds__(kDenseThreads) dense_update_kernel(T* A, int N, int k, int j_ofs) {
  constexpr int B = DenseCfg<T>::B, TM = DenseCfg<T>::TM;
  __shared__ __align__(16) T sA[kKC * dense_ld<T>()];
  __shared__ __align__(16) T sB[kKC * dense_ld<T>()];
  int I = (int)blockIdx.x, J = 0;
  if (!COL) dense_tri((int)blockIdx.x, I, J);
  const int i = k + 1 + j_ofs + I, j = k + 1 + j_ofs + J;
  const T* Lik = A + (size_t)k * B * N + (size_t)i * B;
  const T* Ljk = A + (size_t)k * B * N + (size_t)j * B;
  T acc[TM][TM];
  dense_zero<T>(acc);
  dense_mma<T, false, false>(acc, Lik, N, Ljk, N, sA, sB);
  dense_store<T, 1>(A + (size_t)j * B * N + (size_t)i * B, N, acc);
}

// W = L^-1, right-looking over tile rows.  W's lower tiles below the
// diagonal start at 0 and accumulate R_ij = -sum_{l<i} L_il W_lj; step k
// finishes tile row k (dense_wfin_kernel: W_kj = W_kk R_kj, j < k) and
// subtracts it from the rows below (dense_wupd_kernel: R_ij -= L_ik W_kj,
// i > k, j <= k), one tile product per CTA.
template <typename T>
__global__ void __launch_bounds__(kDenseThreads) dense_wfin_kernel(T* W, int N, int k) {
  constexpr int B = DenseCfg<T>::B, TM = DenseCfg<T>::TM;
  __shared__ __align__(16) T sA[kKC * dense_ld<T>()];
  __shared__ __align__(16) T sB[kKC * dense_ld<T>()];
  const int j = (int)blockIdx.x;
  T* Wkj = W + (size_t)j * B * N + (size_t)k * B;
  T acc[TM][TM];
  dense_zero<T>(acc);
  // (W_kk R_kj)(r, c) = sum_q W_kk(r, q) R_kj(q, c)
  dense_mma<T, false, true>(acc, W + (size_t)k * B * N + (size_t)k * B, N, Wkj, N, sA, sB);
  __syncthreads();
  dense_store<T, 0>(Wkj, N, acc);
}

template <typename T>
__global__ void __launch_bounds__(kDenseThreads) dense_wupd_kernel(const T* A, T* W, int N, int k) {
  constexpr int B = DenseCfg<T>::B, TM = DenseCfg<T>::TM;
  __shared__ __align__(16) T sA[kKC * dense_ld<T>()];
  __shared__ __align__(16) T sB[kKC * dense_ld<T>()];
  const int j = (int)blockIdx.x % (k + 1), i = k + 1 + (int)blockIdx.x / (k + 1);
  T acc[TM][TM];
  dense_zero<T>(acc);
  // (L_ik W_kj)(r, c) = sum_q L_ik(r, q) W_kj(q, c)
  dense_mma<T, false, true>(acc, A + (size_t)k * B * N + (size_t)i * B, N, W + (size_t)j * B * N + (size_t)k * B, N,
                            sA, sB);
  dense_store<T, 1>(W + (size_t)j * B * N + (size_t)i * B, N, acc);
}

// (A^-1)_ij = sum_{l=i}^{nt-1} W_li^T W_lj for the lower tiles i >= j; out
// holds the n x n result column-major (entries beyond n are the padding's).
template <typename T, typename TO>
__global__ void __launch_bounds__(kDenseThreads) dense_syrk_kernel(const T* W, int N, int nt, TO* out, int n) {
  constexpr int B = DenseCfg<T>::B, TM = DenseCfg<T>::TM;
  __shared__ __align__(16) T sA[kKC * dense_ld<T>()];
  __shared__ __align__(16) T sB[kKC * dense_ld<T>()];
  int i, j;
  dense_tri((int)blockIdx.x, i, j);
  T acc[TM][TM];
  dense_zero<T>(acc);
  // X(r, c) = sum_l sum_q W_li(q, r) W_lj(q, c): both operands k-contiguous
  for (int l = i; l < nt; ++l)
    dense_mma<T, true, true>(acc, W + (size_t)i * B * N + (size_t)l * B, N, W + (size_t)j * B * N + (size_t)l * B, N,
                             sA, sB);
  const int ty = threadIdx.x & 15, tx = threadIdx.x >> 4;
#pragma unroll
  for (int b = 0; b < TM; ++b)
#pragma unroll
    for (int a = 0; a < TM; ++a) {
      const int r = i * B + dense_rc<T>(ty, a), c = j * B + dense_rc<T>(tx, b);
      if (r < n && c < n) out[(size_t)c * n + r] = (TO)acc[a][b];
    }
}

// ───────────── tensor-core (tcgen05, TF32) product W^T W ─────────────
// One 128 x 128 FP32 output tile per CTA of 128 threads,
//   acc(r, c) = sum_k Aop(r, k) Bop(c, k),
// over K in chunks of kTcKC = 32.  All threads stage a chunk's two operands
// in shared memory (two buffers); thread 0 issues four
// tcgen05.mma.cta_group::1.kind::tf32 (M = N = 128, K = 8) into a 128-column
// TMEM accumulator and commits them to the buffer's mbarrier, which every
// thread waits on (bounded) before it refills that buffer, so staging the
// next chunk overlaps the MMAs of the current one.  Both operands are
// k-contiguous in global memory and staged K-major (tc_stage).  The epilogue
// reads the accumulator row by row (thread t owns row t) and writes
// column-major tiles in coalesced 128-byte column pieces.  The operands are rounded to TF32 (10-bit mantissa) by the
// tensor core; the sums are FP32.  A completion wait that gives up sets
// *info = -1, waits once more (bounded) for the MMAs in flight, frees the
// TMEM columns and returns.
constexpr int kTcKC = 32;
constexpr int kTcOpBytes = 128 * kTcKC * 4;  // one staged operand chunk: 16 KB
constexpr int kTcSmem = 4 * kTcOpBytes;      // two buffers of (A, B)
constexpr int kTcPolls = 1 << 22;

// Stages k0 .. k0 + kTcKC - 1 of a 128-row operand whose element (m, k) is
// at p[m ld + k], in the K-major canonical layout (16-byte k-quads of 8-row
// core matrices, k-quads 128 B apart, 8-row groups 1024 B apart): one 16-byte
// load and one 16-byte store per k-quad; each warp's 32 stores fill four
// 128-byte runs, one per 8-row group, so no bank conflicts.
__device__ __forceinline__ void tc_stage(const float* __restrict__ p, int ld, int k0, unsigned char* s) {
#pragma unroll 2
  for (int q = (int)threadIdx.x; q < 128 * kTcKC / 4; q += 128) {
    const int mr = q & 7, kq = (q >> 3) & 7, m = (q >> 6) * 8 + mr;
    const float4 v = __ldcg(reinterpret_cast<const float4*>(p + (size_t)m * ld + k0 + kq * 4));
    *reinterpret_cast<float4*>(s + (m >> 3) * 1024 + kq * 128 + mr * 16) = v;
  }
}

// Grid nt(nt+1)/2: the lower tile (i, j) of W^T W, (W^T W)_ij =
// sum_{l >= i} W_li^T W_lj, into out (n x n column-major, TO).
template <typename TO>
__global__ void __launch_bounds__(128) dense_syrk_tc_kernel(const float* __restrict__ W, int N, int nt, TO* out,
                                                            int n, int* info) {
  extern __shared__ __align__(1024) unsigned char s_tc[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  constexpr int B = 128;
  const int tid = (int)threadIdx.x, warp = tid >> 5;
  int ti, tj;
  dense_tri((int)blockIdx.x, ti, tj);
  const int nch = (nt - ti) * (B / kTcKC);
  if (warp == 0) umma::tmem_alloc(&tmem_base, 128);
  if (tid == 0) {
    umma::mbar_init(&mbar[0], 1);
    umma::mbar_init(&mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tb = tmem_base;
  constexpr uint32_t idesc = umma::idesc_tf32(128, 128, false, false);
  bool ok = true;
  int issued = 0;
  for (int ch = 0; ch < nch; ++ch) {
    const int b = ch & 1;
    unsigned char* sA = s_tc + b * 2 * kTcOpBytes;
    unsigned char* sB = sA + kTcOpBytes;
    // the MMAs that read this buffer two chunks ago must be done
    if (ch >= 2 && ok) ok = umma::mbar_wait(&mbar[b], (uint32_t)(((ch - 2) >> 1) & 1), kTcPolls);
    const int l = ti + ch / (B / kTcKC), k0 = (ch % (B / kTcKC)) * kTcKC;
    if (ok) {
      tc_stage(W + (size_t)ti * B * N + (size_t)l * B, N, k0, sA);  // W_li(q, r) at [r N + q]
      tc_stage(W + (size_t)tj * B * N + (size_t)l * B, N, k0, sB);  // W_lj(q, c) at [c N + q]
    }
    umma::fence_async_smem();
    umma::fence_before_sync();
    ok = __syncthreads_and(ok) != 0;
    umma::fence_after_sync();
    if (!ok) break;
    if (tid == 0) {
      const uint32_t a0 = umma::smem_u32(sA), b0 = umma::smem_u32(sB);
#pragma unroll
      for (int st = 0; st < kTcKC / 8; ++st) {
        const uint64_t ad = umma::smem_desc_lbo_sbo(a0 + 256 * st, 128, 1024);
        const uint64_t bd = umma::smem_desc_lbo_sbo(b0 + 256 * st, 128, 1024);
        umma::mma_tf32(tb, ad, bd, idesc, (ch > 0 || st > 0) ? 1u : 0u);
      }
      umma::commit(&mbar[b]);
    }
    ++issued;
  }
  if (ok && issued > 0) ok = umma::mbar_wait(&mbar[(issued - 1) & 1], (uint32_t)(((issued - 1) >> 1) & 1), kTcPolls);
  ok = __syncthreads_and(ok) != 0;
  umma::fence_after_sync();
  if (ok) {
    const int r = tid;  // TMEM lane = accumulator row
#pragma unroll 1
    for (int c0 = 0; c0 < B; c0 += 16) {
      float v[16];
      umma::tmem_ld16(umma::taddr(tb, 32 * warp, c0), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int gr = ti * B + r, gc = tj * B + c0 + q;
        if (gr < n && gc < n) out[(size_t)gc * n + gr] = (TO)v[q];
      }
    }
  } else {
    if (tid == 0) atomicExch(info, -1);
    if (issued > 0) umma::drain_mma(&mbar[(issued - 1) & 1], (uint32_t)(((issued - 1) >> 1) & 1), false, kTcPolls);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tb, 128);
}

static inline int dense_nblk(size_t n, int t) { return (int)((n + t - 1) / t); }

int dense_tile(bool fp64) { return fp64 ? DenseCfg<double>::B : DenseCfg<float>::B; }

// TC (FP32 only): the inverse's triangular-inverse and product steps on the
// TF32 tensor-core tile kernel instead of the SIMT one.
template <typename T, typename TO, bool TC = false>
static cudaError_t dense_inverse_t(const double* Ac, int n, T* A, T* W, int* info, TO* out, cudaStream_t s,
                                   int* launches, DenseSched* sched, const int* row_first) {
  constexpr int B = DenseCfg<T>::B;
  const int nt = (n + B - 1) / B, N = nt * B;
  // Envelope: row r of Ac's lower triangle is zero left of row_first[r], and
  // the Cholesky factor's fill stays inside that envelope, so tile (i, k)
  // of L is zero unless first tile column of tile row i <= k.  With the
  // suffix minimum over tile rows (a superset, non-decreasing in i), column
  // k's nonzero tiles are rows k + 1 .. last[k], and every product outside
  // them would add exact zeros: skipping them leaves the result bitwise
  // unchanged.  No row_first: dense (last[k] = nt - 1).
  std::vector<int> last((size_t)nt, nt - 1);
  if (row_first) {
    std::vector<int> fm((size_t)nt);
    for (int i = 0; i < nt; ++i) {
      int f = i;  // the diagonal tile (padding rows: the identity)
      for (int r = i * B; r < std::min(n, (i + 1) * B); ++r) f = std::min(f, std::max(0, row_first[r]) / B);
      fm[i] = f;
    }
    for (int i = nt - 2; i >= 0; --i) fm[i] = std::min(fm[i], fm[i + 1]);
    for (int k = 0, i = 0; k < nt; ++k) {
      while (i + 1 < nt && fm[i + 1] <= k) ++i;
      last[k] = std::max(i, k);
    }
  }
  const size_t diag_smem = sizeof(T) * (2 * (size_t)B * (B + 1) + 32 * 32);
  cudaError_t e = cudaFuncSetAttribute(dense_diag_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)diag_smem);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(info, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  int nl = 0;
  dense_pad_kernel<T><<<dense_nblk((size_t)N * N, 256), 256, 0, s>>>(Ac, n, A, W, N);
  ++nl;
  // W = L^-1 runs right-looking on a second stream, step k as soon as panel k
  // is done (it reads L's column k, W_kk and the rows of W its earlier steps
  // wrote; the trailing update k writes only columns > k), so it overlaps the
  // factorisation's later diagonal and update kernels.  Its products have an
  // inner dimension of one tile (128), too short for the tensor-core
  // kernel's staging to pay (measured slower), so they stay on the SIMT
  // tiles; the product W^T W sums over whole tile columns and runs on the
  // TF32 tensor cores when TC is set.
  //
  // The trailing update looks one step ahead: the main stream updates only
  // tile column k + 1 and goes on to diagonal tile and panel k + 1, while a
  // third stream updates the columns > k + 1 (ordered before the next
  // step's column update by an event), so the single-CTA diagonal kernel
  // overlaps the bulk of the update.  The critical path (diagonal, panel,
  // column update) runs on a stream of the highest priority forked from s,
  // so its CTAs are scheduled ahead of the two bulk streams'.
  DenseSched local;
  DenseSched* sc = sched ? sched : &local;
  if ((e = sc->ensure(nt)) != cudaSuccess) {
    local.release();
    return e;
  }
  cudaStream_t side = sc->side, rest = sc->rest, crit = sc->crit;
  cudaEvent_t* ev = sc->ev.data();
  cudaEvent_t* evr = sc->evr.data();
  cudaEventRecord(ev[nt], s);
  cudaStreamWaitEvent(crit, ev[nt], 0);
  for (int k = 0; k < nt; ++k) {
    dense_diag_kernel<T><<<1, kDenseThreads, diag_smem, crit>>>(A, W, N, k, info);
    ++nl;
    const int m = last[k] - k;  // nonzero tiles below the diagonal in column k
    if (m > 0) {
      dense_panel_kernel<T><<<m, kDenseThreads, 0, crit>>>(A, W, N, k);
      ++nl;
    }
    cudaEventRecord(ev[k], crit);
    cudaStreamWaitEvent(side, ev[k], 0);
    if (k > 0) {
      dense_wfin_kernel<T><<<k, kDenseThreads, 0, side>>>(W, N, k);
      ++nl;
    }
    if (m > 0) {
      dense_wupd_kernel<T><<<m * (k + 1), kDenseThreads, 0, side>>>(A, W, N, k);
      ++nl;
      // columns > k + 1 on the rest stream (after its step k - 1 there)
      cudaStreamWaitEvent(rest, ev[k], 0);
      if (m > 1) {
        dense_update_kernel<T, false><<<(m - 1) * m / 2, kDenseThreads, 0, rest>>>(A, N, k, 1);
        ++nl;
      }
      cudaEventRecord(evr[k], rest);
      // column k + 1 on the main stream, after step k - 1's columns > k
      if (k > 0) cudaStreamWaitEvent(crit, evr[k - 1], 0);
      dense_update_kernel<T, true><<<m, kDenseThreads, 0, crit>>>(A, N, k, 0);
      ++nl;
    }
  }
  // join: s waits for the three streams
  cudaEventRecord(ev[nt], side);
  cudaStreamWaitEvent(s, ev[nt], 0);
  if (nt > 1) cudaStreamWaitEvent(s, evr[nt - 2], 0);
  cudaEventRecord(ev[nt - 1], crit);
  cudaStreamWaitEvent(s, ev[nt - 1], 0);
  if constexpr (TC) {
    static_assert(sizeof(T) == 4 && B == 128, "the tensor-core product takes FP32 128-wide tiles");
    raise_smem_limit_k(dense_syrk_tc_kernel<TO>);
    dense_syrk_tc_kernel<TO><<<nt * (nt + 1) / 2, 128, kTcSmem, s>>>(W, N, nt, out, n, info);
    ++nl;
  } else {
    dense_syrk_kernel<T, TO><<<nt * (nt + 1) / 2, kDenseThreads, 0, s>>>(W, N, nt, out, n);
    ++nl;
  }
  local.release();
  if (launches) *launches += nl;
  return cudaGetLastError();
}

cudaError_t DenseSched::ensure(int nt) {
  cudaError_t e;
  if (!crit) {
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if ((e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&rest, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithPriority(&crit, cudaStreamNonBlocking, prio_hi)) != cudaSuccess)
      return e;
  }
  for (auto* v : {&ev, &evr}) {
    const size_t want = (size_t)nt + (v == &ev ? 1 : 0);
    while (v->size() < want) {
      cudaEvent_t x = nullptr;
      if ((e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming)) != cudaSuccess) return e;
      v->push_back(x);
    }
  }
  return cudaSuccess;
}

void DenseSched::release() {
  for (auto* v : {&ev, &evr}) {
    for (cudaEvent_t x : *v)
      if (x) cudaEventDestroy(x);
    v->clear();
  }
  for (cudaStream_t* x : {&side, &rest, &crit}) {
    if (*x) cudaStreamDestroy(*x);
    *x = nullptr;
  }
}

cudaError_t dense_spd_inverse_f32(const double* Ac, int n, float* A, float* W, int* info, float* out,
                                  cudaStream_t s, int* launches, DenseSched* sched, const int* row_first) {
  return dense_inverse_t<float, float>(Ac, n, A, W, info, out, s, launches, sched, row_first);
}

cudaError_t dense_spd_inverse_tf32(const double* Ac, int n, float* A, float* W, int* info, float* out,
                                   cudaStream_t s, int* launches, DenseSched* sched, const int* row_first) {
  return dense_inverse_t<float, float, true>(Ac, n, A, W, info, out, s, launches, sched, row_first);
}

cudaError_t dense_spd_inverse_f64(const double* Ac, int n, double* A, double* W, int* info, double* out,
                                  cudaStream_t s, int* launches, DenseSched* sched, const int* row_first) {
  return dense_inverse_t<double, double>(Ac, n, A, W, info, out, s, launches, sched, row_first);
}

}  // namespace femb200

using namespace femb200;

static int dense_spd_inverse_c(const double* A, int32_t n, int32_t precision, const int32_t* row_first,
                               double* out, void* stream) {
  if (!A || !out) return set_global_error(FEM_ERR_INVALID, "null matrix");
  if (n < 1 || n > 32768) return set_global_error(FEM_ERR_INVALID, "n = %d not in [1, 32768]", n);
  if (precision != 32 && precision != 64 && precision != 19)
    return set_global_error(FEM_ERR_INVALID, "precision %d: 64, 32 or 19 (TF32 tensor cores)", precision);
  if (row_first)
    for (int r = 0; r < n; ++r)
      if (row_first[r] < 0 || row_first[r] > r)
        return set_global_error(FEM_ERR_INVALID, "row_first[%d] = %d not in [0, %d]", r, row_first[r], r);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool f64 = precision == 64;
  const int B = dense_tile(f64);
  const size_t N = (size_t)((n + B - 1) / B) * B;
  const size_t elem = f64 ? sizeof(double) : sizeof(float);
  void *wa = nullptr, *ww = nullptr;
  int* info = nullptr;
  if (cudaMalloc(&wa, N * N * elem) != cudaSuccess || cudaMalloc(&ww, N * N * elem) != cudaSuccess ||
      cudaMalloc(&info, sizeof(int)) != cudaSuccess) {
    cudaFree(wa);
    cudaFree(ww);
    return set_global_error(FEM_ERR_CUDA, "cudaMalloc of the dense work space (%zu bytes) failed", 2 * N * N * elem);
  }
  cudaError_t e = f64 ? dense_inverse_t<double, double>(A, n, static_cast<double*>(wa), static_cast<double*>(ww),
                                                          info, out, s, nullptr, nullptr, row_first)
                  : precision == 19
                      ? dense_inverse_t<float, double, true>(A, n, static_cast<float*>(wa), static_cast<float*>(ww),
                                                             info, out, s, nullptr, nullptr, row_first)
                      : dense_inverse_t<float, double>(A, n, static_cast<float*>(wa), static_cast<float*>(ww), info,
                                                         out, s, nullptr, nullptr, row_first);
  int h_info = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(wa);
  cudaFree(ww);
  cudaFree(info);
  if (e != cudaSuccess) return set_global_error(FEM_ERR_CUDA, "dense inverse: %s", cudaGetErrorString(e));
  if (h_info < 0) return set_global_error(FEM_ERR_BUDGET, "dense inverse: a tensor-core completion wait timed out");
  if (h_info != 0)
    return set_global_error(FEM_ERR_NAN, "matrix is not positive definite (pivot %d is not positive)", h_info);
  return FEM_OK;
}

extern "C" int fem_dense_spd_inverse(const double* A, int32_t n, int32_t precision, double* out, void* stream) {
  return dense_spd_inverse_c(A, n, precision, nullptr, out, stream);
}

extern "C" int fem_dense_spd_inverse_banded(const double* A, int32_t n, int32_t precision, const int32_t* row_first,
                                            double* out, void* stream) {
  if (!row_first) return set_global_error(FEM_ERR_INVALID, "null row_first");
  return dense_spd_inverse_c(A, n, precision, row_first, out, stream);
}
