// sm_100a kernels of the HEX8 (8-node hexahedron, 2 x 2 x 2 Gauss points)
// static-solve path.
//
// Same two-phase structure as the TET4 tangent matvec: one thread per
// element evaluates all eight Gauss points and writes its eight slot vectors
// at their positions in the node-major slot list (spos), then one pass over
// the nodes adds each node's contiguous slot range in list order.  No
// atomics touch the outputs, so results are bitwise reproducible; this
// replaces the reference's per-Gauss-point ti.atomic_add scatter
// (e.g. backend/fea/fem/material/neo_hookean.py:152-190 with n_gauss = 8).
//
// Geometry is recomputed per Gauss point from the eight vertices
// (core/mesh.py:123-151, 240-291): J = sum_a X_a (x) dN_a/dxi,
// dN/dX = dN/dxi J^-1, volume |det J| (weight 1).  Vertex coordinates are
// taken relative to vertex 0 (J is unchanged because sum_a dN_a/dxi = 0),
// which keeps the FP32 tangent's Jacobian free of the absolute position.
#include <cuda_runtime.h>

#include "fem_internal.h"
#include "fem_lattice.cuh"
#include "fem_reduce.cuh"

namespace femb200 {

namespace {

constexpr double kGaussHex = 0.5773502691896257;  // 1 / sqrt(3), core/mesh.py:184

// sign of natural coordinate d (0 xi, 1 eta, 2 zeta) of vertex / Gauss point
// a in the reference's ordering (core/element.py:297-315, core/mesh.py:186-200)
__host__ __device__ constexpr int hex_sign(int a, int d) {
  return d == 0 ? (((a ^ (a >> 1)) & 1) ? 1 : -1) : (d == 1 ? (((a >> 1) & 1) ? 1 : -1) : (((a >> 2) & 1) ? 1 : -1));
}

// dN/dX (8 x 3) and |det J| at Gauss point g of a hexahedron with vertex
// coordinates xr (relative to vertex 0).
template <typename T>
__device__ __forceinline__ void hex_point(const T xr[8][3], int g, T dN[8][3], T& vol) {
  const T gx = T(hex_sign(g, 0)) * T(kGaussHex);
  const T gy = T(hex_sign(g, 1)) * T(kGaussHex);
  const T gz = T(hex_sign(g, 2)) * T(kGaussHex);
  T J[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) J[i][j] = T(0);
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const T sx = T(hex_sign(a, 0)), sy = T(hex_sign(a, 1)), sz = T(hex_sign(a, 2));
    const T fx = T(1) + sx * gx, fy = T(1) + sy * gy, fz = T(1) + sz * gz;
    dN[a][0] = T(0.125) * sx * fy * fz;
    dN[a][1] = T(0.125) * fx * sy * fz;
    dN[a][2] = T(0.125) * fx * fy * sz;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) J[i][j] += xr[a][i] * dN[a][j];
  }
  // J^-1 by cofactors
  const T c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const T c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const T c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const T det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const T id = T(1) / det;
  T Ji[3][3];
  Ji[0][0] = c00 * id;
  Ji[1][0] = c01 * id;
  Ji[2][0] = c02 * id;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  vol = det < T(0) ? -det : det;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const T d0 = dN[a][0], d1 = dN[a][1], d2 = dN[a][2];
#pragma unroll
    for (int j = 0; j < 3; ++j) dN[a][j] = d0 * Ji[0][j] + d1 * Ji[1][j] + d2 * Ji[2][j];
  }
}

__device__ __forceinline__ void hex_nodes(const MeshDev& m, int e, int nid[8]) {
  const int4 c0 = __ldg(m.conn + 2 * e), c1 = __ldg(m.conn + 2 * e + 1);
  nid[0] = c0.x; nid[1] = c0.y; nid[2] = c0.z; nid[3] = c0.w;
  nid[4] = c1.x; nid[5] = c1.y; nid[6] = c1.z; nid[7] = c1.w;
}

__device__ __forceinline__ void hex_slots(const MeshDev& m, int e, int pos[8]) {
  const int4 s0 = __ldg(m.spos + 2 * e), s1 = __ldg(m.spos + 2 * e + 1);
  pos[0] = s0.x; pos[1] = s0.y; pos[2] = s0.z; pos[3] = s0.w;
  pos[4] = s1.x; pos[5] = s1.y; pos[6] = s1.z; pos[7] = s1.w;
}

// G_ij = sum_a v_a[i] dN_a[j]
template <typename T>
__device__ __forceinline__ void hex_grad(const T v[8][3], const T dN[8][3], T G[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      T s = T(0);
#pragma unroll
      for (int a = 0; a < 8; ++a) s += v[a][i] * dN[a][j];
      G[3 * i + j] = s;
    }
}

// f_a[i] += coef * sum_j S_ij dN_a[j]
template <typename T>
__device__ __forceinline__ void hex_add_slots(const T S[9], const T dN[8][3], T coef, T f[8][3]) {
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      f[a][i] += coef * (S[3 * i] * dN[a][0] + S[3 * i + 1] * dN[a][1] + S[3 * i + 2] * dN[a][2]);
}

// Trilinear form of a vertex field v: v(xi) = c_1 + sum_m C_m m(xi) over the
// monomials m = xi, eta, zeta, xi eta, eta zeta, xi zeta, xi eta zeta, with
// C_m = 1/8 sum_a sigma_a^m v_a (sigma_a^m: the product of vertex a's signs
// in the monomial's coordinates).  Its natural-coordinate gradient at a
// point then costs 4 terms per entry instead of 8 vertex products, and the
// vertex forces f_a = sum_j T_j dN_a/dxi_j of a point's stress-like tensor T
// are 1/8 sum_m sigma_a^m A_m over 7 accumulated moments A_m.
__host__ __device__ constexpr int hex_msign(int a, int m) {
  return m < 3 ? hex_sign(a, m)
               : (m == 3 ? hex_sign(a, 0) * hex_sign(a, 1)
                         : (m == 4 ? hex_sign(a, 1) * hex_sign(a, 2)
                                   : (m == 5 ? hex_sign(a, 0) * hex_sign(a, 2)
                                             : hex_sign(a, 0) * hex_sign(a, 1) * hex_sign(a, 2))));
}

template <typename T>
__device__ __forceinline__ void hex_coeffs(const T v[8][3], T C[7][3]) {
#pragma unroll
  for (int m = 0; m < 7; ++m)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T s = T(0);
#pragma unroll
      for (int a = 0; a < 8; ++a) s += hex_msign(a, m) > 0 ? v[a][d] : -v[a][d];
      C[m][d] = T(0.125) * s;
    }
}

// G[i][j] = d v_i / d xi_j at (gx, gy, gz) from the coefficients
template <typename T>
__device__ __forceinline__ void hex_nat_grad(const T C[7][3], T gx, T gy, T gz, T G[3][3]) {
  const T yz = gy * gz, xz = gx * gz, xy = gx * gy;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    G[i][0] = C[0][i] + C[3][i] * gy + C[5][i] * gz + C[6][i] * yz;
    G[i][1] = C[1][i] + C[3][i] * gx + C[4][i] * gz + C[6][i] * xz;
    G[i][2] = C[2][i] + C[4][i] * gy + C[5][i] * gx + C[6][i] * xy;
  }
}

// J^-1 by cofactors and |det J|
template <typename T>
__device__ __forceinline__ void hex_inv(const T J[3][3], T Ji[3][3], T& vol) {
  const T c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const T c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const T c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const T det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const T id = T(1) / det;
  Ji[0][0] = c00 * id;
  Ji[1][0] = c01 * id;
  Ji[2][0] = c02 * id;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  vol = det < T(0) ? -det : det;
}

// A_m += moments of T_ij = coef sum_k S_ik Ji_jk (the point's contribution
// f_a = coef S dN_a, with dN_a = J^-T dN_a/dxi)
template <typename T>
__device__ __forceinline__ void hex_moments(const T S[9], const T Ji[3][3], T coef, T gx, T gy, T gz, T A[7][3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    T t[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) t[j] = coef * (S[3 * i] * Ji[j][0] + S[3 * i + 1] * Ji[j][1] + S[3 * i + 2] * Ji[j][2]);
    A[0][i] += t[0];
    A[1][i] += t[1];
    A[2][i] += t[2];
    A[3][i] += t[0] * gy + t[1] * gx;
    A[4][i] += t[1] * gz + t[2] * gy;
    A[5][i] += t[0] * gz + t[2] * gx;
    A[6][i] += t[0] * (gy * gz) + t[1] * (gx * gz) + t[2] * (gx * gy);
  }
}

// vertex a's vector 1/8 sum_m sigma_a^m A_m (a a constant after unrolling)
template <typename T>
__device__ __forceinline__ void hex_vertex(const T A[7][3], int a, T f[3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    T s = T(0);
#pragma unroll
    for (int mm = 0; mm < 7; ++mm) s += hex_msign(a, mm) > 0 ? A[mm][i] : -A[mm][i];
    f[i] = T(0.125) * s;
  }
}

// ───────────────────────── residual (FP64) ─────────────────────────

template <int MODEL>
__global__ void __launch_bounds__(128) hex_res_elem_kernel(const __grid_constant__ ResArgs a) {
  const MeshDev& m = a.m;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n_elems) return;
  const size_t Ne = (size_t)m.n_elems, Nq = kHexGauss * Ne;
  int nid[8];
  hex_nodes(m, e, nid);
  double cx[7][3], cu[7][3];
  {
    double xr[8][3], uv[8][3];
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        xr[k][d] = __ldg(m.X64 + 3 * nid[k] + d);
        uv[k][d] = __ldg(a.u + 3 * nid[k] + d);
      }
    hex_coeffs(xr, cx);   // the monomial coefficients do not see the position
    hex_coeffs(uv, cu);
  }
  const DevMat<double>& mat = a.matD[__ldg(m.mat_id + e)];
  const double scale = (double)__ldg(m.scale + e);
  const int model = MODEL >= 0 ? MODEL : mat.model;
  const int npay = model_pay_words(model);
  double A[7][3];
#pragma unroll
  for (int k = 0; k < 7; ++k) A[k][0] = A[k][1] = A[k][2] = 0.0;
#pragma unroll 1
  for (int g = 0; g < kHexGauss; ++g) {
    const size_t q = (size_t)g * Ne + e;
    const double gx = hex_sign(g, 0) * kGaussHex, gy = hex_sign(g, 1) * kGaussHex, gz = hex_sign(g, 2) * kGaussHex;
    double J[3][3], Gu[3][3], Ji[3][3], vol;
    hex_nat_grad(cx, gx, gy, gz, J);
    hex_nat_grad(cu, gx, gy, gz, Gu);
    hex_inv(J, Ji, vol);
    double Hg[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int k = 0; k < 3; ++k) Hg[3 * i + k] = Gu[i][0] * Ji[0][k] + Gu[i][1] * Ji[1][k] + Gu[i][2] * Ji[2][k];
    double S[9];
    float pay[kPay];
    if (model == M_NH) {
      nh_stress(mat, scale, Hg, S, pay);
    } else if (model == M_MR || model == M_FMR) {
      mr_stress(mat, scale, Hg, S, pay);
    } else if (model == M_J2) {
      double ep[6], epn[6], epe_n;
#pragma unroll
      for (int k = 0; k < 6; ++k) ep[k] = a.ep_c[(size_t)k * Nq + q];
      j2_stress(mat, scale, Hg, ep, a.epe_c[q], S, epn, epe_n, pay);
#pragma unroll
      for (int k = 0; k < 6; ++k) a.ep_t[(size_t)k * Nq + q] = epn[k];
      a.epe_t[q] = epe_n;
    } else if (model == M_TI) {
      ti_stress(mat, scale, Hg, S);
    } else {
      le_stress(mat, scale, Hg, S);
    }
#pragma unroll
    for (int k = 0; k < kPay; ++k)
      if (k < npay) a.payload[(size_t)k * Nq + q] = pay[k];
    hex_moments(S, Ji, -vol, gx, gy, gz, A);
  }
  int pos[8];
  hex_slots(m, e, pos);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double f[3];
    hex_vertex(A, k, f);
#pragma unroll
    for (int d = 0; d < 3; ++d) a.stage_d[3 * (size_t)pos[k] + d] = f[d];
  }
}

__global__ void __launch_bounds__(256) hex_res_gather_kernel(const __grid_constant__ ResArgs a) {
  __shared__ double sred[8];
  __shared__ bool am_last;
  const MeshDev& m = a.m;
  const int n = blockIdx.x * 256 + threadIdx.x;
  double r2 = 0.0;
  if (n < m.n_nodes) {
    double acc[3] = {0.0, 0.0, 0.0};
    const int j0 = __ldg(m.node_row + n), j1 = __ldg(m.node_row + n + 1);
    for (int j = j0; j < j1; ++j)
#pragma unroll
      for (int d = 0; d < 3; ++d) acc[d] += a.stage_d[3 * (size_t)j + d];
    const uint8_t fx = m.fixed[n];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (a.fneg) a.fneg[3 * n + d] = acc[d];
      const double r = ((fx >> d) & 1) ? 0.0 : a.f_ext[3 * n + d] + acc[d];
      a.R[3 * n + d] = r;
      r2 += r * r;
    }
  }
  double bsum = block_sum<256>(r2, sred);
  if (publish_partial(a.red, a.red_site, 1, &bsum, &am_last)) {
    double tot = final_sum<256>(a.red, a.red_site, 0, sred);
    if (threadIdx.x == 0) {
      *a.rnorm2 = tot;
      a.red.counters[a.red_site] = 0u;
    }
  }
}

// ───────────────────────── tangent matvec (FP32) ─────────────────────────

// Tangent action of one hexahedron in the trilinear basis: per point,
// J and the natural gradient of p from the coefficients, dF = G_p J^-1,
// T = |det J| dP J^-T, and T is accumulated into the 7 monomial moments A;
// the vertex vectors f_a = 1/8 sum_m sigma_a^m A_m are formed once.
template <int MODEL, bool CG, bool MASK>
__device__ __forceinline__ void hex_mv_one(const MvArgs& a, int e) {
  const MeshDev& m = a.m;
  const size_t Ne = (size_t)m.n_elems, Nq = kHexGauss * Ne;
  int nid[8];
  hex_nodes(m, e, nid);
  const float4* __restrict__ xin = reinterpret_cast<const float4*>(a.x);
  float cx[7][3], cp[7][3];
  {
    float xr[8][3], pv[8][3];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float4 X = __ldg(m.X32 + nid[k]);
      const float4 P = __ldg(xin + nid[k]);
      xr[k][0] = X.x;
      xr[k][1] = X.y;
      xr[k][2] = X.z;
      const int fx = MASK ? (int)X.w : 0;
      pv[k][0] = (fx & 1) ? 0.f : P.x;
      pv[k][1] = (fx & 2) ? 0.f : P.y;
      pv[k][2] = (fx & 4) ? 0.f : P.z;
    }
#pragma unroll
    for (int k = 7; k >= 0; --k)
#pragma unroll
      for (int d = 0; d < 3; ++d) xr[k][d] -= xr[0][d];
    hex_coeffs(xr, cx);
    hex_coeffs(pv, cp);
  }
  const DevMat<float>& mat = a.matF[__ldg(m.mat_id + e)];
  const float scale = __ldg(m.scale + e);
  const int npay = model_pay_words(MODEL >= 0 ? MODEL : mat.model);
  float A[7][3];
#pragma unroll
  for (int k = 0; k < 7; ++k) A[k][0] = A[k][1] = A[k][2] = 0.f;
#pragma unroll 1
  for (int g = 0; g < kHexGauss; ++g) {
    const size_t q = (size_t)g * Ne + e;
    float pay[kPay];
#pragma unroll
    for (int k = 0; k < kPay; ++k) pay[k] = (k < npay) ? __ldg(a.payload + (size_t)k * Nq + q) : 0.f;
    const float gx = (float)hex_sign(g, 0) * (float)kGaussHex;
    const float gy = (float)hex_sign(g, 1) * (float)kGaussHex;
    const float gz = (float)hex_sign(g, 2) * (float)kGaussHex;
    float J[3][3], Gp[3][3], Ji[3][3], vol;
    hex_nat_grad(cx, gx, gy, gz, J);
    hex_nat_grad(cp, gx, gy, gz, Gp);
    hex_inv(J, Ji, vol);
    float dF[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int k = 0; k < 3; ++k) dF[3 * i + k] = Gp[i][0] * Ji[0][k] + Gp[i][1] * Ji[1][k] + Gp[i][2] * Ji[2][k];
    float dP[9];
    dP_any<MODEL>(mat, scale, pay, dF, dP);
    hex_moments(dP, Ji, vol, gx, gy, gz, A);
  }
  int pos[8];
  hex_slots(m, e, pos);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    float f[3];
    hex_vertex(A, k, f);
    __stcg(a.stage + pos[k], make_float4(f[0], f[1], f[2], 0.f));
  }
}

// 5 CTAs per SM (96 registers, a few spilled words) instead of 4 (120):
// 105 -> 98 us at n = 96, unchanged at n = 64
template <int MODEL, bool CG>
__global__ void __launch_bounds__(128, 5) hex_mv_elem_kernel(const __grid_constant__ MvArgs a) {
  chain_enter();
  if (CG) {
    if (a.cg->done) return;
  }
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.m.n_elems) return;
  if (!CG && a.mask_input)
    hex_mv_one<MODEL, CG, true>(a, e);
  else
    hex_mv_one<MODEL, CG, false>(a, e);
}

// ───────────────────────── Jacobi diagonal (FP32) ─────────────────────────

template <int MODEL, bool BLOCK>
__global__ void __launch_bounds__(128) hex_diag_elem_kernel(const __grid_constant__ DiagArgs a) {
  constexpr int W = BLOCK ? 6 : 3;
  const MeshDev& m = a.m;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n_elems) return;
  const size_t Ne = (size_t)m.n_elems, Nq = kHexGauss * Ne;
  int nid[8];
  hex_nodes(m, e, nid);
  float xr[8][3];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const float4 X = __ldg(m.X32 + nid[k]);
    xr[k][0] = X.x;
    xr[k][1] = X.y;
    xr[k][2] = X.z;
  }
#pragma unroll
  for (int k = 7; k >= 0; --k)
#pragma unroll
    for (int d = 0; d < 3; ++d) xr[k][d] -= xr[0][d];
  const DevMat<float>& mat = a.matF[__ldg(m.mat_id + e)];
  const float scale = __ldg(m.scale + e);
  const int npay = model_pay_words(MODEL >= 0 ? MODEL : mat.model);
  float acc[8][W];
#pragma unroll
  for (int s = 0; s < 8; ++s)
#pragma unroll
    for (int k = 0; k < W; ++k) acc[s][k] = 0.f;
#pragma unroll 1
  for (int g = 0; g < kHexGauss; ++g) {
    const size_t q = (size_t)g * Ne + e;
    float dN[8][3], vol;
    hex_point(xr, g, dN, vol);
    float pay[kPay];
#pragma unroll
    for (int k = 0; k < kPay; ++k) pay[k] = (k < npay) ? __ldg(a.payload + (size_t)k * Nq + q) : 0.f;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        // force at the slot's node for a unit displacement of it in direction i
        float dF[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) dF[k] = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) dF[3 * i + j] = dN[s][j];
        float dP[9];
        dP_any<MODEL>(mat, scale, pay, dF, dP);
        if (BLOCK) {
#pragma unroll
          for (int k = i; k < 3; ++k) {
            const int ent = (i == 0) ? k : (i == 1 ? 2 + k : 5);
            acc[s][ent] += vol * (dP[3 * k] * dN[s][0] + dP[3 * k + 1] * dN[s][1] + dP[3 * k + 2] * dN[s][2]);
          }
        } else {
          acc[s][i] += vol * (dP[3 * i] * dN[s][0] + dP[3 * i + 1] * dN[s][1] + dP[3 * i + 2] * dN[s][2]);
        }
      }
    }
  }
  int pos[8];
  hex_slots(m, e, pos);
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    a.stage[2 * (size_t)pos[s]] = make_float4(acc[s][0], acc[s][1], acc[s][2], BLOCK ? acc[s][W - 3] : 0.f);
    if (BLOCK) a.stage[2 * (size_t)pos[s] + 1] = make_float4(acc[s][W - 2], acc[s][W - 1], 0.f, 0.f);
  }
}

template <bool BLOCK>
__global__ void __launch_bounds__(256) hex_diag_gather_kernel(const __grid_constant__ DiagArgs a) {
  const MeshDev& m = a.m;
  const int n = blockIdx.x * 256 + threadIdx.x;
  if (n >= m.n_nodes) return;
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const int j0 = __ldg(m.node_row + n), j1 = __ldg(m.node_row + n + 1);
  for (int j = j0; j < j1; ++j) {
    const float4 v = a.stage[2 * (size_t)j];
    acc[0] += v.x;
    acc[1] += v.y;
    acc[2] += v.z;
    if (BLOCK) {
      const float4 w = a.stage[2 * (size_t)j + 1];
      acc[3] += v.w;
      acc[4] += w.x;
      acc[5] += w.y;
    }
  }
  diag_store<BLOCK>(acc, m.fixed[n], n, a.dinv, a.boff);
}

// ───────────────────────── per-point outputs (FP64) ─────────────────────────

template <int MODEL>
__global__ void hex_stress_kernel(const MeshDev m, const DevMat<double>* matD, const double* u,
                                  const double* ep_c, const double* epe_c, const int* perm_elem,
                                  double* F_out, double* sig_out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n_elems) return;
  const size_t Ne = (size_t)m.n_elems, Nq = kHexGauss * Ne;
  int nid[8];
  hex_nodes(m, e, nid);
  double xr[8][3], uv[8][3];
  for (int k = 0; k < 8; ++k)
    for (int d = 0; d < 3; ++d) {
      xr[k][d] = m.X64[3 * nid[k] + d];
      uv[k][d] = u[3 * nid[k] + d];
    }
  for (int k = 7; k >= 0; --k)
    for (int d = 0; d < 3; ++d) xr[k][d] -= xr[0][d];
  const DevMat<double>& mat = matD[m.mat_id[e]];
  const double scale = (double)m.scale[e];
  const int model = MODEL >= 0 ? MODEL : mat.model;
  const int eu = perm_elem[e];
  for (int g = 0; g < kHexGauss; ++g) {
    const size_t q = (size_t)g * Ne + e;
    double dN[8][3], vol;
    hex_point(xr, g, dN, vol);
    double Hg[9], F[9];
    hex_grad(uv, dN, Hg);
    for (int k = 0; k < 9; ++k) F[k] = Hg[k] + ((k % 4 == 0) ? 1.0 : 0.0);
    double sig[9];
    float pay[kPay];
    if (model == M_NH || model == M_MR || model == M_FMR) {
      // Cauchy stress sigma = P F^T / J_s, as the TET4 stress output
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
      for (int k = 0; k < 6; ++k) ep[k] = ep_c[(size_t)k * Nq + q];
      j2_stress(mat, scale, Hg, ep, epe_c[q], sig, epn, epe_n, pay);
    } else if (model == M_TI) {
      ti_stress(mat, scale, Hg, sig);
    } else {
      le_stress(mat, scale, Hg, sig);
    }
    // caller layout: point e * 8 + g (the reference's gp_idx)
    const size_t o = (size_t)9 * ((size_t)eu * kHexGauss + g);
    for (int k = 0; k < 9; ++k) {
      if (F_out) F_out[o + k] = F[k];
      if (sig_out) sig_out[o + k] = sig[k];
    }
  }
}

__global__ void hex_refq_kernel(const MeshDev m, const int* perm_elem, double* dNdX, double* vol) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n_elems) return;
  int nid[8];
  hex_nodes(m, e, nid);
  double xr[8][3];
  for (int k = 0; k < 8; ++k)
    for (int d = 0; d < 3; ++d) xr[k][d] = m.X64[3 * nid[k] + d];
  for (int k = 7; k >= 0; --k)
    for (int d = 0; d < 3; ++d) xr[k][d] -= xr[0][d];
  const size_t eu = (size_t)perm_elem[e];
  for (int g = 0; g < kHexGauss; ++g) {
    double dN[8][3], v;
    hex_point(xr, g, dN, v);
    const size_t q = eu * kHexGauss + g;
    if (dNdX)
      for (int a = 0; a < 8; ++a)
        for (int j = 0; j < 3; ++j) dNdX[q * 24 + 3 * a + j] = dN[a][j];
    if (vol) vol[q] = v;
  }
}

// ───────────────────────── two-level coarse operator ─────────────────────────
// Galerkin block of a lattice cell, W^T K_e W summed over the cell's
// elements (W: the trilinear weights of the element's vertices in the cell;
// fixed rows and columns of K_e zeroed), as the TET4 cell kernel, here one
// warp per element: lane l < 24 forms column l = 3 c2 + d2 of K_e W as the
// element's tangent action on the field w_b(c2) e_d2 and contracts it with
// W for the 24 rows.  Each warp keeps its share of the cell's 24 x 24 block
// in registers (element order, FP32 products, FP64 accumulation) and writes
// it to its own slot; the dense kernel adds the slots in order.
constexpr int kHexCellCtas = 8;   // CTAs per cell (4 warps each): 32 block shares

template <int MODEL>
__global__ void __launch_bounds__(128) coarse_cell_hex_kernel(const __grid_constant__ CoarseArgs a) {
  __shared__ float sW[4][64];     // per warp: W[vertex][corner]
  __shared__ int sfx[4][8];
  const MeshDev& m = a.m;
  const CoarseDev& c = a.c;
  const int cell = blockIdx.x / kHexCellCtas;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nsl = kHexCellCtas * 4;
  const int slice = (blockIdx.x - cell * kHexCellCtas) * 4 + warp;
  const int3 ijk = c.cell_ijk[cell];
  const int e0 = c.cell_elem_ptr[cell], e1 = c.cell_elem_ptr[cell + 1];
  const size_t Ne = (size_t)m.n_elems, Nq = kHexGauss * Ne;
  const int c2 = lane / 3, d2 = lane - 3 * (lane / 3);
  double acc[24];
#pragma unroll
  for (int r = 0; r < 24; ++r) acc[r] = 0.0;
  for (int idx = e0 + slice; idx < e1; idx += nsl) {
    const int e = __ldg(c.cell_elems + idx);
    int nid[8];
    hex_nodes(m, e, nid);
    __syncwarp();
    if (lane < 8) {
      const float4 X = __ldg(m.X32 + nid[lane]);
      float t[3];
      cell_local(c, ijk, X.x, X.y, X.z, t);
#pragma unroll
      for (int q = 0; q < 8; ++q) sW[warp][lane * 8 + q] = tri_weight(t[0], t[1], t[2], q);
      sfx[warp][lane] = (int)m.fixed[nid[lane]];
    }
    __syncwarp();
    if (lane < 24) {
      float xr[8][3], wcol[8], f[8][3];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float4 X = __ldg(m.X32 + nid[k]);
        xr[k][0] = X.x;
        xr[k][1] = X.y;
        xr[k][2] = X.z;
        wcol[k] = ((sfx[warp][k] >> d2) & 1) ? 0.f : sW[warp][k * 8 + c2];
        f[k][0] = f[k][1] = f[k][2] = 0.f;
      }
#pragma unroll
      for (int k = 7; k >= 0; --k)
#pragma unroll
        for (int d = 0; d < 3; ++d) xr[k][d] -= xr[0][d];
      const DevMat<float>& mat = a.matF[__ldg(m.mat_id + e)];
      const float scale = __ldg(m.scale + e);
      const int npay = model_pay_words(MODEL >= 0 ? MODEL : mat.model);
#pragma unroll 1
      for (int g = 0; g < kHexGauss; ++g) {
        const size_t q = (size_t)g * Ne + e;
        float dN[8][3], vol;
        hex_point(xr, g, dN, vol);
        float dF[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) dF[k] = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          float s = 0.f;
#pragma unroll
          for (int b = 0; b < 8; ++b) s += wcol[b] * dN[b][j];
          dF[3 * d2 + j] = s;
        }
        float pay[kPay];
#pragma unroll
        for (int k = 0; k < kPay; ++k) pay[k] = (k < npay) ? __ldg(a.payload + (size_t)k * Nq + q) : 0.f;
        float dP[9];
        dP_any<MODEL>(mat, scale, pay, dF, dP);
        hex_add_slots(dP, dN, vol, f);
      }
#pragma unroll
      for (int r = 0; r < 24; ++r) {
        const int c1 = r / 3, d1 = r - 3 * (r / 3);
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (!((sfx[warp][k] >> d1) & 1)) s += sW[warp][k * 8 + c1] * f[k][d1];
        acc[r] += (double)s;
      }
    }
  }
  if (lane < 24) {
    double* out = c.blocks + ((size_t)cell * nsl + slice) * 576;
#pragma unroll
    for (int r = 0; r < 24; ++r) out[r * 24 + lane] = acc[r];
  }
}

inline int nblk(int n, int t) { return (n + t - 1) / t; }

}  // namespace

void launch_coarse_cells_hex(const CoarseArgs& a, int model, cudaStream_t s) {
  const int g = a.c.n_cells * kHexCellCtas;
  switch (model) {
    case M_LE: coarse_cell_hex_kernel<M_LE><<<g, 128, 0, s>>>(a); break;
    case M_NH: coarse_cell_hex_kernel<M_NH><<<g, 128, 0, s>>>(a); break;
    case M_MR: coarse_cell_hex_kernel<M_MR><<<g, 128, 0, s>>>(a); break;
    case M_J2: coarse_cell_hex_kernel<M_J2><<<g, 128, 0, s>>>(a); break;
    case M_TI: coarse_cell_hex_kernel<M_TI><<<g, 128, 0, s>>>(a); break;
    case M_FMR: coarse_cell_hex_kernel<M_FMR><<<g, 128, 0, s>>>(a); break;
    default: coarse_cell_hex_kernel<-1><<<g, 128, 0, s>>>(a); break;
  }
}

void launch_residual_hex(const ResArgs& a, int model, cudaStream_t s) {
  const int ge = nblk(a.m.n_elems, 128);
  switch (model) {
    case M_LE: hex_res_elem_kernel<M_LE><<<ge, 128, 0, s>>>(a); break;
    case M_NH: hex_res_elem_kernel<M_NH><<<ge, 128, 0, s>>>(a); break;
    case M_MR: hex_res_elem_kernel<M_MR><<<ge, 128, 0, s>>>(a); break;
    case M_J2: hex_res_elem_kernel<M_J2><<<ge, 128, 0, s>>>(a); break;
    case M_TI: hex_res_elem_kernel<M_TI><<<ge, 128, 0, s>>>(a); break;
    case M_FMR: hex_res_elem_kernel<M_FMR><<<ge, 128, 0, s>>>(a); break;
    default: hex_res_elem_kernel<-1><<<ge, 128, 0, s>>>(a); break;
  }
  hex_res_gather_kernel<<<nblk(a.m.n_nodes, 256), 256, 0, s>>>(a);
}

template <bool CG>
static void hex_mv(const MvArgs& a, int model, cudaStream_t s) {
  const int ge = nblk(a.m.n_elems, 128);
  switch (model) {
    case M_LE: launch_chain(hex_mv_elem_kernel<M_LE, CG>, ge, 128, 0, s, a); break;
    case M_NH: launch_chain(hex_mv_elem_kernel<M_NH, CG>, ge, 128, 0, s, a); break;
    case M_MR: launch_chain(hex_mv_elem_kernel<M_MR, CG>, ge, 128, 0, s, a); break;
    case M_J2: launch_chain(hex_mv_elem_kernel<M_J2, CG>, ge, 128, 0, s, a); break;
    case M_TI: launch_chain(hex_mv_elem_kernel<M_TI, CG>, ge, 128, 0, s, a); break;
    case M_FMR: launch_chain(hex_mv_elem_kernel<M_FMR, CG>, ge, 128, 0, s, a); break;
    default: launch_chain(hex_mv_elem_kernel<-1, CG>, ge, 128, 0, s, a); break;
  }
  launch_node_gather(a, s);
}

void launch_matvec_hex(const MvArgs& a, int model, cudaStream_t s) {
  a.cg != nullptr ? hex_mv<true>(a, model, s) : hex_mv<false>(a, model, s);
}

template <bool BLOCK>
static void hex_diag(const DiagArgs& a, int model, cudaStream_t s) {
  const int ge = nblk(a.m.n_elems, 128);
  switch (model) {
    case M_LE: hex_diag_elem_kernel<M_LE, BLOCK><<<ge, 128, 0, s>>>(a); break;
    case M_NH: hex_diag_elem_kernel<M_NH, BLOCK><<<ge, 128, 0, s>>>(a); break;
    case M_MR: hex_diag_elem_kernel<M_MR, BLOCK><<<ge, 128, 0, s>>>(a); break;
    case M_J2: hex_diag_elem_kernel<M_J2, BLOCK><<<ge, 128, 0, s>>>(a); break;
    case M_TI: hex_diag_elem_kernel<M_TI, BLOCK><<<ge, 128, 0, s>>>(a); break;
    case M_FMR: hex_diag_elem_kernel<M_FMR, BLOCK><<<ge, 128, 0, s>>>(a); break;
    default: hex_diag_elem_kernel<-1, BLOCK><<<ge, 128, 0, s>>>(a); break;
  }
  hex_diag_gather_kernel<BLOCK><<<nblk(a.m.n_nodes, 256), 256, 0, s>>>(a);
}

void launch_diag_hex(const DiagArgs& a, int model, cudaStream_t s) {
  a.boff ? hex_diag<true>(a, model, s) : hex_diag<false>(a, model, s);
}

void launch_stress_hex(const MeshDev& m, const DevMat<double>* matD, int model, const double* u,
                       const double* ep_c, const double* epe_c, const int* perm_elem, double* F_out,
                       double* sig_out, cudaStream_t s) {
  const int t = 128, gb = nblk(m.n_elems, t);
  switch (model) {
    case M_LE: hex_stress_kernel<M_LE><<<gb, t, 0, s>>>(m, matD, u, ep_c, epe_c, perm_elem, F_out, sig_out); break;
    case M_NH: hex_stress_kernel<M_NH><<<gb, t, 0, s>>>(m, matD, u, ep_c, epe_c, perm_elem, F_out, sig_out); break;
    case M_J2: hex_stress_kernel<M_J2><<<gb, t, 0, s>>>(m, matD, u, ep_c, epe_c, perm_elem, F_out, sig_out); break;
    default: hex_stress_kernel<-1><<<gb, t, 0, s>>>(m, matD, u, ep_c, epe_c, perm_elem, F_out, sig_out); break;
  }
}

void launch_refq_hex(const MeshDev& m, const int* perm_elem, double* dNdX, double* vol, cudaStream_t s) {
  hex_refq_kernel<<<nblk(m.n_elems, 128), 128, 0, s>>>(m, perm_elem, dNdX, vol);
}

}  // namespace femb200
