// Device-side element math for the TET4 static-solve path.
//
// Geometry: for a tet with vertices x0..x3 the edge matrix J has columns
// d_k = x_k - x0, J^-1 has rows c_k / det with c_1 = d2 x d3, c_2 = d3 x d1,
// c_3 = d1 x d2, so dN_k/dX = c_k / det (k = 1..3) and dN_0/dX = -sum.  The
// Gauss volume is |det|/6 (one-point rule, core/mesh.py:123-151), hence
// vol * dN_k = sign(det) c_k / 6 needs no division.
//
// Stress measures follow the reference force kernels: large-strain models
// contract P = J_s sigma F^-T with dN (neo_hookean.py:152-190,
// mooney_rivlin.py:212-250), small-strain models contract sigma itself
// (linear_elastic.py:142-173, j2_plasticity.py:366-393,
// transverse_isotropic.py:366-393).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace femb200 {

constexpr int kPay = 10;          // float words of tangent state per element
constexpr double kJFloor = 1e-8;  // J_safe clamp (neo_hookean.py:119)

enum Model : int {
  M_LE = 0, M_NH = 1, M_MR = 2, M_J2 = 3, M_TI = 4, M_FMR = 5
};

// Material entry, all moduli per unit element scale.
template <typename T>
struct DevMat {
  int model;
  int n_fibers;
  T mu, lam, kappa;     // LE / NH / J2
  T sigma_y, H;         // J2
  T C10, C01, invD1;    // MR, fibre MR (invD1 = 0 disables the volumetric term)
  T fE;                 // fibre stiffness
  T fa[6];              // fibre directions
  T C[36];              // TI global Voigt stiffness
};

template <typename T> __device__ __forceinline__ T dev_log(T x);
template <> __device__ __forceinline__ double dev_log<double>(double x) { return log(x); }
template <> __device__ __forceinline__ float dev_log<float>(float x) { return logf(x); }

template <typename T>
__device__ __forceinline__ void cross3(const T a[3], const T b[3], T c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

template <typename T>
__device__ __forceinline__ T det3(const T A[9]) {
  return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
         A[2] * (A[3] * A[7] - A[4] * A[6]);
}

// Ainv = A^-1 (unguarded, as the reference's F.inverse()); returns det.
template <typename T>
__device__ __forceinline__ T inv3(const T A[9], T Ai[9]) {
  T c00 = A[4] * A[8] - A[5] * A[7];
  T c01 = A[5] * A[6] - A[3] * A[8];
  T c02 = A[3] * A[7] - A[4] * A[6];
  T det = A[0] * c00 + A[1] * c01 + A[2] * c02;
  T id = T(1) / det;
  Ai[0] = c00 * id;
  Ai[1] = (A[2] * A[7] - A[1] * A[8]) * id;
  Ai[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  Ai[3] = c01 * id;
  Ai[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  Ai[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  Ai[6] = c02 * id;
  Ai[7] = (A[1] * A[6] - A[0] * A[7]) * id;
  Ai[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return det;
}

// C = A * B (3x3 row-major)
template <typename T>
__device__ __forceinline__ void mul3(const T A[9], const T B[9], T C[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

// Tet geometry from vertex coordinates: cross-product rows c[3][3],
// inverse determinant and the volume sign factor sign(det)/6.
template <typename T>
struct TetGeom {
  T c[3][3];
  T inv_det;
  T s6;     // sign(det) / 6
  T vol;    // |det| / 6
};

template <typename T>
__device__ __forceinline__ void tet_geom(const T x0[3], const T x1[3], const T x2[3],
                                         const T x3[3], TetGeom<T>& g) {
  T d1[3], d2[3], d3[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    d1[i] = x1[i] - x0[i];
    d2[i] = x2[i] - x0[i];
    d3[i] = x3[i] - x0[i];
  }
  cross3(d2, d3, g.c[0]);
  cross3(d3, d1, g.c[1]);
  cross3(d1, d2, g.c[2]);
  T det = d1[0] * g.c[0][0] + d1[1] * g.c[0][1] + d1[2] * g.c[0][2];
  g.inv_det = T(1) / det;
  g.s6 = det < T(0) ? T(-1.0 / 6.0) : T(1.0 / 6.0);
  g.vol = det < T(0) ? -det * T(1.0 / 6.0) : det * T(1.0 / 6.0);
}

// Gradient G_ij = sum_k D_k[i] dN_k[j] of a nodal field with vertex
// differences D_k = v_k - v_0 (k = 1..3).
template <typename T>
__device__ __forceinline__ void grad_from_diffs(const T D[3][3], const TetGeom<T>& g, T G[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      G[3 * i + j] = (D[0][i] * g.c[0][j] + D[1][i] * g.c[1][j] + D[2][i] * g.c[2][j]) * g.inv_det;
}

// Slot vectors f_k = coef * S c_k (k = 1..3), f_0 = -sum.  With coef = -s6
// this is the reference's f_a -= S dN_a vol; with +s6 it is the tangent
// action K p.
template <typename T>
__device__ __forceinline__ void slot_vectors(const T S[9], const TetGeom<T>& g, T coef,
                                             T f[4][3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    T acc0 = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      T v = coef * (S[3 * i] * g.c[k][0] + S[3 * i + 1] * g.c[k][1] + S[3 * i + 2] * g.c[k][2]);
      f[k + 1][i] = v;
      acc0 += v;
    }
    f[0][i] = -acc0;
  }
}

// ───────────────────────── stress (residual, FP64) ─────────────────────────
// Each returns the contracted stress S (P or sigma) and fills the float
// tangent payload pay[kPay] used by the matrix-free tangent.

template <typename T>
__device__ __forceinline__ void nh_stress(const DevMat<T>& m, T scale, const T H[9], T S[9],
                                          float pay[kPay]) {
  T F[9], Fi[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) F[k] = H[k] + ((k % 4 == 0) ? T(1) : T(0));
  T J = inv3(F, Fi);
  T Js = J > T(kJFloor) ? J : T(kJFloor);
  T lnJ = dev_log(Js);
  T mu = m.mu * scale, lam = m.lam * scale;
  T c = lam * lnJ - mu;
  // P = mu F + (lam lnJ - mu) F^-T  ==  J_s sigma F^-T with sigma of neo_hookean.py:120-127
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) S[3 * i + j] = mu * F[3 * i + j] + c * Fi[3 * j + i];
#pragma unroll
  for (int k = 0; k < 9; ++k) pay[k] = float(Fi[k]);
  pay[9] = float(lnJ);
}

template <typename T>
__device__ __forceinline__ void mr_stress(const DevMat<T>& m, T scale, const T H[9], T S[9],
                                          float pay[kPay]) {
  T F[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) F[k] = H[k] + ((k % 4 == 0) ? T(1) : T(0));
  T Bm[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      Bm[3 * i + j] = F[3 * i] * F[3 * j] + F[3 * i + 1] * F[3 * j + 1] + F[3 * i + 2] * F[3 * j + 2];
  T I1 = Bm[0] + Bm[4] + Bm[8];
  T C10 = m.C10 * scale, C01 = m.C01 * scale;
  T BF[9];
  mul3(Bm, F, BF);
  T a = T(2) * (C10 + C01 * I1);
  // P = 2(C10 + C01 I1) F - 2 C01 B F + (2/D1) J_s^2 (J_s - 1) F^-T
  // == J_s sigma F^-T with sigma of mooney_rivlin.py:180-189 (volumetric term as written)
#pragma unroll
  for (int k = 0; k < 9; ++k) S[k] = a * F[k] - T(2) * C01 * BF[k];
  if (m.invD1 != T(0)) {
    T Fi[9];
    T J = inv3(F, Fi);
    T Js = J > T(kJFloor) ? J : T(kJFloor);
    T v = T(2) * m.invD1 * scale * Js * Js * (Js - T(1));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) S[3 * i + j] += v * Fi[3 * j + i];
  }
  if (m.model == M_FMR) {
    for (int k = 0; k < m.n_fibers; ++k) {
      const T* A = m.fa + 3 * k;
      T Fa[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) Fa[i] = F[3 * i] * A[0] + F[3 * i + 1] * A[1] + F[3 * i + 2] * A[2];
      T I4 = Fa[0] * Fa[0] + Fa[1] * Fa[1] + Fa[2] * Fa[2];
      if (I4 > T(1)) {
        T cf = T(0.5) * m.fE * scale * (I4 - T(1));
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) S[3 * i + j] += cf * Fa[i] * A[j];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) pay[k] = float(F[k]);
  pay[9] = 0.f;
}

// sym tensor as 6 comps (xx, yy, zz, yz, xz, xy)
template <typename T>
__device__ __forceinline__ void sym6(const T H[9], T e[6]) {
  e[0] = H[0];
  e[1] = H[4];
  e[2] = H[8];
  e[3] = T(0.5) * (H[5] + H[7]);
  e[4] = T(0.5) * (H[2] + H[6]);
  e[5] = T(0.5) * (H[1] + H[3]);
}

template <typename T>
__device__ __forceinline__ void full9(const T s[6], T S[9]) {
  S[0] = s[0]; S[4] = s[1]; S[8] = s[2];
  S[5] = S[7] = s[3];
  S[2] = S[6] = s[4];
  S[1] = S[3] = s[5];
}

template <typename T>
__device__ __forceinline__ void le_stress(const DevMat<T>& m, T scale, const T H[9], T S[9]) {
  T e[6];
  sym6(H, e);
  T mu = m.mu * scale, lam = m.lam * scale;
  T tr = e[0] + e[1] + e[2];
  T s[6];
#pragma unroll
  for (int k = 0; k < 3; ++k) s[k] = lam * tr + T(2) * mu * e[k];
#pragma unroll
  for (int k = 3; k < 6; ++k) s[k] = T(2) * mu * e[k];
  full9(s, S);
}

template <typename T>
__device__ __forceinline__ void ti_stress(const DevMat<T>& m, T scale, const T H[9], T S[9]) {
  T e[6];
  sym6(H, e);
  // Voigt strain [e11, e22, e33, 2e23, 2e13, 2e12] (transverse_isotropic.py:308-311)
  T ev[6] = {e[0], e[1], e[2], T(2) * e[3], T(2) * e[4], T(2) * e[5]};
  T s[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    T acc = T(0);
#pragma unroll
    for (int j = 0; j < 6; ++j) acc += m.C[6 * i + j] * ev[j];
    s[i] = acc * scale;
  }
  full9(s, S);
}

// J2 radial return (j2_plasticity.py:186-249) from the committed history
// (ep: xx,yy,zz,yz,xz,xy; epe).  Writes the trial history and the
// consistent-tangent payload [n(6), theta, gamma2].
template <typename T>
__device__ __forceinline__ void j2_stress(const DevMat<T>& m, T scale, const T H[9],
                                          const T ep[6], T epe, T S[9], T ep_new[6],
                                          T& epe_new, float pay[kPay]) {
  T e[6];
  sym6(H, e);
  T mu = m.mu * scale, lam = m.lam * scale, Hh = m.H * scale;
  T ee[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) ee[k] = e[k] - ep[k];
  T tr = ee[0] + ee[1] + ee[2];
  T st[6];
#pragma unroll
  for (int k = 0; k < 3; ++k) st[k] = lam * tr + T(2) * mu * ee[k];
#pragma unroll
  for (int k = 3; k < 6; ++k) st[k] = T(2) * mu * ee[k];
  T p = (st[0] + st[1] + st[2]) * T(1.0 / 3.0);
  T s[6] = {st[0] - p, st[1] - p, st[2] - p, st[3], st[4], st[5]};
  T n2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + T(2) * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
  T snorm = sqrt(n2 > T(1e-30) ? n2 : T(1e-30));
  const T r15 = T(1.2247448713915890491);  // sqrt(1.5)
  T q = r15 * snorm;
  T f = q - (m.sigma_y + Hh * epe);
  T out[6];
  if (f <= T(0)) {
#pragma unroll
    for (int k = 0; k < 6; ++k) { out[k] = st[k]; ep_new[k] = ep[k]; }
    epe_new = epe;
#pragma unroll
    for (int k = 0; k < 6; ++k) pay[k] = 0.f;
    pay[6] = 1.f;
    pay[7] = 0.f;
  } else {
    T dg = f / (T(3) * mu + Hh);
    T inv_sn = T(1) / snorm;
    T factor = T(1) - T(3) * mu * dg / q;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      T nk = s[k] * inv_sn;
      ep_new[k] = ep[k] + r15 * dg * nk;
      pay[k] = float(nk);
      out[k] = factor * s[k] + (k < 3 ? p : T(0));
    }
    epe_new = epe + dg;
    pay[6] = float(factor);
    pay[7] = float(T(6) * mu * mu * (T(1) / (T(3) * mu + Hh) - dg / q));
  }
  pay[8] = 0.f;
  pay[9] = 0.f;
  full9(out, S);
}

// ───────────────────────── tangent action dP[dF] (FP32) ─────────────────────────

template <typename T>
__device__ __forceinline__ void dP_nh(const DevMat<T>& m, T scale, const float* pay, const T dF[9],
                                      T dP[9]) {
  T Fi[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) Fi[k] = T(pay[k]);
  T lnJ = T(pay[9]);
  T mu = m.mu * scale, lam = m.lam * scale;
  T G[9], GF[9];
  mul3(Fi, dF, G);
  mul3(G, Fi, GF);
  T trG = G[0] + G[4] + G[8];
  T c1 = mu - lam * lnJ;
  T c2 = lam * trG;
  // dP = mu dF + (mu - lam lnJ) (F^-1 dF F^-1)^T + lam tr(F^-1 dF) F^-T
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      dP[3 * i + j] = mu * dF[3 * i + j] + c1 * GF[3 * j + i] + c2 * Fi[3 * j + i];
}

template <typename T>
__device__ __forceinline__ void dP_mr(const DevMat<T>& m, T scale, const float* pay, const T dF[9],
                                      T dP[9]) {
  T F[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) F[k] = T(pay[k]);
  T C10 = m.C10 * scale, C01 = m.C01 * scale;
  T Bm[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      Bm[3 * i + j] = F[3 * i] * F[3 * j] + F[3 * i + 1] * F[3 * j + 1] + F[3 * i + 2] * F[3 * j + 2];
  T I1 = Bm[0] + Bm[4] + Bm[8];
  T FdF = T(0);
#pragma unroll
  for (int k = 0; k < 9; ++k) FdF += F[k] * dF[k];
  // dF F^T F + F dF^T F + B dF
  T dFFt[9], FdFt[9], W[9], X1[9], X2[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      dFFt[3 * i + j] = dF[3 * i] * F[3 * j] + dF[3 * i + 1] * F[3 * j + 1] + dF[3 * i + 2] * F[3 * j + 2];
      FdFt[3 * i + j] = F[3 * i] * dF[3 * j] + F[3 * i + 1] * dF[3 * j + 1] + F[3 * i + 2] * dF[3 * j + 2];
    }
#pragma unroll
  for (int k = 0; k < 9; ++k) W[k] = dFFt[k] + FdFt[k];
  mul3(W, F, X1);
  mul3(Bm, dF, X2);
  T a = T(2) * (C10 + C01 * I1);
#pragma unroll
  for (int k = 0; k < 9; ++k)
    dP[k] = a * dF[k] + T(4) * C01 * FdF * F[k] - T(2) * C01 * (X1[k] + X2[k]);
  if (m.invD1 != T(0)) {
    T Fi[9], G[9], GF[9];
    T J = inv3(F, Fi);
    T Js = J > T(kJFloor) ? J : T(kJFloor);
    mul3(Fi, dF, G);
    mul3(G, Fi, GF);
    T trG = G[0] + G[4] + G[8];
    T k2 = T(2) * m.invD1 * scale;
    T g = Js * Js * (Js - T(1));
    T dg = (T(3) * Js * Js - T(2) * Js) * Js * trG;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) dP[3 * i + j] += k2 * (dg * Fi[3 * j + i] - g * GF[3 * j + i]);
  }
  if (m.model == M_FMR) {
    for (int k = 0; k < m.n_fibers; ++k) {
      const T* A = m.fa + 3 * k;
      T Fa[3], dFa[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        Fa[i] = F[3 * i] * A[0] + F[3 * i + 1] * A[1] + F[3 * i + 2] * A[2];
        dFa[i] = dF[3 * i] * A[0] + dF[3 * i + 1] * A[1] + dF[3 * i + 2] * A[2];
      }
      T I4 = Fa[0] * Fa[0] + Fa[1] * Fa[1] + Fa[2] * Fa[2];
      if (I4 > T(1)) {
        T fE = m.fE * scale;
        T cf = T(0.5) * fE * (I4 - T(1));
        T dc = fE * (Fa[0] * dFa[0] + Fa[1] * dFa[1] + Fa[2] * dFa[2]);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) dP[3 * i + j] += (dc * Fa[i] + cf * dFa[i]) * A[j];
      }
    }
  }
}

template <typename T>
__device__ __forceinline__ void dP_small(const DevMat<T>& m, int model, T scale, const float* pay,
                                         const T dF[9], T dP[9]) {
  T e[6];
  sym6(dF, e);
  T s[6];
  if (model == M_TI) {
    T ev[6] = {e[0], e[1], e[2], T(2) * e[3], T(2) * e[4], T(2) * e[5]};
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      T acc = T(0);
#pragma unroll
      for (int j = 0; j < 6; ++j) acc += m.C[6 * i + j] * ev[j];
      s[i] = acc * scale;
    }
  } else {
    T mu = m.mu * scale, lam = m.lam * scale;
    T tr = e[0] + e[1] + e[2];
    if (model == M_J2) {
      // C_ep = K 1(x)1 + 2 mu theta I_dev - gamma2 n (x) n
      T kap = lam + T(2.0 / 3.0) * mu;
      T theta = T(pay[6]), g2 = T(pay[7]);
      T nd = T(pay[0]) * e[0] + T(pay[1]) * e[1] + T(pay[2]) * e[2] +
             T(2) * (T(pay[3]) * e[3] + T(pay[4]) * e[4] + T(pay[5]) * e[5]);
      T tm = T(2) * mu * theta;
      T c = kap * tr - tm * tr * T(1.0 / 3.0);
#pragma unroll
      for (int k = 0; k < 6; ++k) s[k] = tm * e[k] - g2 * nd * T(pay[k]) + (k < 3 ? c : T(0));
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) s[k] = lam * tr + T(2) * mu * e[k];
#pragma unroll
      for (int k = 3; k < 6; ++k) s[k] = T(2) * mu * e[k];
    }
  }
  full9(s, dP);
}

template <int MODEL, typename T>
__device__ __forceinline__ void dP_any(const DevMat<T>& m, T scale, const float* pay, const T dF[9],
                                       T dP[9]) {
  const int model = MODEL >= 0 ? MODEL : m.model;
  if (model == M_NH) {
    dP_nh(m, scale, pay, dF, dP);
  } else if (model == M_MR || model == M_FMR) {
    dP_mr(m, scale, pay, dF, dP);
  } else {
    dP_small(m, model, scale, pay, dF, dP);
  }
}

template <int MODEL>
__device__ __forceinline__ bool model_has_payload(int model) {
  const int md = MODEL >= 0 ? MODEL : model;
  return md == M_NH || md == M_MR || md == M_FMR || md == M_J2;
}

// payload words a model uses: NH F^-1 + ln J (10), MR F (9), J2 n + theta + gamma2 (8)
__host__ __device__ __forceinline__ int model_pay_words(int model) {
  return model == M_NH ? 10 : (model == M_J2 ? 8 : ((model == M_MR || model == M_FMR) ? 9 : 0));
}

// Jacobi diagonal of one node from its summed element entries acc (BLOCK:
// the 3 x 3 diagonal block 00 01 02 11 12 22; else the 3 diagonal entries):
// dinv = 1 / diag on free DOFs, or (BLOCK) the inverse of the block
// restricted to the free DOFs, computed in FP64, with its diagonal in dinv
// and its off-diagonals (01, 02, 12) in boff.  A block that is not positive
// definite falls back to the scalar inverse of its diagonal.
template <bool BLOCK>
__device__ __forceinline__ void diag_store(const float* acc, uint8_t fx, int node, float* dinv, float* boff) {
  if (!BLOCK) {
    float dv[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) dv[d] = (((fx >> d) & 1) || !(acc[d] > 0.f)) ? 0.f : 1.f / acc[d];
    reinterpret_cast<float4*>(dinv)[node] = make_float4(dv[0], dv[1], dv[2], 0.f);
    return;
  }
  // acc: 00 01 02 11 12 22; fixed rows/columns replaced by the identity
  const bool f0 = fx & 1, f1 = (fx >> 1) & 1, f2 = (fx >> 2) & 1;
  const double k00 = f0 ? 1.0 : acc[0], k11 = f1 ? 1.0 : acc[3], k22 = f2 ? 1.0 : acc[5];
  const double k01 = (f0 || f1) ? 0.0 : acc[1], k02 = (f0 || f2) ? 0.0 : acc[2], k12 = (f1 || f2) ? 0.0 : acc[4];
  const double c00 = k11 * k22 - k12 * k12, c01 = k02 * k12 - k01 * k22, c02 = k01 * k12 - k02 * k11;
  const double det = k00 * c00 + k01 * c01 + k02 * c02;
  float4 dv, ov;
  if (det > 0.0 && k00 > 0.0 && k00 * k11 - k01 * k01 > 0.0 && isfinite(det)) {
    const double id = 1.0 / det;
    const double i11 = (k00 * k22 - k02 * k02) * id, i22 = (k00 * k11 - k01 * k01) * id;
    const double i12 = (k01 * k02 - k00 * k12) * id;
    dv = make_float4(f0 ? 0.f : (float)(c00 * id), f1 ? 0.f : (float)i11, f2 ? 0.f : (float)i22, 0.f);
    ov = make_float4((f0 || f1) ? 0.f : (float)(c01 * id), (f0 || f2) ? 0.f : (float)(c02 * id),
                     (f1 || f2) ? 0.f : (float)i12, 0.f);
  } else {
    dv = make_float4((f0 || !(acc[0] > 0.f)) ? 0.f : 1.f / acc[0], (f1 || !(acc[3] > 0.f)) ? 0.f : 1.f / acc[3],
                     (f2 || !(acc[5] > 0.f)) ? 0.f : 1.f / acc[5], 0.f);
    ov = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  reinterpret_cast<float4*>(dinv)[node] = dv;
  reinterpret_cast<float4*>(boff)[node] = ov;
}

}  // namespace femb200
