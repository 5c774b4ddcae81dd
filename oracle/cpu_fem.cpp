// CPU restatement of the TET4 static solve — TEST / BASELINE INFRASTRUCTURE ONLY.
//
// Same arithmetic as oracle/fem_oracle.py (FP64 throughout), parallelised with
// OpenMP, used as the timed CPU baseline of the benchmark.  It restates:
//   reference quantities / F  backend/fea/fem/core/mesh.py:123-151, 293-313
//   Neo-Hookean               backend/fea/fem/material/neo_hookean.py:99-190
//   J2 radial return          backend/fea/fem/material/j2_plasticity.py:186-249, 366-393
//   linear elastic            backend/fea/fem/material/linear_elastic.py:102-173
//   Newton loop               backend/fea/fem/solver/static_solver.py:135-265
// with the consistent tangent applied matrix-free and Jacobi-PCG as the linear
// solver (the reference's spsolve does not scale to these meshes), i.e. the
// same method the GPU path runs, so iteration counts are comparable.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {

enum { LE = 0, NH = 1, J2 = 3 };

struct Problem {
  int Nn, Ne, model;
  const double* X;
  const int* conn;
  const double* E;   // per element
  double nu, sy, Hr; // J2: yield stress, hardening = Hr * E
  const uint8_t* fixed;
  std::vector<double> c[3][3];  // per element cross-product rows (flattened Ne each)
  std::vector<double> inv_det, s6;
  std::vector<int> row, slot;   // node -> element*4+slot
};

void geometry(Problem& P) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) P.c[a][b].assign(P.Ne, 0.0);
  P.inv_det.assign(P.Ne, 0.0);
  P.s6.assign(P.Ne, 0.0);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.Ne; ++e) {
    const int* cn = P.conn + 4 * e;
    double d[3][3];
    for (int k = 0; k < 3; ++k)
      for (int i = 0; i < 3; ++i) d[k][i] = P.X[3 * cn[k + 1] + i] - P.X[3 * cn[0] + i];
    double c0[3] = {d[1][1] * d[2][2] - d[1][2] * d[2][1], d[1][2] * d[2][0] - d[1][0] * d[2][2],
                    d[1][0] * d[2][1] - d[1][1] * d[2][0]};
    double c1[3] = {d[2][1] * d[0][2] - d[2][2] * d[0][1], d[2][2] * d[0][0] - d[2][0] * d[0][2],
                    d[2][0] * d[0][1] - d[2][1] * d[0][0]};
    double c2[3] = {d[0][1] * d[1][2] - d[0][2] * d[1][1], d[0][2] * d[1][0] - d[0][0] * d[1][2],
                    d[0][0] * d[1][1] - d[0][1] * d[1][0]};
    double det = d[0][0] * c0[0] + d[0][1] * c0[1] + d[0][2] * c0[2];
    for (int j = 0; j < 3; ++j) {
      P.c[0][j][e] = c0[j];
      P.c[1][j][e] = c1[j];
      P.c[2][j][e] = c2[j];
    }
    P.inv_det[e] = 1.0 / det;
    P.s6[e] = det < 0 ? -1.0 / 6.0 : 1.0 / 6.0;
  }
  P.row.assign(P.Nn + 1, 0);
  for (int e = 0; e < P.Ne; ++e)
    for (int k = 0; k < 4; ++k) P.row[P.conn[4 * e + k] + 1]++;
  for (int i = 0; i < P.Nn; ++i) P.row[i + 1] += P.row[i];
  P.slot.assign(P.row[P.Nn], 0);
  std::vector<int> fill(P.row.begin(), P.row.end() - 1);
  for (int e = 0; e < P.Ne; ++e)
    for (int k = 0; k < 4; ++k) P.slot[fill[P.conn[4 * e + k]]++] = 4 * e + k;
}

inline void grad(const Problem& P, int e, const double* v, double G[9]) {
  const int* cn = P.conn + 4 * e;
  double D[3][3];
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i) D[k][i] = v[3 * cn[k + 1] + i] - v[3 * cn[0] + i];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      G[3 * i + j] = (D[0][i] * P.c[0][j][e] + D[1][i] * P.c[1][j][e] + D[2][i] * P.c[2][j][e]) * P.inv_det[e];
}

inline void slots(const Problem& P, int e, const double S[9], double coef, double* fe) {
  for (int i = 0; i < 3; ++i) {
    double a0 = 0;
    for (int k = 0; k < 3; ++k) {
      double v = coef * (S[3 * i] * P.c[k][0][e] + S[3 * i + 1] * P.c[k][1][e] + S[3 * i + 2] * P.c[k][2][e]);
      fe[3 * (k + 1) + i] = v;
      a0 += v;
    }
    fe[i] = -a0;
  }
}

inline double inv3(const double A[9], double Ai[9]) {
  double c00 = A[4] * A[8] - A[5] * A[7], c01 = A[5] * A[6] - A[3] * A[8], c02 = A[3] * A[7] - A[4] * A[6];
  double det = A[0] * c00 + A[1] * c01 + A[2] * c02, id = 1.0 / det;
  Ai[0] = c00 * id; Ai[1] = (A[2] * A[7] - A[1] * A[8]) * id; Ai[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  Ai[3] = c01 * id; Ai[4] = (A[0] * A[8] - A[2] * A[6]) * id; Ai[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  Ai[6] = c02 * id; Ai[7] = (A[1] * A[6] - A[0] * A[7]) * id; Ai[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return det;
}

// per-element tangent state: NH -> Finv(9), lnJ ; J2 -> n(6), theta, gamma2
struct State {
  std::vector<double> t;  // Ne * 10
  std::vector<double> ep_t, epe_t;
};

void element_stress(const Problem& P, int e, const double H[9], const double* ep_c, const double* epe_c,
                    double S[9], double* tan, double* ep_out, double* epe_out) {
  const double E = P.E[e], nu = P.nu;
  const double mu = E / (2 * (1 + nu)), lam = E * nu / ((1 + nu) * (1 - 2 * nu));
  if (P.model == NH) {
    double F[9], Fi[9];
    for (int k = 0; k < 9; ++k) F[k] = H[k] + (k % 4 == 0 ? 1.0 : 0.0);
    double J = inv3(F, Fi);
    double lnJ = std::log(J > 1e-8 ? J : 1e-8);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) S[3 * i + j] = mu * F[3 * i + j] + (lam * lnJ - mu) * Fi[3 * j + i];
    for (int k = 0; k < 9; ++k) tan[k] = Fi[k];
    tan[9] = lnJ;
    return;
  }
  double eps[6] = {H[0], H[4], H[8], 0.5 * (H[5] + H[7]), 0.5 * (H[2] + H[6]), 0.5 * (H[1] + H[3])};
  double s[6];
  if (P.model == J2) {
    const double Hh = P.Hr * E;
    double ee[6];
    for (int k = 0; k < 6; ++k) ee[k] = eps[k] - ep_c[6 * e + k];
    double tr = ee[0] + ee[1] + ee[2];
    double st[6];
    for (int k = 0; k < 3; ++k) st[k] = lam * tr + 2 * mu * ee[k];
    for (int k = 3; k < 6; ++k) st[k] = 2 * mu * ee[k];
    double p = (st[0] + st[1] + st[2]) / 3.0;
    double dv[6] = {st[0] - p, st[1] - p, st[2] - p, st[3], st[4], st[5]};
    double n2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2] + 2 * (dv[3] * dv[3] + dv[4] * dv[4] + dv[5] * dv[5]);
    double sn = std::sqrt(n2 > 1e-30 ? n2 : 1e-30);
    double q = std::sqrt(1.5) * sn;
    double f = q - (P.sy + Hh * epe_c[e]);
    if (f <= 0) {
      for (int k = 0; k < 6; ++k) { s[k] = st[k]; ep_out[6 * e + k] = ep_c[6 * e + k]; tan[k] = 0; }
      epe_out[e] = epe_c[e];
      tan[6] = 1;
      tan[7] = 0;
    } else {
      double dg = f / (3 * mu + Hh), fac = 1 - 3 * mu * dg / q;
      for (int k = 0; k < 6; ++k) {
        double nk = dv[k] / sn;
        ep_out[6 * e + k] = ep_c[6 * e + k] + std::sqrt(1.5) * dg * nk;
        tan[k] = nk;
        s[k] = fac * dv[k] + (k < 3 ? p : 0.0);
      }
      epe_out[e] = epe_c[e] + dg;
      tan[6] = fac;
      tan[7] = 6 * mu * mu * (1 / (3 * mu + Hh) - dg / q);
    }
  } else {
    double tr = eps[0] + eps[1] + eps[2];
    for (int k = 0; k < 3; ++k) s[k] = lam * tr + 2 * mu * eps[k];
    for (int k = 3; k < 6; ++k) s[k] = 2 * mu * eps[k];
  }
  S[0] = s[0]; S[4] = s[1]; S[8] = s[2];
  S[5] = S[7] = s[3]; S[2] = S[6] = s[4]; S[1] = S[3] = s[5];
}

void element_dP(const Problem& P, int e, const double* tan, const double dF[9], double dP[9]) {
  const double E = P.E[e], nu = P.nu;
  const double mu = E / (2 * (1 + nu)), lam = E * nu / ((1 + nu) * (1 - 2 * nu));
  if (P.model == NH) {
    const double* Fi = tan;
    double G[9], GF[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        G[3 * i + j] = Fi[3 * i] * dF[j] + Fi[3 * i + 1] * dF[3 + j] + Fi[3 * i + 2] * dF[6 + j];
      }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) GF[3 * i + j] = G[3 * i] * Fi[j] + G[3 * i + 1] * Fi[3 + j] + G[3 * i + 2] * Fi[6 + j];
    double trG = G[0] + G[4] + G[8], c1 = mu - lam * tan[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) dP[3 * i + j] = mu * dF[3 * i + j] + c1 * GF[3 * j + i] + lam * trG * Fi[3 * j + i];
    return;
  }
  double e6[6] = {dF[0], dF[4], dF[8], 0.5 * (dF[5] + dF[7]), 0.5 * (dF[2] + dF[6]), 0.5 * (dF[1] + dF[3])};
  double tr = e6[0] + e6[1] + e6[2];
  double s[6];
  if (P.model == J2) {
    double kap = lam + 2.0 * mu / 3.0, tm = 2 * mu * tan[6], g2 = tan[7];
    double nd = tan[0] * e6[0] + tan[1] * e6[1] + tan[2] * e6[2] + 2 * (tan[3] * e6[3] + tan[4] * e6[4] + tan[5] * e6[5]);
    double c = kap * tr - tm * tr / 3.0;
    for (int k = 0; k < 6; ++k) s[k] = tm * e6[k] - g2 * nd * tan[k] + (k < 3 ? c : 0.0);
  } else {
    for (int k = 0; k < 3; ++k) s[k] = lam * tr + 2 * mu * e6[k];
    for (int k = 3; k < 6; ++k) s[k] = 2 * mu * e6[k];
  }
  dP[0] = s[0]; dP[4] = s[1]; dP[8] = s[2];
  dP[5] = dP[7] = s[3]; dP[2] = dP[6] = s[4]; dP[1] = dP[3] = s[5];
}

// R = f_ext + f (fixed zeroed); returns ||R||^2, refreshes the tangent state
double residual(const Problem& P, const double* u, const double* fext, const double* ep_c, const double* epe_c,
                State& st, std::vector<double>& fe, double* R) {
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.Ne; ++e) {
    double Hg[9], S[9];
    grad(P, e, u, Hg);
    element_stress(P, e, Hg, ep_c, epe_c, S, &st.t[10 * e], st.ep_t.data(), st.epe_t.data());
    slots(P, e, S, -P.s6[e], &fe[12 * e]);
  }
  double r2 = 0;
#pragma omp parallel for schedule(static) reduction(+ : r2)
  for (int n = 0; n < P.Nn; ++n) {
    double acc[3] = {0, 0, 0};
    for (int j = P.row[n]; j < P.row[n + 1]; ++j)
      for (int d = 0; d < 3; ++d) acc[d] += fe[3 * P.slot[j] + d];
    for (int d = 0; d < 3; ++d) {
      double r = ((P.fixed[3 * n + d]) ? 0.0 : fext[3 * n + d] + acc[d]);
      R[3 * n + d] = r;
      r2 += r * r;
    }
  }
  return r2;
}

void matvec(const Problem& P, const State& st, const double* x, std::vector<double>& fe, double* y) {
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.Ne; ++e) {
    double dF[9], dP[9];
    grad(P, e, x, dF);
    element_dP(P, e, &st.t[10 * e], dF, dP);
    slots(P, e, dP, P.s6[e], &fe[12 * e]);
  }
#pragma omp parallel for schedule(static)
  for (int n = 0; n < P.Nn; ++n) {
    double acc[3] = {0, 0, 0};
    for (int j = P.row[n]; j < P.row[n + 1]; ++j)
      for (int d = 0; d < 3; ++d) acc[d] += fe[3 * P.slot[j] + d];
    for (int d = 0; d < 3; ++d) y[3 * n + d] = P.fixed[3 * n + d] ? 0.0 : acc[d];
  }
}

void jacobi(const Problem& P, const State& st, std::vector<double>& fe, std::vector<double>& dinv) {
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.Ne; ++e) {
    double w[4][3];
    for (int j = 0; j < 3; ++j) {
      w[1][j] = P.c[0][j][e];
      w[2][j] = P.c[1][j][e];
      w[3][j] = P.c[2][j][e];
      w[0][j] = -(w[1][j] + w[2][j] + w[3][j]);
    }
    for (int s = 0; s < 4; ++s)
      for (int i = 0; i < 3; ++i) {
        double dF[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dP[9];
        for (int j = 0; j < 3; ++j) dF[3 * i + j] = w[s][j] * P.inv_det[e];
        element_dP(P, e, &st.t[10 * e], dF, dP);
        fe[12 * e + 3 * s + i] = P.s6[e] * (dP[3 * i] * w[s][0] + dP[3 * i + 1] * w[s][1] + dP[3 * i + 2] * w[s][2]);
      }
  }
#pragma omp parallel for schedule(static)
  for (int n = 0; n < P.Nn; ++n) {
    double acc[3] = {0, 0, 0};
    for (int j = P.row[n]; j < P.row[n + 1]; ++j)
      for (int d = 0; d < 3; ++d) acc[d] += fe[3 * P.slot[j] + d];
    for (int d = 0; d < 3; ++d) dinv[3 * n + d] = (P.fixed[3 * n + d] || !(acc[d] > 0)) ? 0.0 : 1.0 / acc[d];
  }
}

double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
  const int n = (int)a.size();
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

int pcg(const Problem& P, const State& st, const double* b, double rtol, int maxit, std::vector<double>& fe,
        std::vector<double>& x) {
  const int n = 3 * P.Nn;
  std::vector<double> dinv(n), r(b, b + n), z(n), p(n), y(n);
  jacobi(P, st, fe, dinv);
  std::fill(x.begin(), x.end(), 0.0);
  for (int i = 0; i < n; ++i) z[i] = dinv[i] * r[i];
  p = z;
  double rz = dot(r, z), rr0 = dot(r, r), rr = rr0;
  int it = 0;
  while (it < maxit && rr > rtol * rtol * rr0 && rr0 > 0) {
    matvec(P, st, p.data(), fe, y.data());
    double alpha = rz / dot(p, y);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * y[i];
      z[i] = dinv[i] * r[i];
    }
    double rz2 = dot(r, z);
    rr = dot(r, r);
    double beta = rz2 / rz;
    rz = rz2;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    ++it;
  }
  return it;
}

}  // namespace

extern "C" {

// One static solve (one load level).  u, ep (Ne*6: xx,yy,zz,yz,xz,xy), epe are
// in/out; stats[0..4] = newton iterations, cg iterations, final rel residual,
// residual evaluations, converged.  Returns 0.  max_cg_total > 0 caps the CG
// work of the whole call (a bounded sample).
int cpu_fem_solve(int Nn, int Ne, const double* X, const int* conn, int model, const double* E,
                  double nu, double sigma_y, double H_ratio, const uint8_t* fixed, const double* fixed_vals,
                  const double* fext, double* u, double* ep, double* epe, double tol, int max_newton,
                  int max_cg, double cg_rtol_min, int max_cg_total, int threads, double* stats) {
  if (threads > 0) omp_set_num_threads(threads);
  Problem P;
  P.Nn = Nn; P.Ne = Ne; P.model = model; P.X = X; P.conn = conn; P.E = E; P.nu = nu;
  P.sy = sigma_y; P.Hr = H_ratio; P.fixed = fixed;
  geometry(P);
  const int n = 3 * Nn;
  State st;
  st.t.assign((size_t)10 * Ne, 0.0);
  st.ep_t.assign((size_t)6 * Ne, 0.0);
  st.epe_t.assign(Ne, 0.0);
  std::vector<double> fe((size_t)12 * Ne), R(n), du(n), ub(n), dc(n, 0.0), y(n);
  // prescribed-value change of this solve, carried by the first Newton step
  bool has_dc = false;
  for (int i = 0; i < n; ++i)
    if (fixed[i]) {
      dc[i] = fixed_vals[i] - u[i];
      has_dc = has_dc || dc[i] != 0.0;
    }
  int it = 0, cg_total = 0, evals = 0;
  double ref;
  if (has_dc) {
    for (int i = 0; i < n; ++i) ub[i] = u[i] + dc[i];
    ref = std::sqrt(residual(P, ub.data(), fext, ep, epe, st, fe, R.data()));
    residual(P, u, fext, ep, epe, st, fe, R.data());
    evals += 2;
    matvec(P, st, dc.data(), fe, y.data());
    for (int i = 0; i < n; ++i) R[i] -= y[i];
    // the predictor fixes the elastic state of the step: solve it to 1e-3
    double eta = std::max(1e-3, cg_rtol_min);
    cg_total += pcg(P, st, R.data(), eta, max_cg, fe, du);
    for (int i = 0; i < n; ++i) u[i] += du[i] + dc[i];
    it = 1;
  } else {
    ref = -1.0;
  }
  double r2 = residual(P, u, fext, ep, epe, st, fe, R.data());
  ++evals;
  double res = std::sqrt(r2);
  if (ref < 0) ref = res;
  ref = ref > 1e-20 ? ref : 1.0;
  double prev = res;
  bool conv = false;
  for (; it < max_newton; ++it) {
    if (res / ref < tol) { conv = true; break; }
    if (max_cg_total > 0 && cg_total >= max_cg_total) break;
    // forcing term: aim at the target, follow the residual's contraction, and
    // solve tightly (1e-3) when the residual did not drop
    double e2 = (it > 0 && res < prev) ? 0.9 * (res / prev) * (res / prev) : 1e-3;
    double eta = std::min(std::max(std::max(0.1 * tol * ref / res, e2), cg_rtol_min), 0.1);
    int cap = max_cg;
    if (max_cg_total > 0) cap = std::min(cap, max_cg_total - cg_total);
    cg_total += pcg(P, st, R.data(), eta, cap, fe, du);
    std::memcpy(ub.data(), u, n * sizeof(double));
    double alpha = 1.0, trial = res;
    for (int ls = 0; ls < 5; ++ls) {
      for (int i = 0; i < n; ++i) u[i] = ub[i] + alpha * du[i];
      trial = std::sqrt(residual(P, u, fext, ep, epe, st, fe, R.data()));
      ++evals;
      if (std::isfinite(trial) && trial < 1e6 * res) break;
      alpha *= 0.5;
    }
    prev = res;
    res = trial;
  }
  if (conv && model == J2) {
    std::memcpy(ep, st.ep_t.data(), (size_t)6 * Ne * sizeof(double));
    std::memcpy(epe, st.epe_t.data(), (size_t)Ne * sizeof(double));
  }
  stats[0] = std::min(it + 1, max_newton);
  stats[1] = cg_total;
  stats[2] = res / ref;
  stats[3] = evals;
  stats[4] = conv ? 1 : 0;
  return 0;
}

int cpu_fem_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
