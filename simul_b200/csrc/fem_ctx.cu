// Host driver and C ABI of the TET4 static-solve path (include/femb200.h).
//
// Set-up (fem_ctx_create) renumbers nodes by Morton code, groups elements by
// the block of their lowest node, and builds the node-block gather tables the
// element kernels use.  Callers keep their own numbering: every per-call array
// is permuted on entry and exit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/femb200.h"
#include "fem_internal.h"

using namespace femb200;

namespace {

thread_local std::string g_create_error;

enum { SITE_RES = 0, SITE_MV = 1, SITE_CGI = 2, SITE_CGU = 3, SITE_AUX = 4, N_SITES = 5 };
constexpr int kCGBatch = 32;  // CG iterations per captured graph launch

struct FemCtx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int Nn = 0, Ne = 0, nb = 256, n_blocks = 0;
  int ndof = 0, ndof_pad = 0;
  int64_t blk_entries = 0;
  size_t bytes = 0;
  std::string err;
  std::vector<int> perm_node, perm_elem;  // internal -> caller

  // device buffers
  double* X64 = nullptr;
  float4* X32 = nullptr;
  int4* conn = nullptr;
  uint8_t* mat_id = nullptr;
  float* scale = nullptr;
  int* blk_ptr = nullptr;
  int* blk_home = nullptr;
  int* blk_elems = nullptr;
  int* node_row = nullptr;
  uint32_t* node_slots = nullptr;
  uint8_t* fixed = nullptr;
  double* fixed_vals = nullptr;
  double* fext = nullptr;
  double* u = nullptr;
  double* u_base = nullptr;
  double* R = nullptr;
  double* tmpd = nullptr;
  float* payload = nullptr;
  double* ep_c = nullptr;
  double* epe_c = nullptr;
  double* ep_t = nullptr;
  double* epe_t = nullptr;
  float *r = nullptr, *x = nullptr, *p = nullptr, *y = nullptr, *dinv = nullptr, *tmpf = nullptr;
  int* d_perm_node = nullptr;
  int* d_perm_elem = nullptr;
  DevMat<double>* matD = nullptr;
  DevMat<float>* matF = nullptr;
  double* partials = nullptr;
  unsigned int* counters = nullptr;
  int max_blocks = 0;
  double* scalars = nullptr;  // [0] = ||R||^2
  CGState* cg = nullptr;
  // pinned host mirrors
  CGState* h_cg = nullptr;
  double* h_scalars = nullptr;

  // statistics since creation: kernel launches issued by this library, CG
  // iterations, residual evaluations, CG graph launches
  int64_t n_launches = 0, n_cg_iters = 0, n_res_evals = 0, n_graphs = 0;

  int model_kind = M_LE;       // single model, or -1 for mixed tables
  bool has_j2 = false;
  bool materials_set = false;
  bool tangent_valid = false;
  cudaGraphExec_t cg_graph = nullptr;
  int cg_graph_model = -2;
  int cg_graph_precond = -1;

  MeshDev mesh() const {
    MeshDev m;
    m.n_nodes = Nn;
    m.n_elems = Ne;
    m.n_blocks = n_blocks;
    m.nb = nb;
    m.X64 = X64;
    m.X32 = X32;
    m.conn = conn;
    m.mat_id = mat_id;
    m.scale = scale;
    m.blk_ptr = blk_ptr;
    m.blk_home = blk_home;
    m.blk_elems = blk_elems;
    m.node_row = node_row;
    m.node_slots = node_slots;
    m.fixed = fixed;
    return m;
  }
  Reduce red() const {
    Reduce rd;
    rd.partials = partials;
    rd.counters = counters;
    rd.max_blocks = max_blocks;
    return rd;
  }
};

int set_err(FemCtx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c)
    c->err = buf;
  else
    g_create_error = buf;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e__ = (call);                                                             \
    if (e__ != cudaSuccess)                                                               \
      return set_err(c, FEM_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e__), \
                     __FILE__, __LINE__);                                                 \
  } while (0)

#define CKL()                                                                             \
  do {                                                                                    \
    cudaError_t e__ = cudaGetLastError();                                                 \
    if (e__ != cudaSuccess)                                                               \
      return set_err(c, FEM_ERR_CUDA, "kernel launch failed: %s (%s:%d)",                 \
                     cudaGetErrorString(e__), __FILE__, __LINE__);                        \
  } while (0)

template <typename T>
int dalloc(FemCtx* c, T** ptr, size_t count) {
  size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(ptr), bytes);
  if (e != cudaSuccess)
    return set_err(c, FEM_ERR_CUDA, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  c->bytes += bytes;
  e = cudaMemsetAsync(*ptr, 0, bytes, c->stream);
  if (e != cudaSuccess) return set_err(c, FEM_ERR_CUDA, "cudaMemset failed: %s", cudaGetErrorString(e));
  return FEM_OK;
}

inline uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

struct Quant {
  double lo[3], inv[3];
  uint32_t code(const double p[3]) const {
    uint32_t q[3];
    for (int d = 0; d < 3; ++d) {
      double t = (p[d] - lo[d]) * inv[d];
      t = std::min(std::max(t, 0.0), 1023.0);
      q[d] = (uint32_t)t;
    }
    return spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2);
  }
};

void free_ctx(FemCtx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->cg_graph) cudaGraphExecDestroy(c->cg_graph);
  void* ptrs[] = {c->X64, c->X32, c->conn, c->mat_id, c->scale, c->blk_ptr, c->blk_home,
                  c->blk_elems, c->node_row, c->node_slots, c->fixed, c->fixed_vals, c->fext,
                  c->u, c->u_base, c->R, c->tmpd, c->payload, c->ep_c, c->epe_c, c->ep_t,
                  c->epe_t, c->r, c->x, c->p, c->y, c->dinv, c->tmpf, c->d_perm_node,
                  c->d_perm_elem, c->matD, c->matF, c->partials, c->counters, c->scalars, c->cg};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->h_cg) cudaFreeHost(c->h_cg);
  if (c->h_scalars) cudaFreeHost(c->h_scalars);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

// ───────────────────────── set-up ─────────────────────────

int build_tables(FemCtx* c, const double* X, const int32_t* conn_user) {
  const int Nn = c->Nn, Ne = c->Ne, nb = c->nb;
  // Morton renumbering of nodes
  Quant qz;
  for (int d = 0; d < 3; ++d) {
    double lo = X[d], hi = X[d];
    for (int i = 0; i < Nn; ++i) {
      lo = std::min(lo, X[3 * i + d]);
      hi = std::max(hi, X[3 * i + d]);
    }
    qz.lo[d] = lo;
    qz.inv[d] = hi > lo ? 1023.999 / (hi - lo) : 0.0;
  }
  std::vector<uint32_t> ncode(Nn);
  for (int i = 0; i < Nn; ++i) ncode[i] = qz.code(X + 3 * i);
  c->perm_node.resize(Nn);
  std::iota(c->perm_node.begin(), c->perm_node.end(), 0);
  std::stable_sort(c->perm_node.begin(), c->perm_node.end(),
                   [&](int a, int b) { return ncode[a] < ncode[b]; });
  std::vector<int> iperm(Nn);
  for (int i = 0; i < Nn; ++i) iperm[c->perm_node[i]] = i;

  // elements: home block = block of the lowest internal node, then Morton of centroid
  std::vector<int> home(Ne);
  std::vector<uint32_t> ecode(Ne);
  for (int e = 0; e < Ne; ++e) {
    int mn = Nn;
    double cen[3] = {0, 0, 0};
    for (int k = 0; k < 4; ++k) {
      const int nu = conn_user[4 * e + k];
      mn = std::min(mn, iperm[nu]);
      for (int d = 0; d < 3; ++d) cen[d] += 0.25 * X[3 * nu + d];
    }
    home[e] = mn / nb;
    ecode[e] = qz.code(cen);
  }
  c->perm_elem.resize(Ne);
  std::iota(c->perm_elem.begin(), c->perm_elem.end(), 0);
  std::stable_sort(c->perm_elem.begin(), c->perm_elem.end(), [&](int a, int b) {
    if (home[a] != home[b]) return home[a] < home[b];
    return ecode[a] < ecode[b];
  });
  std::vector<int4> conn(Ne);
  std::vector<int> ehome(Ne);
  for (int e = 0; e < Ne; ++e) {
    const int eu = c->perm_elem[e];
    conn[e] = make_int4(iperm[conn_user[4 * eu]], iperm[conn_user[4 * eu + 1]],
                        iperm[conn_user[4 * eu + 2]], iperm[conn_user[4 * eu + 3]]);
    ehome[e] = home[eu];
  }
  // node -> (element, slot) adjacency, sorted by element id
  std::vector<int> arow(Nn + 1, 0);
  for (int e = 0; e < Ne; ++e) {
    const int* cn = &conn[e].x;
    for (int k = 0; k < 4; ++k) arow[cn[k] + 1]++;
  }
  for (int i = 0; i < Nn; ++i) arow[i + 1] += arow[i];
  std::vector<int> acol(arow[Nn]);
  std::vector<int> fill(arow.begin(), arow.end() - 1);
  for (int e = 0; e < Ne; ++e) {
    const int* cn = &conn[e].x;
    for (int k = 0; k < 4; ++k) acol[fill[cn[k]]++] = (e << 2) | k;
  }
  // blocks
  const int nblkn = (Nn + nb - 1) / nb;
  c->n_blocks = nblkn;
  std::vector<int> hs(nblkn + 1, Ne);
  {
    int e = 0;
    for (int b = 0; b <= nblkn; ++b) {
      while (e < Ne && ehome[e] < b) ++e;
      hs[b] = e;
    }
  }
  std::vector<int> blk_ptr(nblkn + 1, 0), blk_home(nblkn, 0), blk_elems;
  std::vector<int> node_row(Nn + 1, 0);
  std::vector<uint32_t> node_slots(arow[Nn]);
  blk_elems.reserve((size_t)Ne * 3 / 2);
  std::vector<int> foreign;
  std::vector<uint32_t> ents;
  for (int b = 0; b < nblkn; ++b) {
    const int n0 = b * nb, n1 = std::min(Nn, n0 + nb);
    const int h0 = hs[b], h1 = hs[b + 1];
    foreign.clear();
    for (int n = n0; n < n1; ++n)
      for (int j = arow[n]; j < arow[n + 1]; ++j) {
        const int e = acol[j] >> 2;
        if (ehome[e] != b) foreign.push_back(e);
      }
    std::sort(foreign.begin(), foreign.end());
    foreign.erase(std::unique(foreign.begin(), foreign.end()), foreign.end());
    blk_ptr[b] = (int)blk_elems.size();
    blk_home[b] = h1 - h0;
    for (int e = h0; e < h1; ++e) blk_elems.push_back(e);
    for (int e : foreign) blk_elems.push_back(e);
    for (int n = n0; n < n1; ++n) {
      ents.clear();
      for (int j = arow[n]; j < arow[n + 1]; ++j) {
        const int e = acol[j] >> 2, s = acol[j] & 3;
        int li;
        if (ehome[e] == b) {
          li = e - h0;
        } else {
          li = (h1 - h0) + (int)(std::lower_bound(foreign.begin(), foreign.end(), e) - foreign.begin());
        }
        ents.push_back(((uint32_t)li << 2) | (uint32_t)s);
      }
      std::sort(ents.begin(), ents.end());
      node_row[n + 1] = node_row[n] + (int)ents.size();
      std::copy(ents.begin(), ents.end(), node_slots.begin() + node_row[n]);
    }
  }
  blk_ptr[nblkn] = (int)blk_elems.size();
  c->blk_entries = (int64_t)blk_elems.size();

  // device uploads
  std::vector<double> X64(3 * (size_t)Nn);
  std::vector<float4> X32(Nn);
  for (int i = 0; i < Nn; ++i) {
    const int iu = c->perm_node[i];
    for (int d = 0; d < 3; ++d) X64[3 * i + d] = X[3 * iu + d];
    X32[i] = make_float4((float)X[3 * iu], (float)X[3 * iu + 1], (float)X[3 * iu + 2], 0.f);
  }
  int st;
  if ((st = dalloc(c, &c->X64, X64.size()))) return st;
  if ((st = dalloc(c, &c->X32, (size_t)Nn))) return st;
  if ((st = dalloc(c, &c->conn, (size_t)Ne))) return st;
  if ((st = dalloc(c, &c->blk_ptr, blk_ptr.size()))) return st;
  if ((st = dalloc(c, &c->blk_home, blk_home.size()))) return st;
  if ((st = dalloc(c, &c->blk_elems, blk_elems.size()))) return st;
  if ((st = dalloc(c, &c->node_row, node_row.size()))) return st;
  if ((st = dalloc(c, &c->node_slots, node_slots.size()))) return st;
  if ((st = dalloc(c, &c->d_perm_node, (size_t)Nn))) return st;
  if ((st = dalloc(c, &c->d_perm_elem, (size_t)Ne))) return st;
  CK(cudaMemcpyAsync(c->X64, X64.data(), X64.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->X32, X32.data(), X32.size() * sizeof(float4), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->conn, conn.data(), conn.size() * sizeof(int4), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->blk_ptr, blk_ptr.data(), blk_ptr.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->blk_home, blk_home.data(), blk_home.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->blk_elems, blk_elems.data(), blk_elems.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->node_row, node_row.data(), node_row.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->node_slots, node_slots.data(), node_slots.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_perm_node, c->perm_node.data(), Nn * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_perm_elem, c->perm_elem.data(), Ne * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  // the host vectors go out of scope: finish the copies first
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int alloc_state(FemCtx* c) {
  const size_t nd = (size_t)c->ndof_pad, Ne = (size_t)c->Ne;
  int st;
  if ((st = dalloc(c, &c->mat_id, Ne))) return st;
  if ((st = dalloc(c, &c->scale, Ne))) return st;
  if ((st = dalloc(c, &c->fixed, (size_t)c->Nn))) return st;
  if ((st = dalloc(c, &c->fixed_vals, nd))) return st;
  if ((st = dalloc(c, &c->fext, nd))) return st;
  if ((st = dalloc(c, &c->u, nd))) return st;
  if ((st = dalloc(c, &c->u_base, nd))) return st;
  if ((st = dalloc(c, &c->R, nd))) return st;
  if ((st = dalloc(c, &c->tmpd, nd))) return st;
  if ((st = dalloc(c, &c->payload, Ne * kPay))) return st;
  if ((st = dalloc(c, &c->ep_c, Ne * 6))) return st;
  if ((st = dalloc(c, &c->epe_c, Ne))) return st;
  if ((st = dalloc(c, &c->ep_t, Ne * 6))) return st;
  if ((st = dalloc(c, &c->epe_t, Ne))) return st;
  if ((st = dalloc(c, &c->r, nd))) return st;
  if ((st = dalloc(c, &c->x, nd))) return st;
  if ((st = dalloc(c, &c->p, nd))) return st;
  if ((st = dalloc(c, &c->y, nd))) return st;
  if ((st = dalloc(c, &c->dinv, nd))) return st;
  if ((st = dalloc(c, &c->tmpf, nd))) return st;
  if ((st = dalloc(c, &c->matD, (size_t)FEM_MAX_MATERIALS))) return st;
  if ((st = dalloc(c, &c->matF, (size_t)FEM_MAX_MATERIALS))) return st;
  // every reducing kernel's grid must fit: node blocks, float4 vector blocks, node-parallel blocks
  c->max_blocks = std::max({c->n_blocks, (c->ndof_pad / 4 + 255) / 256, (c->Nn + 255) / 256}) + 1;
  if ((st = dalloc(c, &c->partials, (size_t)N_SITES * 2 * c->max_blocks))) return st;
  if ((st = dalloc(c, &c->counters, (size_t)N_SITES))) return st;
  if ((st = dalloc(c, &c->scalars, (size_t)8))) return st;
  if ((st = dalloc(c, &c->cg, (size_t)1))) return st;
  CK(cudaMallocHost(reinterpret_cast<void**>(&c->h_cg), sizeof(CGState)));
  CK(cudaMallocHost(reinterpret_cast<void**>(&c->h_scalars), 8 * sizeof(double)));
  // default material: unit-scale linear elastic placeholder, every element id 0, scale 1
  std::vector<float> ones(Ne, 1.0f);
  CK(cudaMemcpyAsync(c->scale, ones.data(), Ne * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

template <typename T>
DevMat<T> to_dev(const FemMaterial& s) {
  DevMat<T> d;
  std::memset(&d, 0, sizeof(d));
  d.model = s.model;
  const double mu = s.E / (2.0 * (1.0 + s.nu));
  const double lam = s.E * s.nu / ((1.0 + s.nu) * (1.0 - 2.0 * s.nu));
  d.mu = (T)mu;
  d.lam = (T)lam;
  d.kappa = (T)(lam + 2.0 * mu / 3.0);
  d.sigma_y = (T)s.sigma_y;
  d.H = (T)s.H;
  d.C10 = (T)s.C10;
  d.C01 = (T)s.C01;
  d.invD1 = (T)(s.D1 > 1e-20 ? 1.0 / s.D1 : 0.0);
  d.fE = (T)s.fiber_E;
  d.n_fibers = s.n_fibers;
  for (int k = 0; k < 6; ++k) d.fa[k] = (T)s.fiber_dir[k / 3][k % 3];
  for (int k = 0; k < 36; ++k) d.C[k] = (T)s.C_voigt[k];
  return d;
}

// ───────────────────────── kernels wrappers ─────────────────────────

int eval_residual(FemCtx* c, double* fneg_out_int, double* rnorm2) {
  ResArgs a;
  a.m = c->mesh();
  a.matD = c->matD;
  a.u = c->u;
  a.f_ext = c->fext;
  a.R = c->R;
  a.fneg = fneg_out_int;
  a.payload = c->payload;
  a.ep_c = c->ep_c;
  a.epe_c = c->epe_c;
  a.ep_t = c->ep_t;
  a.epe_t = c->epe_t;
  a.rnorm2 = c->scalars;
  a.red = c->red();
  a.red_site = SITE_RES;
  ++c->n_launches; launch_residual(a, c->model_kind, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->h_scalars, c->scalars, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->tangent_valid = true;
  if (rnorm2) *rnorm2 = c->h_scalars[0];
  return FEM_OK;
}

int compute_dinv(FemCtx* c, int precond) {
  if (precond == FEM_PRECOND_JACOBI) {
    DiagArgs a;
    a.m = c->mesh();
    a.matF = c->matF;
    a.payload = c->payload;
    a.dinv = c->dinv;
    ++c->n_launches; launch_diag(a, c->model_kind, c->stream);
    CKL();
  } else {
    // identity on free DOFs: dinv = 1 where not fixed
    ++c->n_launches; launch_dinv_identity(c->dinv, c->fixed, c->Nn, c->stream);
    CKL();
  }
  return FEM_OK;
}

void enqueue_cg_iter(FemCtx* c) {
  MvArgs mv;
  mv.m = c->mesh();
  mv.matF = c->matF;
  mv.payload = c->payload;
  mv.x = c->p;
  mv.y = c->y;
  mv.cg = c->cg;
  mv.red = c->red();
  mv.red_site = SITE_MV;
  mv.mask_input = 1;
  const int ndof4 = c->ndof_pad / 4;
  launch_matvec(mv, c->model_kind, c->stream);
  launch_cg_update(c->x, c->r, c->p, c->y, c->dinv, ndof4, c->cg, c->red(), SITE_CGU, c->stream);
  launch_cg_pupdate(c->p, c->r, c->dinv, ndof4, c->cg, c->stream);
}

int ensure_cg_graph(FemCtx* c) {
  if (c->cg_graph && c->cg_graph_model == c->model_kind) return FEM_OK;
  if (c->cg_graph) {
    cudaGraphExecDestroy(c->cg_graph);
    c->cg_graph = nullptr;
  }
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < kCGBatch; ++i) enqueue_cg_iter(c);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (e != cudaSuccess) return set_err(c, FEM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&c->cg_graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_err(c, FEM_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
  c->cg_graph_model = c->model_kind;
  return FEM_OK;
}

// Solves K_T x = b (b: FP64 internal order, fixed DOFs zero) into c->x.
int run_pcg(FemCtx* c, const double* b_int, int precond, double rtol, int maxit, int* iters,
            double* rel) {
  if (!c->tangent_valid) return set_err(c, FEM_ERR_STATE, "no tangent state: evaluate forces first");
  int st;
  if ((st = compute_dinv(c, precond))) return st;
  if ((st = ensure_cg_graph(c))) return st;
  const int ndof4 = c->ndof_pad / 4;
  ++c->n_launches; launch_cg_init(b_int, c->r, c->x, c->p, c->dinv, ndof4, c->cg, rtol, maxit, c->red(), SITE_CGI,
                 c->stream);
  CKL();
  const int max_batches = maxit / kCGBatch + 2;
  CK(cudaMemcpyAsync(c->h_cg, c->cg, sizeof(CGState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int batches = 0;
  while (!c->h_cg->done && batches < max_batches) {
    CK(cudaGraphLaunch(c->cg_graph, c->stream));
    c->n_graphs++;
    CK(cudaMemcpyAsync(c->h_cg, c->cg, sizeof(CGState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    ++batches;
  }
  const CGState& h = *c->h_cg;
  c->n_cg_iters += h.iter;
  // kernels that did work: 3 per CG iteration (the rest of a batch exits at entry)
  c->n_launches += 3LL * h.iter;
  if (iters) *iters = h.iter;
  if (rel) *rel = h.rr0 > 0 ? std::sqrt(h.rr / h.rr0) : 0.0;
  if (h.done == 3) return set_err(c, FEM_ERR_NAN, "PCG breakdown (non-positive curvature or NaN) at iteration %d", h.iter);
  if (!h.done) return set_err(c, FEM_ERR_BUDGET, "PCG batch budget exhausted");
  if (h.done == 2) return FEM_NOT_CONVERGED;
  return FEM_OK;
}

int check_ctx(FemCtx* c) {
  if (!c) return FEM_ERR_INVALID;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return set_err(c, FEM_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return FEM_OK;
}

}  // namespace

int femb200::set_global_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_create_error = buf;
  return code;
}

// ───────────────────────── C ABI ─────────────────────────

extern "C" {

const char* fem_last_error(void* ctx) {
  if (!ctx) return g_create_error.c_str();
  return static_cast<FemCtx*>(ctx)->err.c_str();
}

int fem_ctx_create(const FemMeshDesc* desc, void** ctx_out) {
  FemCtx* c = nullptr;
  if (!desc || !ctx_out) return set_err(nullptr, FEM_ERR_INVALID, "null descriptor or output");
  *ctx_out = nullptr;
  if (desc->n_nodes <= 0 || desc->n_elements <= 0)
    return set_err(nullptr, FEM_ERR_INVALID, "mesh must have nodes and elements (got %lld, %lld)",
                   (long long)desc->n_nodes, (long long)desc->n_elements);
  if (desc->n_nodes > (1LL << 28) || desc->n_elements > (1LL << 28))
    return set_err(nullptr, FEM_ERR_INVALID, "mesh too large for 32-bit tables");
  if (!desc->X || !desc->conn) return set_err(nullptr, FEM_ERR_INVALID, "null X or conn");
  const int nb = desc->nodes_per_block == 0 ? 256 : desc->nodes_per_block;
  if (nb != 128 && nb != 256 && nb != 512)
    return set_err(nullptr, FEM_ERR_INVALID, "nodes_per_block must be 128, 256 or 512");
  for (int64_t i = 0; i < 4 * desc->n_elements; ++i)
    if (desc->conn[i] < 0 || desc->conn[i] >= desc->n_nodes)
      return set_err(nullptr, FEM_ERR_INVALID, "connectivity entry %lld = %d out of range [0, %lld)",
                     (long long)i, desc->conn[i], (long long)desc->n_nodes);
  for (int64_t e = 0; e < desc->n_elements; ++e) {
    const int32_t* cn = desc->conn + 4 * e;
    for (int a = 0; a < 4; ++a)
      for (int b = a + 1; b < 4; ++b)
        if (cn[a] == cn[b])
          return set_err(nullptr, FEM_ERR_INVALID, "element %lld repeats node %d", (long long)e, cn[a]);
  }
  for (int64_t i = 0; i < 3 * desc->n_nodes; ++i)
    if (!std::isfinite(desc->X[i]))
      return set_err(nullptr, FEM_ERR_INVALID, "non-finite coordinate at %lld", (long long)i);
  cudaError_t e = cudaSetDevice(desc->device);
  if (e != cudaSuccess) return set_err(nullptr, FEM_ERR_CUDA, "cudaSetDevice(%d): %s", desc->device, cudaGetErrorString(e));
  c = new FemCtx();
  c->device = desc->device;
  c->Nn = (int)desc->n_nodes;
  c->Ne = (int)desc->n_elements;
  c->nb = nb;
  c->ndof = 3 * c->Nn;
  c->ndof_pad = (c->ndof + 3) / 4 * 4;
  if (desc->stream) {
    c->stream = (cudaStream_t)desc->stream;
  } else {
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      int st = set_err(nullptr, FEM_ERR_CUDA, "stream create: %s", cudaGetErrorString(e));
      delete c;
      return st;
    }
    c->own_stream = true;
  }
  int st = build_tables(c, desc->X, desc->conn);
  if (!st) st = alloc_state(c);
  if (st) {
    g_create_error = c->err;
    free_ctx(c);
    return st;
  }
  *ctx_out = c;
  return FEM_OK;
}

int fem_ctx_destroy(void* ctx) {
  free_ctx(static_cast<FemCtx*>(ctx));
  return FEM_OK;
}

int fem_ctx_info(void* ctx, int64_t* out) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  if (!c || !out) return FEM_ERR_INVALID;
  out[0] = c->Nn;
  out[1] = c->Ne;
  out[2] = c->n_blocks;
  out[3] = c->blk_entries;
  out[4] = c->nb;
  out[5] = (int64_t)c->bytes;
  return FEM_OK;
}

int fem_ctx_stats(void* ctx, int64_t* out) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  if (!c || !out) return FEM_ERR_INVALID;
  out[0] = c->n_launches;
  out[1] = c->n_cg_iters;
  out[2] = c->n_res_evals;
  out[3] = c->n_graphs;
  return FEM_OK;
}

void* fem_ctx_stream(void* ctx) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  return c ? (void*)c->stream : nullptr;
}

int fem_set_materials(void* ctx, const FemMaterial* table, int32_t n, const uint8_t* elem_mat,
                      const float* elem_scale) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!table || n <= 0 || n > FEM_MAX_MATERIALS)
    return set_err(c, FEM_ERR_INVALID, "material table size %d outside [1, %d]", n, FEM_MAX_MATERIALS);
  bool has_j2 = false;
  int kind = table[0].model;
  std::vector<DevMat<double>> md(FEM_MAX_MATERIALS);
  std::vector<DevMat<float>> mf(FEM_MAX_MATERIALS);
  for (int i = 0; i < n; ++i) {
    const FemMaterial& s = table[i];
    if (s.model < FEM_LINEAR_ELASTIC || s.model > FEM_FIBRE_MOONEY_RIVLIN)
      return set_err(c, FEM_ERR_INVALID, "material %d: unknown model %d", i, s.model);
    if (s.model == FEM_LINEAR_ELASTIC || s.model == FEM_NEO_HOOKEAN || s.model == FEM_J2) {
      if (!(s.E > 0)) return set_err(c, FEM_ERR_INVALID, "material %d: E must be > 0 (got %g)", i, s.E);
      if (!(s.nu > -1.0 && s.nu < 0.5))
        return set_err(c, FEM_ERR_INVALID, "material %d: nu must be in (-1, 0.5) (got %g)", i, s.nu);
    }
    if (s.model == FEM_J2) {
      if (!(s.sigma_y > 0)) return set_err(c, FEM_ERR_INVALID, "material %d: yield stress must be > 0", i);
      if (!(s.H >= 0)) return set_err(c, FEM_ERR_INVALID, "material %d: hardening modulus must be >= 0", i);
      has_j2 = true;
    }
    if ((s.model == FEM_MOONEY_RIVLIN || s.model == FEM_FIBRE_MOONEY_RIVLIN) &&
        (!(s.C10 + s.C01 > 0) || s.D1 < 0))
      return set_err(c, FEM_ERR_INVALID, "material %d: need C10 + C01 > 0 and D1 >= 0", i);
    if (s.model == FEM_FIBRE_MOONEY_RIVLIN && (s.n_fibers < 0 || s.n_fibers > 2))
      return set_err(c, FEM_ERR_INVALID, "material %d: n_fibers must be 0..2", i);
    if (s.model != kind) kind = -1;
    md[i] = to_dev<double>(s);
    mf[i] = to_dev<float>(s);
  }
  std::vector<uint8_t> ids(c->Ne, 0);
  std::vector<float> sc(c->Ne, 1.0f);
  for (int e = 0; e < c->Ne; ++e) {
    const int eu = c->perm_elem[e];
    if (elem_mat) {
      if (elem_mat[eu] >= n)
        return set_err(c, FEM_ERR_INVALID, "element %d: material id %d >= table size %d", eu, elem_mat[eu], n);
      ids[e] = elem_mat[eu];
    }
    if (elem_scale) {
      if (!(elem_scale[eu] > 0.f) || !std::isfinite(elem_scale[eu]))
        return set_err(c, FEM_ERR_INVALID, "element %d: modulus scale must be finite and > 0", eu);
      sc[e] = elem_scale[eu];
    }
  }
  // a mixed table whose elements all use one model runs the specialised kernels
  if (kind == -1 && elem_mat) {
    int used = -2;
    for (int e = 0; e < c->Ne && used != -1; ++e) {
      const int m = table[ids[e]].model;
      used = (used == -2 || used == m) ? m : -1;
    }
    kind = used;
  } else if (kind == -1 && !elem_mat) {
    kind = table[0].model;
  }
  CK(cudaMemcpyAsync(c->matD, md.data(), md.size() * sizeof(DevMat<double>), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->matF, mf.data(), mf.size() * sizeof(DevMat<float>), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->mat_id, ids.data(), ids.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->scale, sc.data(), sc.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->model_kind = kind;
  c->has_j2 = has_j2;
  c->materials_set = true;
  c->tangent_valid = false;
  return FEM_OK;
}

int fem_set_bc(void* ctx, const uint8_t* fixed_mask, const double* fixed_values, const double* f_ext) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (fixed_mask) {
    ++c->n_launches; launch_gather_mask(fixed_mask, c->fixed, c->d_perm_node, c->Nn, c->stream);
    CKL();
  }
  if (fixed_values) {
    ++c->n_launches; launch_gather_d(fixed_values, c->fixed_vals, c->d_perm_node, c->Nn, c->stream);
    CKL();
  }
  if (f_ext) {
    ++c->n_launches; launch_gather_d(f_ext, c->fext, c->d_perm_node, c->Nn, c->stream);
    CKL();
  }
  CK(cudaStreamSynchronize(c->stream));
  c->tangent_valid = false;
  return FEM_OK;
}

int fem_apply_bc(void* ctx) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  ++c->n_launches; launch_apply_bc(c->u, c->fixed_vals, c->fixed, c->Nn, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int fem_set_displacement(void* ctx, const double* u) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!u) return set_err(c, FEM_ERR_INVALID, "null displacement");
  ++c->n_launches; launch_gather_d(u, c->u, c->d_perm_node, c->Nn, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  c->tangent_valid = false;
  return FEM_OK;
}

int fem_get_displacement(void* ctx, double* u_out) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!u_out) return set_err(c, FEM_ERR_INVALID, "null output");
  ++c->n_launches; launch_scatter_d(c->u, u_out, c->d_perm_node, c->Nn, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int fem_reference_quantities(void* ctx, double* dNdX_out, double* vol_out) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  ++c->n_launches; launch_refq(c->mesh(), c->d_perm_elem, dNdX_out, vol_out, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int fem_compute_stress(void* ctx, const double* u, double* F_out, double* sigma_out) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!c->materials_set) return set_err(c, FEM_ERR_STATE, "materials not set");
  if (u) {
    ++c->n_launches; launch_gather_d(u, c->u, c->d_perm_node, c->Nn, c->stream);
    CKL();
  }
  ++c->n_launches; launch_stress(c->mesh(), c->matD, c->model_kind, c->u, c->ep_c, c->epe_c, c->d_perm_elem, F_out,
                sigma_out, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int fem_element_forces(void* ctx, const double* u, double* f_out, double* residual_out, double* rnorm) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!c->materials_set) return set_err(c, FEM_ERR_STATE, "materials not set");
  if (u) {
    ++c->n_launches; launch_gather_d(u, c->u, c->d_perm_node, c->Nn, c->stream);
    CKL();
  }
  double r2 = 0;
  if ((st = eval_residual(c, f_out ? c->tmpd : nullptr, &r2))) return st;
  if (f_out) {
    ++c->n_launches; launch_scatter_d(c->tmpd, f_out, c->d_perm_node, c->Nn, c->stream);
    CKL();
  }
  if (residual_out) {
    ++c->n_launches; launch_scatter_d(c->R, residual_out, c->d_perm_node, c->Nn, c->stream);
    CKL();
  }
  CK(cudaStreamSynchronize(c->stream));
  if (rnorm) *rnorm = std::sqrt(r2);
  return FEM_OK;
}

int fem_tangent_matvec(void* ctx, const float* xin, float* yout) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!c->tangent_valid) return set_err(c, FEM_ERR_STATE, "no tangent state: evaluate forces first");
  if (!xin || !yout) return set_err(c, FEM_ERR_INVALID, "null vector");
  ++c->n_launches; launch_gather_f(xin, c->tmpf, c->d_perm_node, c->Nn, c->stream);
  CKL();
  MvArgs mv;
  mv.m = c->mesh();
  mv.matF = c->matF;
  mv.payload = c->payload;
  mv.x = c->tmpf;
  mv.y = c->y;
  mv.cg = nullptr;
  mv.red = c->red();
  mv.red_site = SITE_MV;
  mv.mask_input = 1;
  ++c->n_launches; launch_matvec(mv, c->model_kind, c->stream);
  CKL();
  ++c->n_launches; launch_scatter_f(c->y, yout, c->d_perm_node, c->Nn, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int fem_pcg(void* ctx, int32_t precond, const double* r, double* du, double rtol, int32_t maxit,
            int32_t* iters, double* rel) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!r || !du) return set_err(c, FEM_ERR_INVALID, "null vector");
  if (maxit <= 0 || !(rtol > 0)) return set_err(c, FEM_ERR_INVALID, "need max_iterations > 0 and rtol > 0");
  // caller order -> internal order, fixed DOFs of the right-hand side zeroed
  ++c->n_launches; launch_gather_d_masked(r, c->tmpd, c->d_perm_node, c->fixed, c->Nn, c->stream);
  CKL();
  int it = 0;
  double rl = 0;
  st = run_pcg(c, c->tmpd, precond, rtol, maxit, &it, &rl);
  if (iters) *iters = it;
  if (rel) *rel = rl;
  if (st && st != FEM_NOT_CONVERGED) return st;
  ++c->n_launches; launch_scatter_f2d(c->x, du, c->d_perm_node, c->Nn, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  return st;
}

void fem_default_solve_params(FemSolveParams* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->max_iterations = 50;
  p->tol = 1e-8;
  p->line_search = FEM_LS_GUARDED;
  p->precond = FEM_PRECOND_JACOBI;
  p->cg_max_iterations = 20000;
  p->cg_rtol_min = 1e-5;
  p->cg_rtol_max = 1e-1;
  p->auto_commit = 1;
  p->verbose = 0;
}

int fem_newton_solve(void* ctx, const FemSolveParams* prm_in, FemSolveResult* res) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!c->materials_set) return set_err(c, FEM_ERR_STATE, "materials not set");
  FemSolveParams prm;
  if (prm_in)
    prm = *prm_in;
  else
    fem_default_solve_params(&prm);
  if (prm.max_iterations <= 0 || !(prm.tol > 0))
    return set_err(c, FEM_ERR_INVALID, "need max_iterations > 0 and tol > 0");
  FemSolveResult out;
  std::memset(&out, 0, sizeof(out));
  // Change of the prescribed values in this solve.  It is carried by the first
  // Newton step (K_ff du_f = R - K_fc du_c): moving only the boundary nodes would
  // leave a one-element layer at large strain, which yields under J2 and stalls
  // Newton.  Relative convergence is measured, as in the reference
  // (static_solver.py:159-218), against the residual of the state it evaluates
  // first: the previous u with the new prescribed values applied.
  ++c->n_launches; launch_bc_delta(c->u, c->fixed_vals, c->fixed, c->tmpf, c->Nn, c->red(), SITE_AUX,
                  c->scalars + 1, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->h_scalars + 1, c->scalars + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const bool has_dc = c->h_scalars[1] > 0.0;
  double r2 = 0;
  double ref_norm = -1.0;
  int it0 = 0;
  if (has_dc) {
    CK(cudaMemcpyAsync(c->u_base, c->u, c->ndof_pad * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    ++c->n_launches; launch_apply_bc(c->u, c->fixed_vals, c->fixed, c->Nn, c->stream);
    CKL();
    if ((st = eval_residual(c, nullptr, &r2))) return st;
    ref_norm = std::sqrt(r2);
    CK(cudaMemcpyAsync(c->u, c->u_base, c->ndof_pad * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if ((st = eval_residual(c, nullptr, &r2))) return st;
    out.residual_evals = 2;
    if (!std::isfinite(ref_norm) || !std::isfinite(r2)) {
      if (res) *res = out;
      return set_err(c, FEM_ERR_NAN, "NaN/Inf residual at iteration 0");
    }
    MvArgs mv;
    mv.m = c->mesh();
    mv.matF = c->matF;
    mv.payload = c->payload;
    mv.x = c->tmpf;
    mv.y = c->y;
    mv.cg = nullptr;
    mv.red = c->red();
    mv.red_site = SITE_MV;
    mv.mask_input = 0;
    ++c->n_launches; launch_matvec(mv, c->model_kind, c->stream);
    CKL();
    ++c->n_launches; launch_rhs_minus(c->R, c->y, c->fixed, c->tmpd, c->Nn, c->stream);
    CKL();
    // the predictor fixes the elastic state of the step: solve it to 1e-3
    const double eta = std::max(1e-3, prm.cg_rtol_min);
    int cgit = 0;
    double cgrel = 0;
    st = run_pcg(c, c->tmpd, prm.precond, eta, prm.cg_max_iterations, &cgit, &cgrel);
    out.cg_iterations += cgit;
    if (st && st != FEM_NOT_CONVERGED) return st;
    ++c->n_launches; launch_u_update(c->u, c->u_base, c->x, 1.0, c->ndof, c->stream);
    CKL();
    it0 = 1;
  }
  // apply_boundary_conditions (core/mesh.py:321-327): prescribed DOFs held exactly
  ++c->n_launches; launch_apply_bc(c->u, c->fixed_vals, c->fixed, c->Nn, c->stream);
  CKL();
  if ((st = eval_residual(c, nullptr, &r2))) return st;
  out.residual_evals += 1;
  double res_norm = std::sqrt(r2);
  if (!std::isfinite(res_norm)) {
    if (res) *res = out;
    return set_err(c, FEM_ERR_NAN, "NaN/Inf residual at iteration %d", it0);
  }
  if (ref_norm < 0) ref_norm = res_norm;
  const double ref = ref_norm > 1e-20 ? ref_norm : 1.0;
  out.first_residual = ref_norm;
  double rel = res_norm / ref;
  double prev_norm = res_norm;
  int it = 0;
  bool converged = false;
  for (it = it0; it < prm.max_iterations; ++it) {
    rel = res_norm / ref;
    if (prm.verbose) fprintf(stderr, "[femb200] Newton %d: |R| = %.4e rel = %.4e\n", it, res_norm, rel);
    if (prm.progress) {
      if (prm.progress(prm.progress_user, it, res_norm, rel) == 0) {
        out.cancelled = 1;
        out.iterations = it;
        out.residual = res_norm;
        out.relative_residual = rel;
        if (res) *res = out;
        return FEM_OK;
      }
    }
    if (rel < prm.tol) {
      converged = true;
      break;
    }
    // inexact-Newton forcing term: aim at the target, follow the residual's
    // contraction (Eisenstat-Walker), and solve tightly (1e-3) when the
    // residual did not drop — loose solves there let J2 iterations wander
    const bool dropped = it > it0 && res_norm < prev_norm;
    const double ew = dropped ? 0.9 * (res_norm / prev_norm) * (res_norm / prev_norm) : 1e-3;
    double eta = std::max(0.1 * prm.tol * ref / res_norm, ew);
    eta = std::min(std::max(eta, prm.cg_rtol_min), prm.cg_rtol_max);
    int cgit = 0;
    double cgrel = 0;
    st = run_pcg(c, c->R, prm.precond, eta, prm.cg_max_iterations, &cgit, &cgrel);
    out.cg_iterations += cgit;
    if (st == FEM_ERR_NAN) {
      // the reference breaks out of Newton when the linear solve fails (static_solver.py:229-233)
      break;
    }
    if (st && st != FEM_NOT_CONVERGED) return st;
    if (prm.verbose) fprintf(stderr, "[femb200]   PCG: %d its, rel %.3e (eta %.1e)\n", cgit, cgrel, eta);
    CK(cudaMemcpyAsync(c->u_base, c->u, c->ndof_pad * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    double alpha = 1.0;
    double trial = res_norm;
    const int n_trials = prm.line_search == FEM_LS_NONE ? 1 : 5;
    for (int ls = 0; ls < n_trials; ++ls) {
      ++c->n_launches; launch_u_update(c->u, c->u_base, c->x, alpha, c->ndof, c->stream);
      CKL();
      if ((st = eval_residual(c, nullptr, &r2))) return st;
      out.residual_evals++;
      trial = std::sqrt(r2);
      bool accept;
      if (prm.line_search == FEM_LS_REFERENCE)
        accept = trial < res_norm;
      else
        accept = std::isfinite(trial) && trial < 1e6 * res_norm;
      if (accept) break;
      alpha *= 0.5;
    }
    prev_norm = res_norm;
    res_norm = trial;
    if (!std::isfinite(res_norm)) {
      out.iterations = it + 1;
      out.residual = res_norm;
      if (res) *res = out;
      return set_err(c, FEM_ERR_NAN, "NaN/Inf residual at Newton iteration %d", it + 1);
    }
  }
  if (converged && c->has_j2 && prm.auto_commit) {
    CK(cudaMemcpyAsync(c->ep_c, c->ep_t, (size_t)6 * c->Ne * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->epe_c, c->epe_t, (size_t)c->Ne * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  out.converged = converged ? 1 : 0;
  out.iterations = std::min(it + 1, prm.max_iterations);
  out.residual = res_norm;
  out.relative_residual = res_norm / ref;
  if (res) *res = out;
  return converged ? FEM_OK : FEM_NOT_CONVERGED;
}

int fem_profile_kernels(void* ctx, int32_t reps, double* ms_out) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!c->tangent_valid) return set_err(c, FEM_ERR_STATE, "no tangent state: evaluate forces first");
  if (reps <= 0 || !ms_out) return set_err(c, FEM_ERR_INVALID, "need reps > 0 and an output array");
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int ndof4 = c->ndof_pad / 4;
  // a CG state that never finishes, so the fused kernels do their full work
  CGState hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.rz = 1.0;
  hs.rr = 1.0;
  hs.rr0 = 1.0;
  hs.tol2 = 0.0;
  hs.alpha = 1e-30;
  hs.beta = 0.0;
  hs.max_iter = 1 << 30;
  auto reset_cg = [&]() { return cudaMemcpyAsync(c->cg, &hs, sizeof(hs), cudaMemcpyHostToDevice, c->stream); };
  MvArgs mv;
  mv.m = c->mesh();
  mv.matF = c->matF;
  mv.payload = c->payload;
  mv.x = c->p;
  mv.y = c->y;
  mv.cg = c->cg;
  mv.red = c->red();
  mv.red_site = SITE_MV;
  mv.mask_input = 1;
  ResArgs ra;
  ra.m = c->mesh();
  ra.matD = c->matD;
  ra.u = c->u;
  ra.f_ext = c->fext;
  ra.R = c->tmpd;
  ra.fneg = nullptr;
  ra.payload = c->payload;
  ra.ep_c = c->ep_c;
  ra.epe_c = c->epe_c;
  ra.ep_t = c->ep_t;
  ra.epe_t = c->epe_t;
  ra.rnorm2 = c->scalars + 2;
  ra.red = c->red();
  ra.red_site = SITE_RES;
  for (int k = 0; k < 4; ++k) {
    CK(reset_cg());
    for (int w = 0; w < 2; ++w) {
      if (k == 0) launch_matvec(mv, c->model_kind, c->stream);
      if (k == 1) launch_residual(ra, c->model_kind, c->stream);
      if (k == 2) launch_cg_update(c->tmpf, c->r, c->p, c->y, c->dinv, ndof4, c->cg, c->red(), SITE_CGU, c->stream);
      if (k == 3) launch_cg_pupdate(c->tmpf, c->r, c->dinv, ndof4, c->cg, c->stream);
    }
    CK(reset_cg());
    CK(cudaEventRecord(e0, c->stream));
    for (int r = 0; r < reps; ++r) {
      if (k == 0) launch_matvec(mv, c->model_kind, c->stream);
      if (k == 1) launch_residual(ra, c->model_kind, c->stream);
      if (k == 2) launch_cg_update(c->tmpf, c->r, c->p, c->y, c->dinv, ndof4, c->cg, c->red(), SITE_CGU, c->stream);
      if (k == 3) launch_cg_pupdate(c->tmpf, c->r, c->dinv, ndof4, c->cg, c->stream);
    }
    CK(cudaEventRecord(e1, c->stream));
    CKL();
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    ms_out[k] = ms / reps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->tangent_valid = true;
  return FEM_OK;
}

int fem_commit_history(void* ctx) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  CK(cudaMemcpyAsync(c->ep_c, c->ep_t, (size_t)6 * c->Ne * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->epe_c, c->epe_t, (size_t)c->Ne * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int fem_reset_history(void* ctx) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  CK(cudaMemsetAsync(c->ep_c, 0, (size_t)6 * c->Ne * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->epe_c, 0, (size_t)c->Ne * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->ep_t, 0, (size_t)6 * c->Ne * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->epe_t, 0, (size_t)c->Ne * sizeof(double), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->tangent_valid = false;
  return FEM_OK;
}

int fem_get_history(void* ctx, double* ep_out, double* epe_out) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  std::vector<double> ep((size_t)6 * c->Ne), epe(c->Ne);
  CK(cudaMemcpyAsync(ep.data(), c->ep_c, ep.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(epe.data(), c->epe_c, epe.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // internal SoA (xx,yy,zz,yz,xz,xy) -> caller (Ne,3,3) / (Ne)
  std::vector<double> full((size_t)9 * c->Ne), e1(c->Ne);
  for (int e = 0; e < c->Ne; ++e) {
    const int eu = c->perm_elem[e];
    double s[6];
    for (int k = 0; k < 6; ++k) s[k] = ep[(size_t)k * c->Ne + e];
    double* F = &full[(size_t)9 * eu];
    F[0] = s[0]; F[4] = s[1]; F[8] = s[2];
    F[5] = F[7] = s[3];
    F[2] = F[6] = s[4];
    F[1] = F[3] = s[5];
    e1[eu] = epe[e];
  }
  if (ep_out) CK(cudaMemcpyAsync(ep_out, full.data(), full.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (epe_out) CK(cudaMemcpyAsync(epe_out, e1.data(), e1.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

}  // extern "C"
