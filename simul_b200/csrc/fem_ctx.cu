// Host driver and C ABI of the TET4 static-solve path (include/femb200.h).
//
// Set-up (fem_ctx_create) renumbers nodes by Morton code, groups elements by
// the block of their lowest node, and builds the node-block gather tables the
// element kernels use.  Callers keep their own numbering: every per-call array
// is permuted on entry and exit.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <thread>
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

enum { SITE_RES = 0, SITE_MV = 1, SITE_CGI = 2, SITE_CGU = 3, SITE_AUX = 4, SITE_RZ = 5, SITE_RZ2 = 6, N_SITES = 7 };
// captured CG iteration graphs: Jacobi / identity preconditioner, two-level,
// learned (flexible PCG)
enum { GRAPH_JACOBI = 0, GRAPH_TWO_LEVEL = 1, GRAPH_LEARNED = 2, N_GRAPHS = 3 };
// CG iterations per captured graph launch (Jacobi needs hundreds per solve;
// the two-level and learned preconditioners tens, so their graphs are shorter
// and fewer early-exit iterations run after convergence)
constexpr int kCGBatch = 32;
constexpr int kCGBatchShort = 12;
inline int cg_batch(int kind) { return kind == 0 ? kCGBatch : kCGBatchShort; }
inline int step_chunks(int n_nodes) { return (n_nodes + kStepThreads - 1) / kStepThreads; }

struct FemCtx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int Nn = 0, Ne = 0, nb = 256, n_blocks = 0;
  int npe = 4;                 // nodes per element: 4 TET4, 8 HEX8
  int ngp = 1;                 // Gauss points per element: 1 TET4, 8 HEX8
  size_t Nq = 0;               // integration points Ne * ngp (payload and J2 history rows)
  double* stage_d = nullptr;   // two-phase FP64 residual: element slot forces in node_slots order
  bool res_two_phase = true;   // TET4: two-phase FP64 residual (else the fused node-block kernel)
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
  int4* spos = nullptr;
  int max_slots = 0;
  uint8_t* fixed = nullptr;
  double* fixed_vals = nullptr;
  double* fixed_vals_full = nullptr;  // last values given to fem_set_bc (fem_set_load_scale scales them)
  double* fext_full = nullptr;
  double* fext = nullptr;
  double* u = nullptr;
  double* u_base = nullptr;
  double* R = nullptr;
  // load-step extrapolation (FEM_OPT_EXTRAPOLATE): the end state of the last
  // converged solve, its change of u, and this solve's starting u
  bool extrap = false;
  bool extrap_ready = false;
  double* u_last = nullptr;
  double* du_last = nullptr;
  double* u_start = nullptr;
  // learned FPCG hand-over: the flexible iterate and its residual in FP64
  float* ho_x = nullptr;
  double* ho_rhs = nullptr;
  int64_t n_handovers = 0;
  double* tmpd = nullptr;
  float* payload = nullptr;
  double* ep_c = nullptr;
  double* epe_c = nullptr;
  double* ep_t = nullptr;
  double* epe_t = nullptr;
  // FP32 node vectors, one float4 per node
  float *r = nullptr, *x = nullptr, *p = nullptr, *y = nullptr, *dinv = nullptr, *tmpf = nullptr;
  float4* stage = nullptr;  // [4 Ne] two-phase matvec slot vectors
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
  cudaGraphExec_t cg_graph[N_GRAPHS] = {nullptr, nullptr, nullptr};
  // whole-solve graphs: a conditional WHILE node repeats kLoopIters CG
  // iterations until the device-side CG state says done (null: not
  // available, the batched graphs above are used)
  cudaGraphExec_t loop_graph[N_GRAPHS] = {nullptr, nullptr, nullptr};
  bool use_loop_graph = true;
  int64_t n_loop_graphs = 0;   // PCG solves run as one whole-solve graph launch
  int cg_graph_model[N_GRAPHS] = {-2, -2, -2};
  int cg_graph_variant[N_GRAPHS] = {-1, -1, -1};
  int cg_graph_flags[N_GRAPHS] = {-1, -1, -1};
  // fused CG step (one cooperative kernel after each matvec; off by default:
  // on B200 its four grid barriers and the cooperative launch cost more than
  // the launch gaps of the kernel chain they replace): wanted by the
  // option, still available (a refused capture turns it off), and not while
  // fem_batch_solve runs several contexts at once (cooperative grids of
  // concurrent contexts could wait on each other's SMs)
  bool fused_step = false;
  bool fused_ok = true;
  // programmatic dependent launch between the CG chain's kernels inside the
  // captured graphs (a refused capture turns it off)
  bool pdl = true;
  bool pdl_ok = true;
  // two-level CG: direction by recurrence in the matvec's node gather
  bool direction_recurrence = true;
  // two-level smoother: nodal 3x3 block inverse instead of 1 / diag
  bool block_jacobi = true;
  float* boff = nullptr;  // [Nn] float4 off-diagonals (01, 02, 12) of the block inverse
  bool in_batch = false;
  unsigned int* step_bar = nullptr;  // [4] grid barrier words
  double* jac_part = nullptr;        // [2 n_chunks] Jacobi step shares
  double* tl_part = nullptr;         // two-level step: [n_cells r_slices + n_chunks]

  // learned preconditioner: node graph, features, weights, activations
  MpnnDev mdev{};
  bool mpnn_built = false;
  bool mpnn_feat_valid = false;
  bool mpnn_has_weights = false;
  bool learned_coarse = true;   // add the two-level coarse correction to M(r)
  std::vector<void*> mpnn_bufs;
  float* mpnn_w = nullptr;
  __nv_bfloat16 *We_p = nullptr, *Wl_p = nullptr, *WlT_p = nullptr;
  float* cfeat = nullptr;
  std::vector<double> elem_modulus;  // internal element order
  int64_t n_fallbacks = 0;
  int64_t n_alt_steps = 0;    // learned FPCG steps that used the Jacobi (+ coarse) direction
  int64_t n_learned_steps = 0;
  float* zalt = nullptr;      // [Nn] float4 alternative direction of learned FPCG
  int* h_err = nullptr;
  // training state: backward buffers, gradient, Adam moments, per-sample vectors
  MpnnTrain mtrain{};
  bool mpnn_train_ready = false;
  float *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  int adam_t = 0;
  float *tr_r = nullptr, *tr_e = nullptr, *tr_z = nullptr, *tr_q = nullptr, *tr_g = nullptr;
  double* tr_scal = nullptr;  // [0] loss sum, [1] dL/dz scale

  // two-level preconditioner: coarse lattice tables (built on first use),
  // dense coarse operator and its inverse, dense-inverse work space
  CoarseDev cdev{};
  bool coarse_built = false;
  bool coarse_valid = false;   // Ainv matches the current tangent policy
  bool coarse_have_inverse = false;  // an inverse of this lattice has been formed
  int64_t n_coarse_kept = 0;   // refreshes whose operator was not SPD (the last inverse kept)
  int64_t n_coarse_fallbacks = 0;  // two-level solves run as Jacobi-PCG (no SPD coarse operator)
  int coarse_cell_voxels = 8;  // lattice cell edge in mesh lengths
  bool coarse_bf16 = false;    // store the coarse inverse in BF16
  int coarse_max_nodes = 4096; // the lattice cell grows until at most this many coarse nodes remain
  int coarse_reuse = -1;       // PCG solves one assembly serves; 0 = once per state, -1 = adaptive
  double coarse_base_ipd = -1;  // CG iterations per decade right after the last assembly
  int coarse_uses = 0;
  double coarse_H = 0.0;
  int64_t n_coarse_assemblies = 0;
  std::vector<uint8_t> fixed_host;  // last constraint pattern (internal order)
  double coarse_ms_last = 0.0;
  double coarse_ms_assembly = 0.0;   // of which cell blocks + dense assembly
  cudaEvent_t coarse_ev[3] = {nullptr, nullptr, nullptr};
  std::vector<void*> coarse_bufs;
  // coarse inverse (fem_dense.cu: blocked Cholesky, W = L^-1, Ac^-1 = W^T W):
  // 0 and 1 (default) in FP64, 2 and 3 in FP32 (option values of earlier
  // library versions, which chose between library routines)
  int coarse_inverse = 1;
  void* dense_work = nullptr;   // padded factor and W (and the FP32 result)
  size_t dense_bytes = 0;
  int* dense_info = nullptr;    // first non-positive pivot, 0 if none
  DenseSched dense_sched;       // streams and events of the dense inverse
  std::vector<int> coarse_row_first;  // Ac's row envelope (lowest coupled DOF per row)
  int* h_info = nullptr;
  // matvec variant: forced by fem_set_option (>= 0) or chosen by timing all
  int mv_forced = -1;
  int mv_variant = MV_FUSED;
  bool mv_tuned = false;
  int mv_tuned_model = -2;
  double mv_ns[MV_N_VARIANTS] = {0.0, 0.0, 0.0, 0.0, 0.0};
  // element-block matvec (TET4): tables for blocks of eb_size elements (0:
  // not built), the block size forced by FEM_OPT_EB_SIZE (0: timed choice
  // among kEbSizes), and the timed ns per launch of each candidate size
  EbDev ebdev{};
  std::vector<void*> eb_bufs;
  // warp-aggregated two-phase matvec tables (TET4; built when selected or timed)
  WaggDev wadev{};
  std::vector<void*> wa_bufs;
  int eb_size = 0;
  int eb_forced = 0;
  double eb_ns[4] = {0.0, 0.0, 0.0, 0.0};

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
    m.max_slots = max_slots;
    m.spos = spos;
    m.npe = npe;
    m.slot_shift = npe == 8 ? 3 : 2;
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

// Two CUDA events destroyed on every return path.
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t create() {
    cudaError_t e = cudaEventCreate(&a);
    return e == cudaSuccess ? cudaEventCreate(&b) : e;
  }
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
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
  for (int k = 0; k < N_GRAPHS; ++k) {
    if (c->cg_graph[k]) cudaGraphExecDestroy(c->cg_graph[k]);
    if (c->loop_graph[k]) cudaGraphExecDestroy(c->loop_graph[k]);
  }
  for (void* p : c->coarse_bufs)
    if (p) cudaFree(p);
  for (void* p : c->mpnn_bufs)
    if (p) cudaFree(p);
  for (void* p : c->eb_bufs)
    if (p) cudaFree(p);
  for (void* p : c->wa_bufs)
    if (p) cudaFree(p);
  if (c->h_err) cudaFreeHost(c->h_err);
  if (c->dense_work) cudaFree(c->dense_work);
  if (c->dense_info) cudaFree(c->dense_info);
  c->dense_sched.release();
  if (c->h_info) cudaFreeHost(c->h_info);
  for (cudaEvent_t ev : c->coarse_ev)
    if (ev) cudaEventDestroy(ev);
  if (c->stage) cudaFree(c->stage);
  if (c->stage_d) cudaFree(c->stage_d);
  if (c->u_last) cudaFree(c->u_last);
  if (c->du_last) cudaFree(c->du_last);
  if (c->u_start) cudaFree(c->u_start);
  if (c->ho_x) cudaFree(c->ho_x);
  if (c->ho_rhs) cudaFree(c->ho_rhs);
  if (c->spos) cudaFree(c->spos);
  void* ptrs[] = {c->X64, c->X32, c->conn, c->mat_id, c->scale, c->blk_ptr, c->blk_home,
                  c->blk_elems, c->node_row, c->node_slots, c->fixed, c->fixed_vals, c->fext,
                  c->fixed_vals_full, c->fext_full,
                  c->u, c->u_base, c->R, c->tmpd, c->payload, c->ep_c, c->epe_c, c->ep_t,
                  c->epe_t, c->r, c->x, c->p, c->y, c->dinv, c->tmpf, c->d_perm_node,
                  c->d_perm_elem, c->matD, c->matF, c->partials, c->counters, c->scalars, c->cg,
                  c->step_bar, c->jac_part, c->boff};
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
  const int npe = c->npe;
  const int sh = npe == 8 ? 3 : 2;              // slot bits in the (element, slot) codes
  const uint32_t smask = (1u << sh) - 1u;
  for (int e = 0; e < Ne; ++e) {
    int mn = Nn;
    double cen[3] = {0, 0, 0};
    for (int k = 0; k < npe; ++k) {
      const int nu = conn_user[npe * e + k];
      mn = std::min(mn, iperm[nu]);
      for (int d = 0; d < 3; ++d) cen[d] += X[3 * nu + d] / npe;
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
  // npe / 4 int4 per element (HEX8: vertices 0-3, then 4-7)
  const int cw = npe / 4;
  std::vector<int4> conn((size_t)cw * Ne);
  std::vector<int> ehome(Ne);
  for (int e = 0; e < Ne; ++e) {
    const int eu = c->perm_elem[e];
    int* cn = &conn[(size_t)cw * e].x;
    for (int k = 0; k < npe; ++k) cn[k] = iperm[conn_user[(size_t)npe * eu + k]];
    ehome[e] = home[eu];
  }
  // node -> (element, slot) adjacency, sorted by element id
  std::vector<int> arow(Nn + 1, 0);
  for (int e = 0; e < Ne; ++e) {
    const int* cn = &conn[(size_t)cw * e].x;
    for (int k = 0; k < npe; ++k) arow[cn[k] + 1]++;
  }
  for (int i = 0; i < Nn; ++i) arow[i + 1] += arow[i];
  std::vector<int> acol(arow[Nn]);
  std::vector<int> fill(arow.begin(), arow.end() - 1);
  for (int e = 0; e < Ne; ++e) {
    const int* cn = &conn[(size_t)cw * e].x;
    for (int k = 0; k < npe; ++k) acol[fill[cn[k]]++] = (e << sh) | k;
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
  std::vector<std::pair<uint32_t, int>> ents;  // (li << sh | slot, element)
  std::vector<int4> spos((size_t)cw * Ne);
  int max_slots = 0;
  for (int b = 0; b < nblkn; ++b) {
    const int n0 = b * nb, n1 = std::min(Nn, n0 + nb);
    const int h0 = hs[b], h1 = hs[b + 1];
    foreign.clear();
    for (int n = n0; n < n1; ++n)
      for (int j = arow[n]; j < arow[n + 1]; ++j) {
        const int e = acol[j] >> sh;
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
        const int e = acol[j] >> sh, s = acol[j] & (int)smask;
        int li;
        if (ehome[e] == b) {
          li = e - h0;
        } else {
          li = (h1 - h0) + (int)(std::lower_bound(foreign.begin(), foreign.end(), e) - foreign.begin());
        }
        ents.push_back({((uint32_t)li << sh) | (uint32_t)s, e});
      }
      std::sort(ents.begin(), ents.end());
      node_row[n + 1] = node_row[n] + (int)ents.size();
      for (size_t k = 0; k < ents.size(); ++k) {
        const int pos = node_row[n] + (int)k;
        node_slots[pos] = ents[k].first;
        (&spos[(size_t)cw * ents[k].second].x)[ents[k].first & smask] = pos;
      }
    }
    max_slots = std::max(max_slots, node_row[n1] - node_row[n0]);
  }
  c->max_slots = max_slots;
  // the fused residual kernel stages 12 NB doubles plus the block's slot list
  const size_t smem_need = sizeof(double) * 12 * (size_t)nb + sizeof(uint32_t) * (size_t)max_slots;
  if (npe == 4 && smem_need > 200u * 1024u)
    return set_err(nullptr, FEM_ERR_INVALID,
                   "node block of %d nodes needs %zu bytes of shared memory (max 204800): use a smaller block",
                   nb, smem_need);
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
  if ((st = dalloc(c, &c->conn, conn.size()))) return st;
  if ((st = dalloc(c, &c->blk_ptr, blk_ptr.size()))) return st;
  if ((st = dalloc(c, &c->blk_home, blk_home.size()))) return st;
  if ((st = dalloc(c, &c->blk_elems, blk_elems.size()))) return st;
  if ((st = dalloc(c, &c->node_row, node_row.size()))) return st;
  if ((st = dalloc(c, &c->node_slots, node_slots.size()))) return st;
  if ((st = dalloc(c, &c->spos, spos.size()))) return st;
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
  CK(cudaMemcpyAsync(c->spos, spos.data(), spos.size() * sizeof(int4), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_perm_node, c->perm_node.data(), Nn * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_perm_elem, c->perm_elem.data(), Ne * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  // the host vectors go out of scope: finish the copies first
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int alloc_state(FemCtx* c) {
  const size_t nd = (size_t)c->ndof_pad, Ne = (size_t)c->Ne, nf = 4 * (size_t)c->Nn;
  int st;
  if ((st = dalloc(c, &c->mat_id, Ne))) return st;
  if ((st = dalloc(c, &c->scale, Ne))) return st;
  if ((st = dalloc(c, &c->fixed, (size_t)c->Nn))) return st;
  if ((st = dalloc(c, &c->fixed_vals, nd))) return st;
  if ((st = dalloc(c, &c->fext, nd))) return st;
  if ((st = dalloc(c, &c->fixed_vals_full, nd))) return st;
  if ((st = dalloc(c, &c->fext_full, nd))) return st;
  if ((st = dalloc(c, &c->u, nd))) return st;
  if ((st = dalloc(c, &c->u_base, nd))) return st;
  if ((st = dalloc(c, &c->R, nd))) return st;
  if ((st = dalloc(c, &c->tmpd, nd))) return st;
  const size_t Nq = c->Nq;
  if ((st = dalloc(c, &c->payload, Nq * kPay))) return st;
  if ((st = dalloc(c, &c->ep_c, Nq * 6))) return st;
  if ((st = dalloc(c, &c->epe_c, Nq))) return st;
  if ((st = dalloc(c, &c->ep_t, Nq * 6))) return st;
  if ((st = dalloc(c, &c->epe_t, Nq))) return st;
  if ((st = dalloc(c, &c->r, nf))) return st;
  if ((st = dalloc(c, &c->x, nf))) return st;
  if ((st = dalloc(c, &c->p, nf))) return st;
  if ((st = dalloc(c, &c->y, nf))) return st;
  if ((st = dalloc(c, &c->dinv, nf))) return st;
  if ((st = dalloc(c, &c->tmpf, nf))) return st;
  if ((st = dalloc(c, &c->boff, nf))) return st;
  // slot vectors of the two-phase passes; HEX8 diagonal blocks take 2 per slot
  if ((st = dalloc(c, &c->stage, c->npe == 8 ? 16 * Ne : 4 * Ne))) return st;
  if ((st = dalloc(c, &c->stage_d, (c->npe == 8 ? 24 : 12) * Ne))) return st;
  if ((st = dalloc(c, &c->matD, (size_t)FEM_MAX_MATERIALS))) return st;
  if ((st = dalloc(c, &c->matF, (size_t)FEM_MAX_MATERIALS))) return st;
  // every reducing kernel's grid must fit: node blocks and node-parallel blocks
  // (node gather: 64 nodes per CTA; element-block matvec: at least kEbThreads elements per CTA)
  c->max_blocks = std::max(std::max(c->n_blocks, (c->Nn + 63) / 64), (c->Ne + kEbThreads - 1) / kEbThreads) + 1;
  if ((st = dalloc(c, &c->partials, (size_t)N_SITES * 2 * c->max_blocks))) return st;
  if ((st = dalloc(c, &c->counters, (size_t)N_SITES))) return st;
  if ((st = dalloc(c, &c->scalars, (size_t)8))) return st;
  if ((st = dalloc(c, &c->cg, (size_t)1))) return st;
  if ((st = dalloc(c, &c->step_bar, (size_t)4))) return st;
  if ((st = dalloc(c, &c->jac_part, 2 * (size_t)step_chunks(c->Nn)))) return st;
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

// ───────────────────────── element-block matvec tables ─────────────────────────

// Candidate elements per block of the element-block matvec (timed on the
// first PCG solve unless FEM_OPT_EB_SIZE fixes one).
constexpr int kEbSizes[4] = {256, 512, 768, 1024};

// Frees the element-block tables and every captured CG graph (a graph
// captured with the element-block variant holds the tables' addresses).
void free_eb_tables(FemCtx* c) {
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (!c->eb_bufs.empty()) {
    for (int k = 0; k < N_GRAPHS; ++k) {
      if (c->cg_graph[k]) cudaGraphExecDestroy(c->cg_graph[k]);
      if (c->loop_graph[k]) cudaGraphExecDestroy(c->loop_graph[k]);
      c->cg_graph[k] = nullptr;
      c->loop_graph[k] = nullptr;
    }
  }
  for (void* p : c->eb_bufs)
    if (p) cudaFree(p);
  c->eb_bufs.clear();
  c->ebdev = EbDev{};
  c->eb_size = 0;
}

template <typename T>
int eb_upload(FemCtx* c, T** dst, const std::vector<T>& v) {
  int st;
  if ((st = dalloc(c, dst, v.size()))) return st;
  c->eb_bufs.push_back(*dst);
  if (!v.empty()) CK(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  return FEM_OK;
}

// Builds the element-block tables for blocks of `eb` consecutive elements
// (TET4).  Per block: its local nodes (distinct vertices, ascending), each
// element's local vertex indices, the node-major position of each of its
// slot vectors (sorted by local node, then element, then slot: the fixed
// summation order), and for every local node shared with another block the
// slot of its partial row; shared nodes' partials are ordered by block, and
// the shared nodes are listed for the completion kernel.
int build_eb_tables(FemCtx* c, int eb) {
  if (c->eb_size == eb) return FEM_OK;
  free_eb_tables(c);
  const int Ne = c->Ne, Nn = c->Nn;
  if (c->npe != 4) return set_err(c, FEM_ERR_INVALID, "the element-block matvec is TET4 only");
  if (eb != 256 && eb != 512 && eb != 768 && eb != 1024)
    return set_err(c, FEM_ERR_INVALID, "element block of %d elements: need 256, 512, 768 or 1024", eb);
  std::vector<int4> conn(Ne);
  CK(cudaMemcpyAsync(conn.data(), c->conn, Ne * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::vector<int> deg(Nn, 0);
  for (int e = 0; e < Ne; ++e) {
    const int* cn = &conn[e].x;
    for (int k = 0; k < 4; ++k) deg[cn[k]]++;
  }
  const int n_blk = (Ne + eb - 1) / eb;
  std::vector<int> node_ptr(n_blk + 1, 0), nodes, nshared(Nn + 1, 0);
  std::vector<int4> ninfo;
  std::vector<uint16_t> lrow;
  std::vector<uint2> lconn(Ne), lspos(Ne);
  nodes.reserve((size_t)Ne / 2);
  std::vector<uint64_t> ent;
  int lmax = 0;
  for (int b = 0; b < n_blk; ++b) {
    const int e0 = b * eb, e1 = std::min(Ne, e0 + eb);
    ent.clear();
    for (int e = e0; e < e1; ++e) {
      const int* cn = &conn[e].x;
      for (int k = 0; k < 4; ++k)
        ent.push_back(((uint64_t)(uint32_t)cn[k] << 32) | ((uint64_t)(e - e0) << 2) | (uint64_t)k);
    }
    std::sort(ent.begin(), ent.end());
    node_ptr[b] = (int)nodes.size();
    int L = 0;
    size_t j = 0;
    while (j < ent.size()) {
      const int n = (int)(ent[j] >> 32);
      size_t j1 = j;
      while (j1 < ent.size() && (int)(ent[j1] >> 32) == n) ++j1;
      lrow.push_back((uint16_t)j);
      for (size_t q = j; q < j1; ++q) {
        const int le = (int)((ent[q] >> 2) & 0x3fffffffu), k = (int)(ent[q] & 3u);
        uint16_t* lc = reinterpret_cast<uint16_t*>(&lconn[e0 + le]);
        uint16_t* sp = reinterpret_cast<uint16_t*>(&lspos[e0 + le]);
        lc[k] = (uint16_t)L;
        sp[k] = (uint16_t)q;
      }
      nodes.push_back(n);
      const bool interior = (int)(j1 - j) == deg[n];
      ninfo.push_back(make_int4(n, interior ? -1 : -2, 0, 0));
      if (!interior) nshared[n + 1]++;
      ++L;
      j = j1;
    }
    lrow.push_back((uint16_t)ent.size());
    if (L > 65535) return set_err(c, FEM_ERR_INVALID, "element block %d touches %d nodes (max 65535)", b, L);
    lmax = std::max(lmax, L);
  }
  node_ptr[n_blk] = (int)nodes.size();
  for (int n = 0; n < Nn; ++n) nshared[n + 1] += nshared[n];
  std::vector<int> fill(nshared.begin(), nshared.end() - 1);
  for (size_t i = 0; i < nodes.size(); ++i) {
    int4& in = ninfo[i];
    if (in.y == -2) {
      in.y = fill[in.x]++;
      in.z = nshared[in.x];
      in.w = nshared[in.x + 1] - nshared[in.x];
    }
  }
  const size_t n_parts = (size_t)nshared[Nn];
  std::vector<int4> snode;
  for (int n = 0; n < Nn; ++n)
    if (nshared[n + 1] > nshared[n]) snode.push_back(make_int4(n, nshared[n], nshared[n + 1] - nshared[n], 0));
  int* d_ptr = nullptr;
  int* d_nodes = nullptr;
  int4* d_ninfo = nullptr;
  uint16_t* d_lrow = nullptr;
  uint2 *d_lconn = nullptr, *d_lspos = nullptr;
  float4* d_parts = nullptr;
  int4* d_snode = nullptr;
  double* d_pap = nullptr;
  int st;
  if ((st = eb_upload(c, &d_ptr, node_ptr))) return st;
  if ((st = eb_upload(c, &d_nodes, nodes))) return st;
  if ((st = eb_upload(c, &d_ninfo, ninfo))) return st;
  if ((st = eb_upload(c, &d_lrow, lrow))) return st;
  if ((st = eb_upload(c, &d_lconn, lconn))) return st;
  if ((st = eb_upload(c, &d_lspos, lspos))) return st;
  if ((st = dalloc(c, &d_parts, std::max<size_t>(n_parts, 1)))) return st;
  c->eb_bufs.push_back(d_parts);
  if ((st = eb_upload(c, &d_snode, snode))) return st;
  if ((st = dalloc(c, &d_pap, (size_t)n_blk))) return st;
  c->eb_bufs.push_back(d_pap);
  CK(cudaStreamSynchronize(c->stream));
  EbDev& t = c->ebdev;
  t.eb = eb;
  t.n_blk = n_blk;
  t.lmax = lmax;
  t.node_ptr = d_ptr;
  t.nodes = d_nodes;
  t.ninfo = d_ninfo;
  t.lrow = d_lrow;
  t.lconn = d_lconn;
  t.lspos = d_lspos;
  t.parts = d_parts;
  t.snode = d_snode;
  t.n_shared = (int)snode.size();
  t.pap_part = d_pap;
  c->eb_size = eb;
  return FEM_OK;
}

// Frees the warp-aggregation tables and every captured CG graph (which may
// hold their addresses).
void free_wagg_tables(FemCtx* c) {
  if (c->wa_bufs.empty()) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int k = 0; k < N_GRAPHS; ++k) {
    if (c->cg_graph[k]) cudaGraphExecDestroy(c->cg_graph[k]);
    if (c->loop_graph[k]) cudaGraphExecDestroy(c->loop_graph[k]);
    c->cg_graph[k] = nullptr;
    c->loop_graph[k] = nullptr;
  }
  for (void* p : c->wa_bufs)
    if (p) cudaFree(p);
  c->wa_bufs.clear();
  c->wadev = WaggDev{};
}

// Builds the warp-aggregation tables (TET4): per warp of 32 consecutive
// elements its distinct vertices (ascending), each element's slot positions
// in the warp's node-major slot order (by vertex, then element, then slot:
// the fixed summation order), and per (warp, vertex) the position of its
// partial row among the vertex's partials, which are ordered by warp.
int build_wagg_tables(FemCtx* c) {
  if (!c->wa_bufs.empty()) return FEM_OK;
  const int Ne = c->Ne, Nn = c->Nn;
  if (c->npe != 4) return set_err(c, FEM_ERR_INVALID, "the warp-aggregated matvec is TET4 only");
  std::vector<int4> conn(Ne);
  CK(cudaMemcpyAsync(conn.data(), c->conn, Ne * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int n_warps = (Ne + 31) / 32;
  std::vector<int> wptr(n_warps + 1, 0), wnode, prow(Nn + 1, 0);
  std::vector<int2> went;
  std::vector<uint32_t> lspos(Ne, 0u), lrow(Ne, 0u);
  wnode.reserve((size_t)Ne);
  went.reserve((size_t)Ne);
  std::vector<uint64_t> ent;
  for (int w = 0; w < n_warps; ++w) {
    const int e0 = 32 * w, e1 = std::min(Ne, e0 + 32);
    ent.clear();
    for (int e = e0; e < e1; ++e) {
      const int* cn = &conn[e].x;
      for (int k = 0; k < 4; ++k)
        ent.push_back(((uint64_t)(uint32_t)cn[k] << 32) | ((uint64_t)(e - e0) << 2) | (uint64_t)k);
    }
    std::sort(ent.begin(), ent.end());
    wptr[w] = (int)went.size();
    size_t j = 0;
    while (j < ent.size()) {
      const int n = (int)(ent[j] >> 32);
      size_t j1 = j;
      while (j1 < ent.size() && (int)(ent[j1] >> 32) == n) ++j1;
      const uint32_t row = (uint32_t)(went.size() - (size_t)wptr[w]);  // < 128: 4 vertices x 32 elements
      for (size_t q = j; q < j1; ++q) {
        const int le = (int)((ent[q] >> 2) & 31u), k = (int)(ent[q] & 3u);
        lspos[e0 + le] |= (uint32_t)q << (8 * k);
        lrow[e0 + le] |= row << (8 * k);
      }
      went.push_back(make_int2(0, (int)j | ((int)j1 << 16)));
      wnode.push_back(n);
      prow[n + 1]++;
      j = j1;
    }
  }
  wptr[n_warps] = (int)went.size();
  for (int n = 0; n < Nn; ++n) prow[n + 1] += prow[n];
  std::vector<int> fill(prow.begin(), prow.end() - 1);
  for (size_t i = 0; i < went.size(); ++i) went[i].x = fill[wnode[i]]++;
  uint32_t *d_lspos = nullptr, *d_lrow = nullptr;
  int *d_wptr = nullptr, *d_prow = nullptr, *d_wnode = nullptr;
  int2* d_went = nullptr;
  float4* d_parts = nullptr;
  int st;
  auto up = [&](auto** dst, const auto& v) -> int {
    int r;
    if ((r = dalloc(c, dst, v.size()))) return r;
    c->wa_bufs.push_back(*dst);
    if (!v.empty())
      CK(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice, c->stream));
    return FEM_OK;
  };
  if ((st = up(&d_lspos, lspos))) return st;
  if ((st = up(&d_wptr, wptr))) return st;
  if ((st = up(&d_went, went))) return st;
  if ((st = up(&d_prow, prow))) return st;
  if ((st = up(&d_lrow, lrow))) return st;
  if ((st = up(&d_wnode, wnode))) return st;
  if ((st = dalloc(c, &d_parts, std::max<size_t>(went.size(), 1)))) return st;
  c->wa_bufs.push_back(d_parts);
  CK(cudaStreamSynchronize(c->stream));
  c->wadev.lspos = d_lspos;
  c->wadev.wptr = d_wptr;
  c->wadev.went = d_went;
  c->wadev.prow = d_prow;
  c->wadev.parts = d_parts;
  c->wadev.lrow = d_lrow;
  c->wadev.wnode = d_wnode;
  return FEM_OK;
}

// ───────────────────────── kernels wrappers ─────────────────────────

// Matvec arguments with the mesh tables and the context's variant filled in.
MvArgs make_mv(const FemCtx* c) {
  MvArgs mv;
  std::memset(&mv, 0, sizeof(mv));
  mv.m = c->mesh();
  mv.variant = c->mv_variant;
  mv.stage = c->stage;
  mv.eb = c->ebdev;
  mv.wa = c->wadev;
  return mv;
}

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
  a.stage_d = (c->npe == 8 || c->res_two_phase) ? c->stage_d : nullptr;
  c->n_launches += c->npe == 8 ? 2 : 1;
  launch_residual(a, c->model_kind, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->h_scalars, c->scalars, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->tangent_valid = true;
  if (rnorm2) *rnorm2 = c->h_scalars[0];
  return FEM_OK;
}

// Jacobi scaling for the PCG solve: 1 / diag(K_T), or with `block` the
// nodal 3 x 3 block inverse (diagonal in dinv, off-diagonals in boff).
int compute_dinv(FemCtx* c, int precond, bool block = false) {
  if (precond == FEM_PRECOND_JACOBI) {
    DiagArgs a;
    a.m = c->mesh();
    a.matF = c->matF;
    a.payload = c->payload;
    a.dinv = c->dinv;
    a.boff = block ? c->boff : nullptr;
    a.stage = c->stage;
    c->n_launches += c->npe == 8 ? 2 : 1;
    launch_diag(a, c->model_kind, c->stream);
    CKL();
  } else {
    // identity on free DOFs: dinv = 1 where not fixed
    ++c->n_launches; launch_dinv_identity(c->dinv, c->fixed, c->Nn, c->stream);
    CKL();
  }
  return FEM_OK;
}

CoarseArgs coarse_args(const FemCtx* c) {
  CoarseArgs a;
  a.m = c->mesh();
  a.c = c->cdev;
  a.matF = c->matF;
  a.payload = c->payload;
  a.boff = c->block_jacobi ? c->boff : nullptr;
  return a;
}

bool use_pdl(const FemCtx* c, int kind) { return kind != GRAPH_LEARNED && c->pdl && c->pdl_ok; }

// Sets chain_pdl() for the launches of one capture, restores it after.
struct ChainPdl {
  bool saved;
  explicit ChainPdl(bool on) : saved(chain_pdl()) { chain_pdl() = on; }
  ~ChainPdl() { chain_pdl() = saved; }
};

// Two-level PCG with the two-phase matvec: the matvec acts on z and its node
// gather forms p = z + beta p, q = K z + beta q (no direction-update kernel).
bool recurrence(const FemCtx* c, int kind) {
  return kind == GRAPH_TWO_LEVEL && (c->mv_variant == MV_TWO_PHASE || c->mv_variant == MV_WARP_AGG || c->mv_variant == MV_PERSIST) &&
         c->direction_recurrence;
}

bool use_fused(const FemCtx* c, int kind) {
  return kind != GRAPH_LEARNED && c->fused_step && c->fused_ok && !c->in_batch &&
         (kind == GRAPH_JACOBI || (c->tl_part != nullptr && c->cdev.Ainv != nullptr && !c->block_jacobi));
}

StepArgs step_args(const FemCtx* c, int kind) {
  StepArgs a;
  a.m = c->mesh();
  a.c = c->cdev;
  a.x = c->x;
  a.r = c->r;
  a.p = c->p;
  a.q = c->y;
  a.dinv = c->dinv;
  a.z = c->tmpf;
  a.cg = c->cg;
  a.part = kind == GRAPH_TWO_LEVEL ? c->tl_part : c->jac_part;
  a.n_chunks = step_chunks(c->Nn);
  a.bar = c->step_bar;
  return a;
}

// Kernels launched per CG iteration (matvec + the rest).
int64_t kernels_per_iter(const FemCtx* c, int kind, bool fused) {
  const int64_t mv = c->mv_variant == MV_FUSED ? 1 : 2;
  if (fused) return mv + 1;
  if (kind == GRAPH_TWO_LEVEL) return mv + 3 + coarse_product_kernels(c->cdev) + (recurrence(c, kind) ? 0 : 1);
  return mv + 2;
}

// Enqueues one CG iteration; returns the first launch error (a refused
// cooperative launch during capture).
cudaError_t enqueue_cg_iter(FemCtx* c, int kind, bool fused) {
  MvArgs mv = make_mv(c);
  mv.matF = c->matF;
  mv.payload = c->payload;
  mv.x = c->p;
  if (!fused && recurrence(c, kind)) {
    mv.x = c->tmpf;  // z
    mv.p_rec = c->p;
  }
  mv.y = c->y;
  mv.cg = c->cg;
  mv.red = c->red();
  mv.red_site = SITE_MV;
  mv.mask_input = 1;
  launch_matvec(mv, c->model_kind, c->stream);
  if (kind == GRAPH_LEARNED) {
    const CoarseArgs ca = coarse_args(c);
    launch_cg_update(c->x, c->r, c->p, c->y, c->dinv, c->Nn, c->cg, c->red(), SITE_CGU, c->stream, 0);
    launch_mpnn_forward(c->mdev, c->r, c->dinv, c->tmpf, c->cg, c->red(), SITE_RZ, c->stream);
    if (c->learned_coarse) launch_coarse_apply(ca, c->r, c->cg, c->stream);
    launch_fpcg_dots(ca, false, c->learned_coarse, c->r, c->y, c->dinv, c->tmpf, c->zalt, c->p, c->cg, c->red(),
                     SITE_RZ, SITE_RZ2, c->stream);
    launch_fpcg_pupdate(c->p, c->tmpf, c->zalt, c->Nn, c->cg, false, c->stream);
    return cudaSuccess;
  }
  if (fused) {
    const StepArgs sa = step_args(c, kind);
    return kind == GRAPH_TWO_LEVEL ? launch_tl_step(sa, c->stream) : launch_jacobi_step(sa, c->stream);
  }
  if (kind == GRAPH_TWO_LEVEL) {
    const CoarseArgs ca = coarse_args(c);
    launch_update_restrict(ca, c->x, c->r, c->p, c->y, c->cg, c->stream);
    launch_coarse_solve(ca, c->cg, c->stream);
    launch_tl_rz(ca, false, c->r, c->dinv, c->tmpf, c->p, c->cg, c->red(), SITE_RZ, c->stream);
    // with the recurrence the next matvec forms the direction
    if (!recurrence(c, kind)) launch_tl_pupdate(c->p, c->tmpf, c->Nn, c->cg, c->stream);
    return cudaSuccess;
  }
  launch_cg_update(c->x, c->r, c->p, c->y, c->dinv, c->Nn, c->cg, c->red(), SITE_CGU, c->stream);
  launch_cg_pupdate(c->p, c->r, c->dinv, c->Nn, c->cg, c->stream);
  return cudaSuccess;
}

// A CG state that never finishes, so the fused CG kernels do their full work
// when timed outside a solve.
CGState endless_cg() {
  CGState hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.rz = 1.0;
  hs.rr = 1.0;
  hs.rr0 = 1.0;
  hs.tol2 = 0.0;
  hs.alpha = 1e-30;
  hs.beta = 0.0;
  hs.max_iter = 1 << 30;
  return hs;
}

// Picks the matvec variant for the current material tables: the forced one
// when fem_set_option set it, else the faster of the two on this mesh, timed
// with CUDA events as they run inside CG (3 warm-up + 10 timed launches each,
// p = 1 on free DOFs).  The CG state is reset by cg_init afterwards.
int choose_matvec_variant(FemCtx* c) {
  if (c->npe == 8) {
    // HEX8 has the two-phase pass only
    c->mv_variant = MV_TWO_PHASE;
    return FEM_OK;
  }
  int st;
  if (c->mv_forced >= 0) {
    c->mv_variant = c->mv_forced;
    if (c->mv_variant == MV_ELEM_BLOCK && c->eb_size == 0)
      return build_eb_tables(c, c->eb_forced > 0 ? c->eb_forced : 512);
    if (c->mv_variant == MV_WARP_AGG) return build_wagg_tables(c);
    return FEM_OK;
  }
  if (c->mv_tuned && c->mv_tuned_model == c->model_kind) return FEM_OK;
  const CGState hs = endless_cg();
  CK(cudaMemcpyAsync(c->cg, &hs, sizeof(hs), cudaMemcpyHostToDevice, c->stream));
  launch_dinv_identity(c->p, c->fixed, c->Nn, c->stream);
  EventPair ev;
  CK(ev.create());
  cudaEvent_t e0 = ev.a, e1 = ev.b;
  // ns per launch of variant v (element-block: with the tables built)
  auto time_variant = [&](int v, double* ns) -> int {
    MvArgs mv = make_mv(c);
    mv.variant = v;
    mv.matF = c->matF;
    mv.payload = c->payload;
    mv.x = c->p;
    mv.y = c->y;
    mv.cg = c->cg;
    mv.red = c->red();
    mv.red_site = SITE_MV;
    mv.mask_input = 1;
    for (int w = 0; w < 3; ++w) launch_matvec(mv, c->model_kind, c->stream);
    CK(cudaEventRecord(e0, c->stream));
    constexpr int kReps = 10;
    for (int r = 0; r < kReps; ++r) launch_matvec(mv, c->model_kind, c->stream);
    CK(cudaEventRecord(e1, c->stream));
    CKL();
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    *ns = 1e6 * ms / kReps;
    c->n_launches += (v == MV_FUSED ? 1 : 2) * 13;
    return FEM_OK;
  };
  for (int v = 0; v < MV_ELEM_BLOCK; ++v)
    if ((st = time_variant(v, &c->mv_ns[v]))) return st;
  // element-block: every candidate block size (or the forced one), keep the
  // fastest; then the warp-aggregated pass
  int best_eb = 0;
  double best_ns = 0.0;
  for (int k = 0; k < 4; ++k) {
    const int eb = kEbSizes[k];
    c->eb_ns[k] = 0.0;
    if (c->eb_forced > 0 && eb != c->eb_forced) continue;
    if ((st = build_eb_tables(c, eb))) return st;
    if ((st = time_variant(MV_ELEM_BLOCK, &c->eb_ns[k]))) return st;
    if (best_eb == 0 || c->eb_ns[k] < best_ns) {
      best_eb = eb;
      best_ns = c->eb_ns[k];
    }
  }
  if ((st = build_eb_tables(c, best_eb))) return st;
  c->mv_ns[MV_ELEM_BLOCK] = best_ns;
  if ((st = build_wagg_tables(c))) return st;
  if ((st = time_variant(MV_WARP_AGG, &c->mv_ns[MV_WARP_AGG]))) return st;
  if ((st = time_variant(MV_PERSIST, &c->mv_ns[MV_PERSIST]))) return st;
  int v_best = MV_FUSED;
  for (int v = 1; v < MV_N_VARIANTS; ++v)
    if (c->mv_ns[v] < c->mv_ns[v_best]) v_best = v;
  c->mv_variant = v_best;
  if (v_best != MV_ELEM_BLOCK) free_eb_tables(c);
  if (v_best != MV_WARP_AGG) free_wagg_tables(c);
  c->mv_tuned = true;
  c->mv_tuned_model = c->model_kind;
  return FEM_OK;
}

// One graph for a whole PCG solve: a conditional WHILE node whose body holds
// kLoopIters CG iterations and cg_loop_cond_kernel, which clears the
// condition once the CG state is done (converged, out of iterations, broken
// down) and also after max_iter / kLoopIters + 2 trips, so the loop ends
// even if the state stopped advancing.  Returns false (and leaves nothing
// behind) if the runtime cannot build it; the batched graphs are used then.
constexpr int kLoopIters = 4;

bool build_loop_graph(FemCtx* c, int kind, bool fused, bool pdl) {
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return false;
  bool ok = false;
  do {
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) break;
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, g, nullptr, 0, &np) != cudaSuccess) break;
    cudaGraph_t body = np.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
      break;
    cudaError_t le = cudaSuccess;
    {
      ChainPdl pdl_scope(pdl);
      for (int i = 0; i < kLoopIters; ++i) {
        const cudaError_t e = enqueue_cg_iter(c, kind, fused);
        if (le == cudaSuccess) le = e;
      }
      launch_cg_loop_cond(h, c->cg, kLoopIters, c->stream);
    }
    cudaGraph_t captured = nullptr;
    if (cudaStreamEndCapture(c->stream, &captured) != cudaSuccess || le != cudaSuccess) break;
    if (cudaGraphInstantiate(&c->loop_graph[kind], g, 0) != cudaSuccess) {
      c->loop_graph[kind] = nullptr;
      break;
    }
    ok = true;
  } while (false);
  cudaGraphDestroy(g);
  cudaGetLastError();  // a refused build leaves no sticky error behind
  return ok;
}

// Frees the coarse lattice and the graphs that captured its buffers (two-level
// and learned); the next two-level / learned solve rebuilds them.
int drop_coarse(FemCtx* c) {
  CK(cudaStreamSynchronize(c->stream));
  for (void* p : c->coarse_bufs)
    if (p) cudaFree(p);
  c->coarse_bufs.clear();
  c->cdev = CoarseDev{};
  c->coarse_have_inverse = false;
  c->tl_part = nullptr;
  if (c->dense_work) cudaFree(c->dense_work);
  c->dense_work = nullptr;
  c->dense_bytes = 0;
  c->coarse_row_first.clear();
  c->coarse_built = false;
  c->coarse_valid = false;
  for (int k : {GRAPH_TWO_LEVEL, GRAPH_LEARNED}) {
    if (c->cg_graph[k]) cudaGraphExecDestroy(c->cg_graph[k]);
    if (c->loop_graph[k]) cudaGraphExecDestroy(c->loop_graph[k]);
    c->cg_graph[k] = nullptr;
    c->loop_graph[k] = nullptr;
  }
  return FEM_OK;
}

// The coarse operator no longer matches the problem (new state, materials
// or constraints): the next two-level solve assembles one.
void invalidate_coarse(FemCtx* c) { c->coarse_valid = false; }

int ensure_cg_graph(FemCtx* c, int kind) {
  int st;
  if ((st = choose_matvec_variant(c))) return st;
  const bool fused = use_fused(c, kind);
  const bool pdl = use_pdl(c, kind);
  const int flags = (kind == GRAPH_LEARNED ? (c->learned_coarse ? 1 : 0) : 0) | (fused ? 2 : 0) | (pdl ? 4 : 0) |
                    (!fused && recurrence(c, kind) ? 8 : 0) | (kind == GRAPH_TWO_LEVEL && c->block_jacobi ? 16 : 0) |
                    (c->mv_variant == MV_ELEM_BLOCK ? c->eb_size << 8 : 0);
  if (c->cg_graph[kind] && c->cg_graph_model[kind] == c->model_kind &&
      c->cg_graph_variant[kind] == c->mv_variant && c->cg_graph_flags[kind] == flags)
    return FEM_OK;
  if (c->cg_graph[kind]) {
    cudaGraphExecDestroy(c->cg_graph[kind]);
    c->cg_graph[kind] = nullptr;
  }
  if (c->loop_graph[kind]) {
    cudaGraphExecDestroy(c->loop_graph[kind]);
    c->loop_graph[kind] = nullptr;
  }
  prepare_kernels(c->mesh(), c->model_kind);
  if (c->mv_variant == MV_ELEM_BLOCK) prepare_eb_kernels(c->model_kind);
  if (kind == GRAPH_TWO_LEVEL || (kind == GRAPH_LEARNED && c->learned_coarse))
    prepare_coarse_kernels(c->model_kind, c->cdev.n_dof);
  if (kind == GRAPH_LEARNED) prepare_mpnn_kernels();
  if (fused) prepare_step_kernels(kind == GRAPH_TWO_LEVEL ? 1 : 0, c->cdev.n_dof);
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t le = cudaSuccess;
  {
    ChainPdl pdl_scope(pdl);
    for (int i = 0; i < cg_batch(kind); ++i) {
      const cudaError_t e1 = enqueue_cg_iter(c, kind, fused);
      if (le == cudaSuccess) le = e1;
    }
    if (le == cudaSuccess) le = cudaGetLastError();
  }
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if ((pdl || fused) && (e != cudaSuccess || le != cudaSuccess)) {
    // the runtime refused programmatic launches or the cooperative step:
    // capture again without them (programmatic launches first)
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    if (pdl)
      c->pdl_ok = false;
    else
      c->fused_ok = false;
    return ensure_cg_graph(c, kind);
  }
  if (e != cudaSuccess) return set_err(c, FEM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&c->cg_graph[kind], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess && (pdl || fused)) {
    c->cg_graph[kind] = nullptr;
    cudaGetLastError();
    if (pdl)
      c->pdl_ok = false;
    else
      c->fused_ok = false;
    return ensure_cg_graph(c, kind);
  }
  if (e != cudaSuccess) return set_err(c, FEM_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
  if (c->use_loop_graph && !build_loop_graph(c, kind, fused, pdl) && !(pdl && build_loop_graph(c, kind, fused, false)))
    c->use_loop_graph = false;
  c->cg_graph_model[kind] = c->model_kind;
  c->cg_graph_variant[kind] = c->mv_variant;
  c->cg_graph_flags[kind] = flags;
  return FEM_OK;
}

template <typename T>
int coarse_upload(FemCtx* c, const T** dst, const std::vector<T>& v) {
  T* d = nullptr;
  int st;
  if ((st = dalloc(c, &d, v.size()))) return st;
  c->coarse_bufs.push_back(d);
  if (!v.empty()) CK(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  *dst = d;
  return FEM_OK;
}

template <typename T>
int coarse_alloc(FemCtx* c, T** dst, size_t n) {
  int st;
  if ((st = dalloc(c, dst, n))) return st;
  c->coarse_bufs.push_back(*dst);
  return FEM_OK;
}

// Builds the coarse lattice: cell edge H = coarse_cell_voxels x the mesh
// length (cube root of 5 x the mean element volume: the voxel edge on
// 5-tet voxel meshes), grown by 25 % steps until at most coarse_max_nodes
// coarse nodes remain.  Along each axis the lattice overhangs the mesh by
// less than one cell; the overhang is split between both ends in whole mesh
// lengths, so no end cell holds a slab thinner than about H/2 (a thin end
// slab leaves coarse nodes with almost no support and an ill-conditioned
// coarse operator).  Elements go to the cell of their centroid; a node to the
// cell of its lowest-numbered element.
constexpr int kMaxCoarseNodesLimit = 16384;
static_assert(kMaxCoarseNodesLimit <= 65535, "node_corners packs coarse node ids in 16 bits");

int build_coarse(FemCtx* c) {
  const int Nn = c->Nn, Ne = c->Ne, npe = c->npe, cw = npe / 4;
  std::vector<double> X(3 * (size_t)Nn);
  std::vector<int4> conn((size_t)cw * Ne);
  CK(cudaMemcpyAsync(X.data(), c->X64, X.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(conn.data(), c->conn, conn.size() * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = hi[d] = X[d];
    for (int i = 0; i < Nn; ++i) {
      lo[d] = std::min(lo[d], X[3 * i + d]);
      hi[d] = std::max(hi[d], X[3 * i + d]);
    }
  }
  double vsum = 0.0;
  std::vector<double> cen(3 * (size_t)Ne);
  // TET4: the three edges at vertex 0 span 6 x the volume; HEX8: vertices
  // 1, 3 and 4 are vertex 0's edge neighbours (the box volume for a voxel)
  const int ea = 1, eb = npe == 8 ? 3 : 2, ec = npe == 8 ? 4 : 3;
  for (int e = 0; e < Ne; ++e) {
    const int* cn = &conn[(size_t)cw * e].x;
    double a[3], b[3], cc[3];
    for (int d = 0; d < 3; ++d) {
      a[d] = X[3 * cn[ea] + d] - X[3 * cn[0] + d];
      b[d] = X[3 * cn[eb] + d] - X[3 * cn[0] + d];
      cc[d] = X[3 * cn[ec] + d] - X[3 * cn[0] + d];
      double s = 0.0;
      for (int k = 0; k < npe; ++k) s += X[3 * cn[k] + d];
      cen[3 * e + d] = s / npe;
    }
    const double det = a[0] * (b[1] * cc[2] - b[2] * cc[1]) - a[1] * (b[0] * cc[2] - b[2] * cc[0]) +
                       a[2] * (b[0] * cc[1] - b[1] * cc[0]);
    vsum += std::fabs(det) / (npe == 8 ? 1.0 : 6.0);
  }
  // mesh length: the edge of a voxel (5 tets, or one hexahedron)
  const double hmesh = std::cbrt((npe == 8 ? 1.0 : 5.0) * vsum / std::max(Ne, 1));
  double H = c->coarse_cell_voxels * hmesh;
  std::vector<int> ecell(Ne), cell_of_lin, act_lin, cn_of_lat;
  int g[3];
  int n_cells = 0, n_cn = 0;
  double org[3] = {lo[0], lo[1], lo[2]};
  for (int attempt = 0; attempt < 64; ++attempt) {
    for (int d = 0; d < 3; ++d) {
      g[d] = std::max(1, (int)std::ceil((hi[d] - lo[d]) / H - 1e-9));
      const double overhang = g[d] * H - (hi[d] - lo[d]);
      org[d] = lo[d] - std::floor(0.5 * overhang / hmesh + 1e-6) * hmesh;
    }
    const int64_t ncell_lat = (int64_t)g[0] * g[1] * g[2];
    if (ncell_lat > (1 << 22)) {
      H *= 1.25;
      continue;
    }
    cell_of_lin.assign(ncell_lat, -1);
    for (int e = 0; e < Ne; ++e) {
      int ijk[3];
      for (int d = 0; d < 3; ++d)
        ijk[d] = std::min(g[d] - 1, std::max(0, (int)std::floor((cen[3 * e + d] - org[d]) / H)));
      const int lin = (ijk[0] * g[1] + ijk[1]) * g[2] + ijk[2];
      ecell[e] = lin;
      cell_of_lin[lin] = 0;
    }
    act_lin.clear();
    for (int64_t l = 0; l < ncell_lat; ++l)
      if (cell_of_lin[l] == 0) {
        cell_of_lin[l] = (int)act_lin.size();
        act_lin.push_back((int)l);
      }
    n_cells = (int)act_lin.size();
    // coarse nodes: corners of active cells on the (g+1)^3 lattice
    const int64_t nlat = (int64_t)(g[0] + 1) * (g[1] + 1) * (g[2] + 1);
    cn_of_lat.assign(nlat, -1);
    for (int cl = 0; cl < n_cells; ++cl) {
      const int l = act_lin[cl];
      const int i = l / (g[1] * g[2]), j = (l / g[2]) % g[1], k = l % g[2];
      for (int q = 0; q < 8; ++q) {
        const int64_t ln = ((int64_t)(i + (q >> 2 & 1)) * (g[1] + 1) + (j + (q >> 1 & 1))) * (g[2] + 1) +
                           (k + (q & 1));
        cn_of_lat[ln] = 0;
      }
    }
    n_cn = 0;
    for (int64_t l = 0; l < nlat; ++l)
      if (cn_of_lat[l] == 0) cn_of_lat[l] = n_cn++;
    if (n_cn <= c->coarse_max_nodes) break;
    H *= 1.25;
  }
  if (n_cn > c->coarse_max_nodes)
    return set_err(c, FEM_ERR_INVALID, "coarse lattice: could not reach %d coarse nodes", c->coarse_max_nodes);
  // tables
  std::vector<int3> cell_ijk(n_cells);
  std::vector<int> cell_corner(8 * (size_t)n_cells);
  for (int cl = 0; cl < n_cells; ++cl) {
    const int l = act_lin[cl];
    const int i = l / (g[1] * g[2]), j = (l / g[2]) % g[1], k = l % g[2];
    cell_ijk[cl] = make_int3(i, j, k);
    for (int q = 0; q < 8; ++q) {
      const int64_t ln = ((int64_t)(i + (q >> 2 & 1)) * (g[1] + 1) + (j + (q >> 1 & 1))) * (g[2] + 1) +
                         (k + (q & 1));
      cell_corner[8 * cl + q] = cn_of_lat[ln];
    }
  }
  std::vector<int> cn_cells(8 * (size_t)n_cn, -1), cn_fill(n_cn, 0);
  for (int cl = 0; cl < n_cells; ++cl)
    for (int q = 0; q < 8; ++q) {
      const int cnode = cell_corner[8 * cl + q];
      cn_cells[8 * cnode + cn_fill[cnode]++] = cl * 8 + q;
    }
  // Envelope of Ac (DOF 3 a + d of coarse node a): two coarse nodes couple
  // only through a shared cell, so row 3 a + d is zero left of column
  // 3 min{b : b shares a cell with a}; the dense inverse skips the tiles
  // outside it (the lattice order makes Ac banded).
  {
    std::vector<int> cn_first(n_cn);
    for (int a = 0; a < n_cn; ++a) cn_first[a] = a;
    for (int cl = 0; cl < n_cells; ++cl) {
      int mn = cell_corner[8 * cl];
      for (int q = 1; q < 8; ++q) mn = std::min(mn, cell_corner[8 * cl + q]);
      for (int q = 0; q < 8; ++q) cn_first[cell_corner[8 * cl + q]] = std::min(cn_first[cell_corner[8 * cl + q]], mn);
    }
    c->coarse_row_first.resize(3 * (size_t)n_cn);
    for (int r = 0; r < 3 * n_cn; ++r) c->coarse_row_first[r] = 3 * cn_first[r / 3];
  }
  std::vector<int> node_cell(Nn, -1);
  std::vector<int> cell_elem_ptr(n_cells + 1, 0), cell_elems(Ne);
  for (int e = 0; e < Ne; ++e) cell_elem_ptr[cell_of_lin[ecell[e]] + 1]++;
  for (int cl = 0; cl < n_cells; ++cl) cell_elem_ptr[cl + 1] += cell_elem_ptr[cl];
  {
    std::vector<int> fill(cell_elem_ptr.begin(), cell_elem_ptr.end() - 1);
    for (int e = 0; e < Ne; ++e) {
      const int cl = cell_of_lin[ecell[e]];
      cell_elems[fill[cl]++] = e;
      const int* cn = &conn[(size_t)cw * e].x;
      for (int k = 0; k < npe; ++k)
        if (node_cell[cn[k]] < 0) node_cell[cn[k]] = cl;
    }
  }
  for (int i = 0; i < Nn; ++i)
    if (node_cell[i] < 0) node_cell[i] = 0;  // node of no element: its DOFs carry no stiffness
  std::vector<int> cell_node_ptr(n_cells + 1, 0), cell_nodes(Nn);
  for (int i = 0; i < Nn; ++i) cell_node_ptr[node_cell[i] + 1]++;
  for (int cl = 0; cl < n_cells; ++cl) cell_node_ptr[cl + 1] += cell_node_ptr[cl];
  {
    std::vector<int> fill(cell_node_ptr.begin(), cell_node_ptr.end() - 1);
    for (int i = 0; i < Nn; ++i) cell_nodes[fill[node_cell[i]]++] = i;
  }
  CoarseDev& cd = c->cdev;
  cd.n_cells = n_cells;
  cd.n_cn = n_cn;
  cd.n_dof = 3 * n_cn;
  cd.inv_H = (float)(1.0 / H);
  cd.lo = make_float3((float)org[0], (float)org[1], (float)org[2]);
  int st;
  if ((st = coarse_upload(c, &cd.cell_ijk, cell_ijk))) return st;
  if ((st = coarse_upload(c, &cd.cell_corner, cell_corner))) return st;
  if ((st = coarse_upload(c, &cd.cell_node_ptr, cell_node_ptr))) return st;
  if ((st = coarse_upload(c, &cd.cell_nodes, cell_nodes))) return st;
  if ((st = coarse_upload(c, &cd.cell_elem_ptr, cell_elem_ptr))) return st;
  if ((st = coarse_upload(c, &cd.cell_elems, cell_elems))) return st;
  if ((st = coarse_upload(c, &cd.node_cell, node_cell))) return st;
  if ((st = coarse_upload(c, &cd.cn_cells, cn_cells))) return st;
  {
    float4* lat = nullptr;
    if ((st = coarse_alloc(c, &lat, (size_t)Nn))) return st;
    cd.node_lat = lat;
    launch_coarse_node_lat(c->mesh(), cd, lat, c->stream);
    CKL();
    uint4* corners = nullptr;
    if ((st = coarse_alloc(c, &corners, (size_t)Nn))) return st;
    cd.node_corners = corners;
    launch_coarse_node_corners(c->mesh(), cd, corners, c->stream);
    CKL();
  }
  const size_t nd = (size_t)cd.n_dof;
  cd.cell_slices = coarse_cell_slices(c->npe);
  if ((st = coarse_alloc(c, &cd.blocks, (size_t)n_cells * cd.cell_slices * 576))) return st;
  if ((st = coarse_alloc(c, &cd.Ac, nd * nd))) return st;
  cd.nb16 = (cd.n_dof + 63) / 64;
  const size_t nb = (size_t)cd.nb16;
  cd.Ainv = nullptr;
  cd.Ainv16 = nullptr;
  cd.yslots = nullptr;
  if (c->coarse_bf16) {
    if ((st = coarse_alloc(c, &cd.Ainv16, nb * (nb + 1) / 2 * 4096))) return st;
    if ((st = coarse_alloc(c, &cd.yslots, nb * nb * 64))) return st;
  } else {
    if ((st = coarse_alloc(c, &cd.Ainv, nd * nd))) return st;
  }
  cd.r_slices = coarse_restrict_slices(n_cells);
  if ((st = coarse_alloc(c, &cd.cell_r, (size_t)n_cells * cd.r_slices * 24))) return st;
  if ((st = coarse_alloc(c, &cd.yc, nb * 64))) return st;
  if ((st = coarse_alloc(c, &cd.rc, nb * 64))) return st;
  // fused two-level step: per (cell, slice) restriction and ||r||^2 shares
  if ((st = coarse_alloc(c, &c->tl_part, (size_t)n_cells * cd.r_slices + step_chunks(Nn)))) return st;
  CK(cudaStreamSynchronize(c->stream));
  c->coarse_H = H;
  c->coarse_built = true;
  c->coarse_valid = false;
  return FEM_OK;
}

// A refreshed coarse operator that is not positive definite (a tangent off
// the stable path, e.g. an arc-length predictor): keep applying the last
// inverse, which is still a symmetric positive definite preconditioner;
// without one the solve fails.
int keep_previous_coarse(FemCtx* c, int info) {
  if (!c->coarse_have_inverse)
    return set_err(c, FEM_ERR_NAN, "coarse operator is not positive definite (potrf info %d)", info);
  ++c->n_coarse_kept;
  c->coarse_valid = true;
  c->coarse_uses = 1;
  c->coarse_base_ipd = -1;
  return FEM_OK;
}

// Assembles Ac = P^T K_T P at the current tangent and inverts it (FP64
// Cholesky + inverse, then an FP32 or BF16 copy), unless the reuse policy keeps the
// previous one.
int ensure_coarse(FemCtx* c) {
  int st;
  if (!c->coarse_built && (st = build_coarse(c))) return st;
  if (c->coarse_valid && (c->coarse_reuse <= 0 || c->coarse_uses < c->coarse_reuse)) {
    ++c->coarse_uses;
    return FEM_OK;
  }
  // timing events live as long as the context (no leak on the error returns)
  for (cudaEvent_t& ev : c->coarse_ev)
    if (!ev) CK(cudaEventCreate(&ev));
  cudaEvent_t e0 = c->coarse_ev[0], em = c->coarse_ev[1], e1 = c->coarse_ev[2];
  CK(cudaEventRecord(e0, c->stream));
  prepare_coarse_kernels(c->model_kind, c->cdev.n_dof);
  const CoarseArgs ca = coarse_args(c);
  launch_coarse_assemble(ca, c->model_kind, c->stream);
  c->n_launches += 2;
  CKL();
  CK(cudaEventRecord(em, c->stream));
  const int n = c->cdev.n_dof;
  const int* row_first = (int)c->coarse_row_first.size() == n ? c->coarse_row_first.data() : nullptr;
  c->cdev.Ac32 = nullptr;
  // Cholesky, W = L^-1, Ac^-1 = W^T W on the project's dense tile kernels:
  // FP32 arithmetic for the FP32 / TF32-class options (the inverse is
  // rounded to FP32 or BF16 afterwards anyway), FP64 otherwise
  const bool f64 = c->coarse_inverse < 2;
  const size_t B = (size_t)dense_tile(f64), N = ((size_t)n + B - 1) / B * B;
  const size_t work = 2 * N * N * (f64 ? sizeof(double) : sizeof(float)) + (f64 ? 0 : (size_t)n * n * sizeof(float));
  if (work > c->dense_bytes) {
    CK(cudaStreamSynchronize(c->stream));
    if (c->dense_work) cudaFree(c->dense_work);
    c->dense_work = nullptr;
    c->dense_bytes = 0;
    CK(cudaMalloc(&c->dense_work, work));
    c->dense_bytes = work;
  }
  if (!c->dense_info) CK(cudaMalloc(reinterpret_cast<void**>(&c->dense_info), sizeof(int)));
  if (!c->h_info) CK(cudaMallocHost(reinterpret_cast<void**>(&c->h_info), sizeof(int)));
  int nl = 0;
  cudaError_t de;
  if (f64) {
    double* A = static_cast<double*>(c->dense_work);
    de = dense_spd_inverse_f64(c->cdev.Ac, n, A, A + N * N, c->dense_info, c->cdev.Ac, c->stream, &nl,
                               &c->dense_sched, row_first);
  } else {
    float* A = static_cast<float*>(c->dense_work);
    float* out = A + 2 * N * N;
    de = c->coarse_inverse == 3
             ? dense_spd_inverse_tf32(c->cdev.Ac, n, A, A + N * N, c->dense_info, out, c->stream, &nl,
                                      &c->dense_sched, row_first)
             : dense_spd_inverse_f32(c->cdev.Ac, n, A, A + N * N, c->dense_info, out, c->stream, &nl,
                                     &c->dense_sched, row_first);
    c->cdev.Ac32 = out;
  }
  if (de != cudaSuccess) return set_err(c, FEM_ERR_CUDA, "dense inverse: %s", cudaGetErrorString(de));
  c->n_launches += nl;
  CK(cudaMemcpyAsync(c->h_info, c->dense_info, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (*c->h_info < 0) {
    c->cdev.Ac32 = nullptr;
    return set_err(c, FEM_ERR_BUDGET, "coarse inverse: a tensor-core completion wait timed out");
  }
  if (*c->h_info != 0) {
    c->cdev.Ac32 = nullptr;
    return keep_previous_coarse(c, *c->h_info);
  }
  launch_coarse_symmetrize(c->cdev, c->stream);
  ++c->n_launches;
  CKL();
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f, ms_asm = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventElapsedTime(&ms_asm, e0, em);
  c->coarse_ms_last = ms;
  c->coarse_ms_assembly = ms_asm;
  ++c->n_coarse_assemblies;
  c->coarse_have_inverse = true;
  c->coarse_valid = true;
  c->coarse_uses = 1;
  c->coarse_base_ipd = -1;
  return FEM_OK;
}

template <typename T>
int mpnn_alloc(FemCtx* c, T** dst, size_t n) {
  int st;
  if ((st = dalloc(c, dst, n))) return st;
  c->mpnn_bufs.push_back(*dst);
  return FEM_OK;
}

// Node graph of the learned preconditioner (nodes sharing an element, ids
// ascending), activations and weight buffers; the log-modulus node feature is
// refreshed whenever the material tables change.
int ensure_mpnn(FemCtx* c) {
  const int Nn = c->Nn, Ne = c->Ne;
  int st;
  if (!c->mpnn_built) {
    std::vector<int4> conn(Ne);
    CK(cudaMemcpyAsync(conn.data(), c->conn, conn.size() * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<uint64_t> pairs;
    pairs.reserve((size_t)Ne * 12);
    for (int e = 0; e < Ne; ++e) {
      const int* cn = &conn[e].x;
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b)
          if (a != b) pairs.push_back(((uint64_t)(uint32_t)cn[a] << 32) | (uint32_t)cn[b]);
    }
    std::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    std::vector<int> ptr(Nn + 1, 0), idx(pairs.size());
    for (size_t k = 0; k < pairs.size(); ++k) {
      ptr[(pairs[k] >> 32) + 1]++;
      idx[k] = (int)(pairs[k] & 0xffffffffu);
    }
    for (int i = 0; i < Nn; ++i) ptr[i + 1] += ptr[i];
    std::vector<float> dinv(Nn);
    for (int i = 0; i < Nn; ++i) dinv[i] = ptr[i + 1] > ptr[i] ? 1.0f / (float)(ptr[i + 1] - ptr[i]) : 0.f;
    MpnnDev& m = c->mdev;
    int *d_ptr, *d_idx;
    float* d_deg;
    if ((st = mpnn_alloc(c, &d_ptr, ptr.size()))) return st;
    if ((st = mpnn_alloc(c, &d_idx, idx.size()))) return st;
    if ((st = mpnn_alloc(c, &d_deg, dinv.size()))) return st;
    if ((st = mpnn_alloc(c, &c->cfeat, (size_t)Nn))) return st;
    CK(cudaMemcpyAsync(d_ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_idx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_deg, dinv.data(), dinv.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    m.n_nodes = Nn;
    m.adj_ptr = d_ptr;
    m.adj_idx = d_idx;
    m.deg_inv = d_deg;
    m.cfeat = c->cfeat;
    m.fixed = c->fixed;
    for (int l = 0; l <= kMpnnLayers; ++l) {
      __nv_bfloat16* h;
      if ((st = mpnn_alloc(c, &h, (size_t)Nn * kMpnnHidden))) return st;
      m.H[l] = h;
    }
    for (int l = 0; l < kMpnnLayers; ++l) {
      uint64_t* mk;
      if ((st = mpnn_alloc(c, &mk, (size_t)Nn))) return st;
      m.mask[l] = mk;
    }
    double* scal;
    int* err;
    if ((st = mpnn_alloc(c, &scal, (size_t)4))) return st;
    if ((st = mpnn_alloc(c, &err, (size_t)1))) return st;
    m.scal = scal;
    m.err = err;
    if (!c->h_err) CK(cudaMallocHost(reinterpret_cast<void**>(&c->h_err), sizeof(int)));
    if ((st = mpnn_alloc(c, &c->zalt, 4 * (size_t)Nn))) return st;
    CK(cudaStreamSynchronize(c->stream));
    c->mpnn_built = true;
  }
  if (!c->mpnn_feat_valid) {
    if (c->elem_modulus.size() != (size_t)Ne)
      return set_err(c, FEM_ERR_STATE, "learned preconditioner: materials not set");
    std::vector<int4> conn(Ne);
    CK(cudaMemcpyAsync(conn.data(), c->conn, conn.size() * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<double> acc(Nn, 0.0), cnt(Nn, 0.0);
    for (int e = 0; e < Ne; ++e) {
      const int* cn = &conn[e].x;
      for (int a = 0; a < 4; ++a) {
        acc[cn[a]] += c->elem_modulus[e];
        cnt[cn[a]] += 1.0;
      }
    }
    double mean = 0.0;
    std::vector<double> lm(Nn);
    for (int i = 0; i < Nn; ++i) {
      lm[i] = cnt[i] > 0 ? std::log(acc[i] / cnt[i]) : 0.0;
      mean += lm[i];
    }
    mean /= std::max(Nn, 1);
    std::vector<float> cf(Nn);
    for (int i = 0; i < Nn; ++i) cf[i] = (float)(lm[i] - mean);
    CK(cudaMemcpyAsync(c->cfeat, cf.data(), cf.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->mpnn_feat_valid = true;
  }
  return FEM_OK;
}

int ensure_mpnn_train(FemCtx* c) {
  if (c->mpnn_train_ready) return FEM_OK;
  const size_t Nn = (size_t)c->Nn;
  const int tiles = (c->Nn + 127) / 128;
  int st;
  MpnnTrain& t = c->mtrain;
  if ((st = mpnn_alloc(c, &t.GH, Nn * kMpnnHidden))) return st;
  if ((st = mpnn_alloc(c, &t.GHn, Nn * kMpnnHidden))) return st;
  if ((st = mpnn_alloc(c, &t.Q, Nn * kMpnnHidden))) return st;
  if ((st = mpnn_alloc(c, &t.gpart, (size_t)tiles * kMpnnParams))) return st;
  if ((st = mpnn_alloc(c, &c->grad, (size_t)kMpnnParams))) return st;
  if ((st = mpnn_alloc(c, &c->adam_m, (size_t)kMpnnParams))) return st;
  if ((st = mpnn_alloc(c, &c->adam_v, (size_t)kMpnnParams))) return st;
  for (float** v : {&c->tr_r, &c->tr_e, &c->tr_z, &c->tr_q, &c->tr_g})
    if ((st = mpnn_alloc(c, v, 4 * Nn))) return st;
  if ((st = mpnn_alloc(c, &c->tr_scal, (size_t)4))) return st;
  c->mpnn_train_ready = true;
  return FEM_OK;
}

// Everything a learned-preconditioner call needs at the current tangent.
int mpnn_prepare(FemCtx* c, bool train, bool coarse) {
  int st;
  if (!c->tangent_valid) return set_err(c, FEM_ERR_STATE, "no tangent state: evaluate forces first");
  if (!c->mpnn_has_weights) return set_err(c, FEM_ERR_STATE, "learned preconditioner has no weights");
  if ((st = compute_dinv(c, FEM_PRECOND_JACOBI))) return st;
  if ((st = ensure_mpnn(c))) return st;
  if (train && (st = ensure_mpnn_train(c))) return st;
  if (coarse && (st = ensure_coarse(c))) return st;
  prepare_mpnn_kernels();
  CK(cudaMemsetAsync(c->mdev.err, 0, sizeof(int), c->stream));
  c->mtrain.m = c->mdev;
  return FEM_OK;
}

// z = M(r) (+ coarse) on internal float4 vectors; base: D^-1 r (+ coarse) instead
void mpnn_apply(FemCtx* c, const float* r, float* z, bool coarse, bool base) {
  if (base) {
    launch_jacobi_apply(r, c->dinv, z, c->Nn, c->stream);
    ++c->n_launches;
  } else {
    launch_mpnn_forward(c->mdev, r, c->dinv, z, nullptr, c->red(), SITE_RZ, c->stream);
    c->n_launches += 6;
  }
  if (coarse) {
    const CoarseArgs ca = coarse_args(c);
    launch_coarse_apply(ca, r, nullptr, c->stream);
    launch_coarse_add(ca, z, c->stream);
    c->n_launches += 3 + coarse_product_kernels(c->cdev);
  }
}

MvArgs train_mv(FemCtx* c, const float* x, float* y) {
  MvArgs mv = make_mv(c);
  mv.matF = c->matF;
  mv.payload = c->payload;
  mv.x = x;
  mv.y = y;
  mv.cg = nullptr;
  mv.red = c->red();
  mv.red_site = SITE_MV;
  mv.mask_input = 1;
  return mv;
}

// One training / evaluation sample k: loss into tr_scal[0] (+=), and with
// grad: dL/dw added (accumulate) or written into c->grad.
void mpnn_sample(FemCtx* c, const float* R, const float* E, int k, bool coarse, bool base, bool grad,
                 bool accumulate) {
  const size_t stride = 3 * (size_t)c->Nn;
  launch_gather_f(R + stride * k, c->tr_r, c->d_perm_node, c->Nn, c->stream);
  launch_gather_f(E + stride * k, c->tr_e, c->d_perm_node, c->Nn, c->stream);
  mpnn_apply(c, c->tr_r, c->tr_z, coarse, base);
  launch_matvec(train_mv(c, c->tr_z, c->tr_q), c->model_kind, c->stream);
  launch_train_loss(c->tr_z, c->tr_q, c->tr_r, c->tr_e, c->Nn, c->tr_scal, c->red(), SITE_AUX, c->stream);
  c->n_launches += 4 + (c->mv_variant == MV_FUSED ? 0 : 1);
  if (grad) {
    launch_train_grad_z(c->tr_q, c->tr_r, c->fixed, c->tr_scal, c->tr_g, c->Nn, c->stream);
    launch_mpnn_backward(c->mtrain, c->tr_r, c->dinv, c->tr_g, c->grad, accumulate ? 1 : 0, c->stream);
    c->n_launches += 1 + 2 + 2 * kMpnnLayers + 1;
  }
}

// Solves K_T x = b (b: FP64 internal order, fixed DOFs zero) into c->x.
int run_pcg(FemCtx* c, const double* b_int, int precond, double rtol, int maxit, int* iters,
            double* rel) {
  if (!c->tangent_valid) return set_err(c, FEM_ERR_STATE, "no tangent state: evaluate forces first");
  int st;
  if (c->npe == 8 && precond == FEM_PRECOND_LEARNED) {
    // the learned network is trained on TET4 graphs: a HEX8 context runs
    // these solves as Jacobi-PCG
    ++c->n_coarse_fallbacks;
    precond = FEM_PRECOND_JACOBI;
  }
  const bool tl = precond == FEM_PRECOND_TWO_LEVEL;
  const bool learned = precond == FEM_PRECOND_LEARNED;
  const int kind = learned ? GRAPH_LEARNED : (tl ? GRAPH_TWO_LEVEL : GRAPH_JACOBI);
  if (learned && !c->mpnn_has_weights)
    return set_err(c, FEM_ERR_STATE, "learned preconditioner has no weights (fem_mpnn_set_weights)");
  if ((st = compute_dinv(c, (tl || learned) ? FEM_PRECOND_JACOBI : precond, tl && c->block_jacobi))) return st;
  if (tl && (st = ensure_coarse(c))) {
    // no positive definite coarse operator on this lattice yet (e.g. cells
    // finer than the elements of an anisotropic mesh): this solve runs as
    // Jacobi-PCG instead of failing
    if (st != FEM_ERR_NAN) return st;
    ++c->n_coarse_fallbacks;
    return run_pcg(c, b_int, FEM_PRECOND_JACOBI, rtol, maxit, iters, rel);
  }
  if (learned && c->learned_coarse && (st = ensure_coarse(c))) return st;
  if (learned && (st = ensure_mpnn(c))) return st;
  if ((st = ensure_cg_graph(c, kind))) return st;
  const bool fused = (c->cg_graph_flags[kind] & 2) != 0;
  if (fused) CK(cudaMemsetAsync(c->step_bar, 0, 4 * sizeof(unsigned int), c->stream));
  if (learned) CK(cudaMemsetAsync(c->mdev.err, 0, sizeof(int), c->stream));
  ++c->n_launches; launch_cg_init(b_int, c->r, c->x, c->p, c->dinv, c->Nn, c->cg, rtol, maxit, c->red(), SITE_CGI,
                 c->stream, (tl || learned) ? 0 : 1);
  CKL();
  if (learned) {
    const CoarseArgs ca = coarse_args(c);
    launch_mpnn_forward(c->mdev, c->r, c->dinv, c->tmpf, c->cg, c->red(), SITE_RZ, c->stream);
    if (c->learned_coarse) launch_coarse_apply(ca, c->r, c->cg, c->stream);
    launch_fpcg_dots(ca, true, c->learned_coarse, c->r, c->y, c->dinv, c->tmpf, c->zalt, c->p, c->cg, c->red(),
                     SITE_RZ, SITE_RZ2, c->stream);
    launch_fpcg_pupdate(c->p, c->tmpf, c->zalt, c->Nn, c->cg, true, c->stream);
    c->n_launches += 6 + 2 + (c->learned_coarse ? 2 + coarse_product_kernels(c->cdev) : 0);
    CKL();
  }
  if (tl) {
    const CoarseArgs ca = coarse_args(c);
    launch_coarse_apply(ca, c->r, c->cg, c->stream);
    launch_tl_rz(ca, true, c->r, c->dinv, c->tmpf, c->p, c->cg, c->red(), SITE_RZ, c->stream);
    c->n_launches += 3 + coarse_product_kernels(c->cdev);
    CKL();
  }
  const int max_batches = maxit / cg_batch(kind) + 2;
  int batches = 0;
  if (c->loop_graph[kind]) {
    // no host check first: a state that is done already makes the body's
    // kernels exit at entry and the condition kernel end the loop
    CK(cudaGraphLaunch(c->loop_graph[kind], c->stream));
    c->n_graphs++;
    c->n_loop_graphs++;
    CK(cudaMemcpyAsync(c->h_cg, c->cg, sizeof(CGState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    batches = max_batches;
  } else {
    CK(cudaMemcpyAsync(c->h_cg, c->cg, sizeof(CGState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  while (!c->h_cg->done && batches < max_batches) {
    CK(cudaGraphLaunch(c->cg_graph[kind], c->stream));
    c->n_graphs++;
    CK(cudaMemcpyAsync(c->h_cg, c->cg, sizeof(CGState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    ++batches;
  }
  const CGState& h = *c->h_cg;
  c->n_cg_iters += h.iter;
  if ((tl || (learned && c->learned_coarse)) && c->coarse_reuse < 0 && h.done == 1 && h.rr0 > 0 && h.rr > 0) {
    // adaptive reuse: iterations per decade of residual reduction; once a
    // solve needs 1.5x the rate measured right after the assembly, the coarse
    // operator is rebuilt at the next tangent
    const double decades = std::max(0.5 * std::log10(h.rr0 / h.rr), 0.25);
    const double ipd = h.iter / decades;
    if (c->coarse_base_ipd < 0)
      c->coarse_base_ipd = ipd;
    else if (ipd > 1.5 * c->coarse_base_ipd + 2.0)
      c->coarse_valid = false;
  }
  // kernels that did work: 3 (Jacobi), 6 (two-level) or 11 + 2 (learned,
  // + coarse) per CG iteration; the rest of a batch exits at entry
  if (learned) {
    // the network's 6 kernels run until it is switched off (after 3 rejected steps)
    const int64_t net_steps = std::max<int64_t>(0, (int64_t)h.iter - h.n_alt + std::min(h.n_alt, 3));
    c->n_launches += (5LL + (c->learned_coarse ? 2 + coarse_product_kernels(c->cdev) : 0)) * h.iter + 6LL * net_steps;
  } else {
    c->n_launches += kernels_per_iter(c, kind, fused) * h.iter;
  }
  if (learned) {
    c->n_alt_steps += h.n_alt;
    c->n_learned_steps += h.iter;
    CK(cudaMemcpyAsync(c->h_err, c->mdev.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (*c->h_err) return set_err(c, FEM_ERR_BUDGET, "learned preconditioner: tensor-core wait gave up");
    if (h.done == 4) {
      // the network was switched off: the rest of the solve runs as plain
      // (two-level or Jacobi) PCG on the current residual, its solution added
      // to the flexible iterate, to the same absolute residual target
      ++c->n_handovers;
      const int iters_done = h.iter;
      const double tol2 = h.tol2, rr_now = h.rr, rr0 = h.rr0;
      if (!c->ho_x && ((st = dalloc(c, &c->ho_x, 4 * (size_t)c->Nn)) || (st = dalloc(c, &c->ho_rhs, (size_t)c->ndof_pad))))
        return st;
      CK(cudaMemcpyAsync(c->ho_x, c->x, 4 * (size_t)c->Nn * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
      ++c->n_launches; launch_f4_to_d3(c->r, c->ho_rhs, c->Nn, c->stream);
      CKL();
      const double rtol2 = rr_now > 0.0 ? std::min(1.0, std::sqrt(tol2 / rr_now)) : 1.0;
      int it2 = 0;
      double rel2 = 0;
      const int fb = c->learned_coarse ? FEM_PRECOND_TWO_LEVEL : FEM_PRECOND_JACOBI;
      st = run_pcg(c, c->ho_rhs, fb, rtol2, std::max(1, maxit - iters_done), &it2, &rel2);
      if (st && st != FEM_NOT_CONVERGED) return st;
      ++c->n_launches; launch_f4_add(c->x, c->ho_x, c->Nn, c->stream);
      CKL();
      if (iters) *iters = iters_done + it2;
      if (rel) *rel = rr0 > 0 ? rel2 * std::sqrt(rr_now / rr0) : 0.0;
      return st;
    }
    if (h.done == 2 || h.done == 3) {
      // Jacobi-based PCG is the fallback: the flexible solve broke down or ran
      // out of iterations; the same convergence test judges the rerun
      ++c->n_fallbacks;
      int it2 = 0;
      double rel2 = 0;
      const int fb = c->learned_coarse ? FEM_PRECOND_TWO_LEVEL : FEM_PRECOND_JACOBI;
      const int iters_done = h.iter;
      st = run_pcg(c, b_int, fb, rtol, maxit, &it2, &rel2);
      if (iters) *iters = iters_done + it2;
      if (rel) *rel = rel2;
      return st;
    }
  }
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
  const int npe = desc->nodes_per_elem == 0 ? 4 : desc->nodes_per_elem;
  if (npe != 4 && npe != 8)
    return set_err(nullptr, FEM_ERR_INVALID, "nodes_per_elem must be 4 (TET4) or 8 (HEX8), got %d",
                   desc->nodes_per_elem);
  if (npe == 8 && desc->n_elements > (1LL << 27))
    return set_err(nullptr, FEM_ERR_INVALID, "HEX8 mesh too large for 32-bit slot tables");
  for (int64_t i = 0; i < npe * desc->n_elements; ++i)
    if (desc->conn[i] < 0 || desc->conn[i] >= desc->n_nodes)
      return set_err(nullptr, FEM_ERR_INVALID, "connectivity entry %lld = %d out of range [0, %lld)",
                     (long long)i, desc->conn[i], (long long)desc->n_nodes);
  for (int64_t e = 0; e < desc->n_elements; ++e) {
    const int32_t* cn = desc->conn + npe * e;
    for (int a = 0; a < npe; ++a)
      for (int b = a + 1; b < npe; ++b)
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
  c->npe = npe;
  c->ngp = npe == 8 ? kHexGauss : 1;
  c->Nq = (size_t)c->Ne * c->ngp;
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
  out[4] = c->mv_variant;
  out[5] = (int64_t)std::llround(c->mv_ns[MV_FUSED]);
  out[6] = (int64_t)std::llround(c->mv_ns[MV_TWO_PHASE]);
  out[7] = c->mv_tuned ? 1 : 0;
  out[8] = c->n_loop_graphs;
  out[9] = c->use_loop_graph ? 1 : 0;
  out[10] = (int64_t)std::llround(c->mv_ns[MV_ELEM_BLOCK]);
  out[11] = c->eb_size;
  for (int k = 0; k < 4; ++k) out[12 + k] = (int64_t)std::llround(c->eb_ns[k]);
  out[16] = (int64_t)std::llround(c->mv_ns[MV_WARP_AGG]);
  out[17] = (int64_t)std::llround(c->mv_ns[MV_PERSIST]);
  return FEM_OK;
}

int fem_learned_stats(void* ctx, int64_t* out4) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  if (!c || !out4) return FEM_ERR_INVALID;
  out4[0] = c->n_fallbacks;
  out4[1] = c->mpnn_has_weights ? 1 : 0;
  out4[2] = c->n_learned_steps;
  out4[3] = c->n_alt_steps;
  return FEM_OK;
}

int fem_set_option(void* ctx, int32_t key, int64_t value) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  switch (key) {
    case FEM_OPT_MATVEC_VARIANT:
      if (value < -1 || value >= MV_N_VARIANTS)
        return set_err(c, FEM_ERR_INVALID,
                       "matvec variant %lld not in {-1 (auto), 0 (fused), 1 (two-phase), 2 (element-block), "
                       "3 (warp-aggregated), 4 (persistent two-phase)}",
                       (long long)value);
      if (value == MV_ELEM_BLOCK && c->npe != 4)
        return set_err(c, FEM_ERR_INVALID, "the element-block matvec is TET4 only");
      if (value == MV_WARP_AGG && c->npe != 4)
        return set_err(c, FEM_ERR_INVALID, "the warp-aggregated matvec is TET4 only");
      if (value == MV_PERSIST && c->npe != 4)
        return set_err(c, FEM_ERR_INVALID, "the persistent two-phase matvec is TET4 only");
      // table-driven variants are only ever selected with their tables built
      if (value == MV_ELEM_BLOCK && (st = build_eb_tables(c, c->eb_forced > 0 ? c->eb_forced : 512))) return st;
      if (value == MV_WARP_AGG && (st = build_wagg_tables(c))) return st;
      c->mv_forced = (int)value;
      c->mv_variant = value >= 0 ? (int)value : MV_FUSED;
      c->mv_tuned = false;
      return FEM_OK;
    case FEM_OPT_EXTRAPOLATE:
      if (value != 0 && value != 1) return set_err(c, FEM_ERR_INVALID, "extrapolation flag must be 0 or 1");
      c->extrap = value != 0;
      c->extrap_ready = false;
      return FEM_OK;
    case FEM_OPT_RESIDUAL_TWO_PHASE:
      if (value != 0 && value != 1) return set_err(c, FEM_ERR_INVALID, "residual variant flag must be 0 or 1");
      c->res_two_phase = value != 0;
      return FEM_OK;
    case FEM_OPT_EB_SIZE:
      if (value != 0 && value != 256 && value != 512 && value != 768 && value != 1024)
        return set_err(c, FEM_ERR_INVALID, "element block size %lld: 0 (timed), 256, 512, 768 or 1024",
                       (long long)value);
      c->eb_forced = (int)value;
      c->mv_tuned = false;
      if (c->mv_variant == MV_ELEM_BLOCK) return build_eb_tables(c, c->eb_forced > 0 ? c->eb_forced : 512);
      if (c->eb_size != 0) free_eb_tables(c);
      return FEM_OK;
    case FEM_OPT_COARSE_CELL:
      if (value < 1 || value > 64)
        return set_err(c, FEM_ERR_INVALID, "coarse cell edge %lld not in [1, 64] mesh lengths", (long long)value);
      if (value != c->coarse_cell_voxels) {
        c->coarse_cell_voxels = (int)value;
        return drop_coarse(c);
      }
      return FEM_OK;
    case FEM_OPT_COARSE_BF16:
      if (value != 0 && value != 1) return set_err(c, FEM_ERR_INVALID, "coarse BF16 flag must be 0 or 1");
      if ((value != 0) != c->coarse_bf16) {
        c->coarse_bf16 = value != 0;
        return drop_coarse(c);
      }
      return FEM_OK;
    case FEM_OPT_LEARNED_COARSE:
      if (value != 0 && value != 1) return set_err(c, FEM_ERR_INVALID, "learned coarse flag must be 0 or 1");
      c->learned_coarse = value != 0;
      return FEM_OK;
    case FEM_OPT_WHOLE_SOLVE_GRAPH:
      if (value != 0 && value != 1) return set_err(c, FEM_ERR_INVALID, "whole-solve graph flag must be 0 or 1");
      if ((value != 0) != c->use_loop_graph) {
        CK(cudaStreamSynchronize(c->stream));
        // recaptured on the next solve, with or without the loop graph
        for (int k = 0; k < N_GRAPHS; ++k) {
          if (c->cg_graph[k]) cudaGraphExecDestroy(c->cg_graph[k]);
          if (c->loop_graph[k]) cudaGraphExecDestroy(c->loop_graph[k]);
          c->cg_graph[k] = nullptr;
          c->loop_graph[k] = nullptr;
        }
        c->use_loop_graph = value != 0;
      }
      return FEM_OK;
    case FEM_OPT_COARSE_MAX_NODES:
      if (value < 8 || value > kMaxCoarseNodesLimit)
        return set_err(c, FEM_ERR_INVALID, "coarse node cap %lld not in [8, %d]", (long long)value,
                       kMaxCoarseNodesLimit);
      if (value != c->coarse_max_nodes) {
        c->coarse_max_nodes = (int)value;
        return drop_coarse(c);
      }
      return FEM_OK;
    case FEM_OPT_COARSE_INVERSE:
      if (value < 0 || value > 3) return set_err(c, FEM_ERR_INVALID, "coarse inverse method must be 0 to 3");
      c->coarse_inverse = (int)value;
      return FEM_OK;
    case FEM_OPT_BLOCK_JACOBI:
      if (value != 0 && value != 1) return set_err(c, FEM_ERR_INVALID, "block smoother flag must be 0 or 1");
      c->block_jacobi = value != 0;
      return FEM_OK;
    case FEM_OPT_DIRECTION_RECURRENCE:
      if (value != 0 && value != 1) return set_err(c, FEM_ERR_INVALID, "direction recurrence flag must be 0 or 1");
      c->direction_recurrence = value != 0;
      return FEM_OK;
    case FEM_OPT_PDL:
      if (value != 0 && value != 1) return set_err(c, FEM_ERR_INVALID, "programmatic launch flag must be 0 or 1");
      c->pdl = value != 0;
      return FEM_OK;
    case FEM_OPT_FUSED_STEP:
      if (value != 0 && value != 1) return set_err(c, FEM_ERR_INVALID, "fused step flag must be 0 or 1");
      c->fused_step = value != 0;
      return FEM_OK;
    case FEM_OPT_COARSE_REUSE:
      if (value < -1 || value > (1 << 20))
        return set_err(c, FEM_ERR_INVALID, "coarse reuse count %lld not in [-1, 2^20]", (long long)value);
      c->coarse_reuse = (int)value;
      return FEM_OK;
    default:
      return set_err(c, FEM_ERR_INVALID, "unknown option key %d", key);
  }
}

int fem_mpnn_set_weights(void* ctx, const float* w, int64_t n) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!w || n != kMpnnParams)
    return set_err(c, FEM_ERR_INVALID, "learned preconditioner takes %d parameters (got %lld)", kMpnnParams,
                   (long long)n);
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(w[i])) return set_err(c, FEM_ERR_INVALID, "parameter %lld is not finite", (long long)i);
  if (!c->mpnn_w) {
    if ((st = mpnn_alloc(c, &c->mpnn_w, (size_t)kMpnnParams))) return st;
    if ((st = mpnn_alloc(c, &c->We_p, (size_t)kMpnnHidden * kMpnnIn))) return st;
    if ((st = mpnn_alloc(c, &c->Wl_p, (size_t)kMpnnLayers * kMpnnHidden * 2 * kMpnnHidden))) return st;
    if ((st = mpnn_alloc(c, &c->WlT_p, (size_t)kMpnnLayers * kMpnnHidden * 2 * kMpnnHidden))) return st;
  }
  CK(cudaMemcpyAsync(c->mpnn_w, w, sizeof(float) * kMpnnParams, cudaMemcpyHostToDevice, c->stream));
  ++c->n_launches; launch_mpnn_pack(c->mpnn_w, c->We_p, c->Wl_p, c->WlT_p, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  c->mdev.w = c->mpnn_w;
  c->mdev.We_p = c->We_p;
  c->mdev.Wl_p = c->Wl_p;
  c->mdev.WlT_p = c->WlT_p;
  c->mpnn_has_weights = true;
  return FEM_OK;
}

int fem_mpnn_get_weights(void* ctx, float* w, int64_t n) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!w || n != kMpnnParams)
    return set_err(c, FEM_ERR_INVALID, "learned preconditioner has %d parameters (got %lld)", kMpnnParams,
                   (long long)n);
  if (!c->mpnn_has_weights) return set_err(c, FEM_ERR_STATE, "learned preconditioner has no weights");
  CK(cudaMemcpyAsync(w, c->mpnn_w, sizeof(float) * kMpnnParams, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int fem_mpnn_forward(void* ctx, const float* r, float* z) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!r || !z) return set_err(c, FEM_ERR_INVALID, "null vector");
  if (!c->tangent_valid) return set_err(c, FEM_ERR_STATE, "no tangent state: evaluate forces first");
  if (!c->mpnn_has_weights) return set_err(c, FEM_ERR_STATE, "learned preconditioner has no weights");
  if ((st = compute_dinv(c, FEM_PRECOND_JACOBI))) return st;
  if ((st = ensure_mpnn(c))) return st;
  prepare_mpnn_kernels();
  CK(cudaMemsetAsync(c->mdev.err, 0, sizeof(int), c->stream));
  ++c->n_launches; launch_gather_f(r, c->r, c->d_perm_node, c->Nn, c->stream);
  launch_mpnn_forward(c->mdev, c->r, c->dinv, c->y, nullptr, c->red(), SITE_RZ, c->stream);
  c->n_launches += 6;
  CKL();
  ++c->n_launches; launch_scatter_f(c->y, z, c->d_perm_node, c->Nn, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->h_err, c->mdev.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (*c->h_err) return set_err(c, FEM_ERR_BUDGET, "learned preconditioner: tensor-core wait gave up");
  return FEM_OK;
}

int fem_mpnn_backward(void* ctx, const float* r, const float* gz, float* grad_out) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!r || !gz || !grad_out) return set_err(c, FEM_ERR_INVALID, "null argument");
  if ((st = mpnn_prepare(c, true, false))) return st;
  launch_gather_f(r, c->tr_r, c->d_perm_node, c->Nn, c->stream);
  launch_gather_f(gz, c->tr_g, c->d_perm_node, c->Nn, c->stream);
  mpnn_apply(c, c->tr_r, c->tr_z, false, false);
  launch_mpnn_backward(c->mtrain, c->tr_r, c->dinv, c->tr_g, c->grad, 0, c->stream);
  c->n_launches += 2 + 2 + 2 * kMpnnLayers + 1;
  CKL();
  CK(cudaMemcpyAsync(grad_out, c->grad, sizeof(float) * kMpnnParams, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->h_err, c->mdev.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (*c->h_err) return set_err(c, FEM_ERR_BUDGET, "learned preconditioner: tensor-core wait gave up");
  return FEM_OK;
}

int fem_mpnn_eval(void* ctx, const float* R, const float* E, int32_t n_pairs, double* loss_net,
                  double* loss_base) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!R || !E || n_pairs <= 0) return set_err(c, FEM_ERR_INVALID, "need pair arrays and n_pairs > 0");
  const bool coarse = c->learned_coarse;
  if ((st = mpnn_prepare(c, true, coarse))) return st;
  double h[2];
  for (int pass = 0; pass < 2; ++pass) {
    CK(cudaMemsetAsync(c->tr_scal, 0, 2 * sizeof(double), c->stream));
    for (int k = 0; k < n_pairs; ++k) mpnn_sample(c, R, E, k, coarse, pass == 1, false, false);
    CKL();
    CK(cudaMemcpyAsync(&h[pass], c->tr_scal, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  if (loss_net) *loss_net = h[0] / n_pairs;
  if (loss_base) *loss_base = h[1] / n_pairs;
  return FEM_OK;
}

int fem_mpnn_train(void* ctx, const float* R, const float* E, int32_t n_pairs, const FemTrainParams* prm,
                   FemTrainResult* res) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!R || !E || n_pairs <= 0 || !prm) return set_err(c, FEM_ERR_INVALID, "need pairs, n_pairs > 0, params");
  if (prm->steps <= 0 || prm->batch <= 0 || !(prm->lr > 0))
    return set_err(c, FEM_ERR_INVALID, "need steps > 0, batch > 0, lr > 0");
  const bool coarse = c->learned_coarse;
  if ((st = mpnn_prepare(c, true, coarse))) return st;
  if (prm->reset_optimizer || c->adam_t == 0) {
    CK(cudaMemsetAsync(c->adam_m, 0, sizeof(float) * kMpnnParams, c->stream));
    CK(cudaMemsetAsync(c->adam_v, 0, sizeof(float) * kMpnnParams, c->stream));
    c->adam_t = 0;
  }
  std::vector<double> losses(prm->steps);
  // sample order: a fixed permutation per epoch (seeded LCG), batches in order
  std::vector<int> order(n_pairs);
  uint64_t state = 0x9E3779B97F4A7C15ull ^ (uint64_t)(uint32_t)prm->seed;
  auto next = [&]() {
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    return (uint32_t)(state >> 33);
  };
  int pos = n_pairs;
  for (int step = 0; step < prm->steps; ++step) {
    CK(cudaMemsetAsync(c->tr_scal, 0, 2 * sizeof(double), c->stream));
    for (int b = 0; b < prm->batch; ++b) {
      if (pos >= n_pairs) {
        std::iota(order.begin(), order.end(), 0);
        for (int i = n_pairs - 1; i > 0; --i) std::swap(order[i], order[next() % (uint32_t)(i + 1)]);
        pos = 0;
      }
      mpnn_sample(c, R, E, order[pos++], coarse, false, true, b > 0);
    }
    ++c->adam_t;
    launch_mpnn_adam(c->mpnn_w, c->adam_m, c->adam_v, c->grad, 1.0f / prm->batch, (float)prm->lr, c->adam_t,
                     c->stream);
    launch_mpnn_pack(c->mpnn_w, c->We_p, c->Wl_p, c->WlT_p, c->stream);
    c->n_launches += 2;
    CKL();
    CK(cudaMemcpyAsync(&losses[step], c->tr_scal, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (prm->progress && (step % 16 == 15 || step + 1 == prm->steps)) {
      CK(cudaStreamSynchronize(c->stream));
      if (!prm->progress(prm->progress_user, step + 1, losses[step] / prm->batch, 0.0)) {
        if (res) res->steps_done = step + 1;
        return FEM_CANCELLED;
      }
    }
  }
  CK(cudaMemcpyAsync(c->h_err, c->mdev.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (*c->h_err) return set_err(c, FEM_ERR_BUDGET, "learned preconditioner: tensor-core wait gave up");
  if (res) {
    res->steps_done = prm->steps;
    const int w = std::max(1, std::min(prm->steps / 10, 16));
    double a = 0, b = 0;
    for (int i = 0; i < w; ++i) {
      a += losses[i];
      b += losses[prm->steps - 1 - i];
    }
    res->loss_first = a / (w * prm->batch);
    res->loss_last = b / (w * prm->batch);
  }
  return FEM_OK;
}

int fem_coarse_info(void* ctx, double* out10) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  if (!c || !out10) return FEM_ERR_INVALID;
  double* out8 = out10;
  double* out6 = out10;
  out10[8] = (double)c->n_coarse_kept;
  out10[9] = (double)c->n_coarse_fallbacks;
  out8[6] = c->coarse_ms_assembly;
  out8[7] = (double)c->coarse_reuse;
  out6[0] = c->cdev.n_cells;
  out6[1] = c->cdev.n_cn;
  out6[2] = c->cdev.n_dof;
  out6[3] = c->coarse_H;
  out6[4] = (double)c->n_coarse_assemblies;
  out6[5] = c->coarse_ms_last;
  return FEM_OK;
}

int fem_step_info(void* ctx, int64_t* out6) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  if (!c || !out6) return FEM_ERR_INVALID;
  int64_t* out4 = out6;
  out6[4] = (c->cg_graph[GRAPH_JACOBI] && (c->cg_graph_flags[GRAPH_JACOBI] & 4)) ? 1 : 0;
  out6[5] = (c->cg_graph[GRAPH_TWO_LEVEL] && (c->cg_graph_flags[GRAPH_TWO_LEVEL] & 4)) ? 1 : 0;
  out4[0] = (c->fused_step && c->fused_ok) ? 1 : 0;
  out4[1] = (c->cg_graph[GRAPH_JACOBI] && (c->cg_graph_flags[GRAPH_JACOBI] & 2)) ? 1 : 0;
  out4[2] = (c->cg_graph[GRAPH_TWO_LEVEL] && (c->cg_graph_flags[GRAPH_TWO_LEVEL] & 2)) ? 1 : 0;
  out4[3] = c->cdev.r_slices;
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
  // stiffness scale per element for the learned preconditioner's node feature
  c->elem_modulus.assign(c->Ne, 0.0);
  for (int e = 0; e < c->Ne; ++e) {
    const FemMaterial& s = table[ids[e]];
    double mod;
    if (s.model == FEM_TRANSVERSE_ISOTROPIC)
      mod = (s.C_voigt[0] + s.C_voigt[7] + s.C_voigt[14]) / 3.0;
    else if (s.model == FEM_MOONEY_RIVLIN || s.model == FEM_FIBRE_MOONEY_RIVLIN)
      mod = (s.D1 > 0 ? 2.0 / s.D1 : 0.0) + 8.0 * (s.C10 + s.C01) / 3.0;
    else
      mod = s.E * (1.0 - s.nu) / ((1.0 + s.nu) * (1.0 - 2.0 * s.nu));
    c->elem_modulus[e] = std::max(mod, 1e-30) * sc[e];
  }
  c->mpnn_feat_valid = false;
  CK(cudaMemcpyAsync(c->matD, md.data(), md.size() * sizeof(DevMat<double>), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->matF, mf.data(), mf.size() * sizeof(DevMat<float>), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->mat_id, ids.data(), ids.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->scale, sc.data(), sc.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->model_kind = kind;
  c->has_j2 = has_j2;
  c->materials_set = true;
  c->tangent_valid = false;
  invalidate_coarse(c);
  return FEM_OK;
}

int fem_set_bc(void* ctx, const uint8_t* fixed_mask, const double* fixed_values, const double* f_ext) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (fixed_mask) {
    ++c->n_launches; launch_gather_mask(fixed_mask, c->fixed, c->d_perm_node, c->Nn, c->stream);
    CKL();
    // the matvec kernels read the fixed bits from the w lane of the FP32 coordinates
    ++c->n_launches; launch_x32_mask(c->X32, c->fixed, c->Nn, c->stream);
    CKL();
    // a changed constraint pattern changes the coarse operator (K_ff)
    std::vector<uint8_t> now(c->Nn);
    CK(cudaMemcpyAsync(now.data(), c->fixed, c->Nn, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (now != c->fixed_host) {
      c->fixed_host.swap(now);
      invalidate_coarse(c);
    }
  }
  if (fixed_values) {
    ++c->n_launches; launch_gather_d(fixed_values, c->fixed_vals, c->d_perm_node, c->Nn, c->stream);
    CKL();
    CK(cudaMemcpyAsync(c->fixed_vals_full, c->fixed_vals, sizeof(double) * c->ndof, cudaMemcpyDeviceToDevice,
                       c->stream));
  }
  if (f_ext) {
    ++c->n_launches; launch_gather_d(f_ext, c->fext, c->d_perm_node, c->Nn, c->stream);
    CKL();
    CK(cudaMemcpyAsync(c->fext_full, c->fext, sizeof(double) * c->ndof, cudaMemcpyDeviceToDevice, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  c->tangent_valid = false;
  return FEM_OK;
}

int fem_set_load_scale(void* ctx, double s) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!std::isfinite(s)) return set_err(c, FEM_ERR_INVALID, "load scale must be finite");
  ++c->n_launches; launch_scale_d(c->fixed_vals_full, s, c->fixed_vals, c->ndof, c->stream);
  ++c->n_launches; launch_scale_d(c->fext_full, s, c->fext, c->ndof, c->stream);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  c->tangent_valid = false;
  return FEM_OK;
}

int fem_batch_solve(void** ctxs, int32_t n, const FemSolveParams* prm, int32_t load_steps,
                    FemSolveResult* results, int32_t* status, double* wall_ms, int32_t n_threads) {
  if (!ctxs || n <= 0 || !results || !status) return set_global_error(FEM_ERR_INVALID, "need contexts and outputs");
  if (load_steps <= 0) return set_global_error(FEM_ERR_INVALID, "load_steps must be > 0");
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i]) return set_global_error(FEM_ERR_INVALID, "context %d is null", i);
    for (int j = 0; j < i; ++j)
      if (ctxs[j] == ctxs[i]) return set_global_error(FEM_ERR_INVALID, "context %d repeats context %d", i, j);
  }
  FemSolveParams p;
  if (prm)
    p = *prm;
  else
    fem_default_solve_params(&p);
  p.progress = nullptr;  // callbacks are not re-entrant across workers
  const int workers = std::max(1, std::min<int>(n, n_threads > 0 ? n_threads : n));
  // contexts leave batch mode on every return path
  struct BatchMode {
    void** ctxs;
    int n;
    ~BatchMode() {
      for (int i = 0; i < n; ++i) static_cast<FemCtx*>(ctxs[i])->in_batch = false;
    }
  } batch_mode{ctxs, n};
  // One thread first brings every instance to a solvable state: tangent at the
  // current displacement, matvec variant, coarse operator and the captured CG
  // graph.  Graph capture then never runs while other workers issue work.
  for (int i = 0; i < n; ++i) {
    FemCtx* c = static_cast<FemCtx*>(ctxs[i]);
    int st;
    if ((st = check_ctx(c))) return st;
    if (!c->materials_set) return set_err(c, FEM_ERR_STATE, "materials not set");
    if (!c->tangent_valid && (st = eval_residual(c, nullptr, nullptr))) return st;
    const bool tl = p.precond == FEM_PRECOND_TWO_LEVEL;
    const bool learned = p.precond == FEM_PRECOND_LEARNED;
    if (learned && !c->mpnn_has_weights) return set_err(c, FEM_ERR_STATE, "learned preconditioner has no weights");
    if ((st = compute_dinv(c, (tl || learned) ? FEM_PRECOND_JACOBI : p.precond, tl && c->block_jacobi))) return st;
    if ((tl || (learned && c->learned_coarse)) && (st = ensure_coarse(c))) return st;
    if (learned && (st = ensure_mpnn(c))) return st;
    c->in_batch = workers > 1;
    if ((st = ensure_cg_graph(c, learned ? GRAPH_LEARNED : (tl ? GRAPH_TWO_LEVEL : GRAPH_JACOBI)))) return st;
  }
  std::atomic<int> next{0};
  auto work = [&]() {
    cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
    cudaThreadExchangeStreamCaptureMode(&mode);
    for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1)) {
      FemCtx* c = static_cast<FemCtx*>(ctxs[i]);
      const auto t0 = std::chrono::steady_clock::now();
      FemSolveResult agg;
      std::memset(&agg, 0, sizeof(agg));
      agg.converged = 1;
      int st = FEM_OK;
      for (int k = 1; k <= load_steps && (st == FEM_OK || st == FEM_NOT_CONVERGED); ++k) {
        st = fem_set_load_scale(c, (double)k / load_steps);
        if (st) break;
        FemSolveResult r;
        std::memset(&r, 0, sizeof(r));
        st = fem_newton_solve(c, &p, &r);
        agg.iterations += r.iterations;
        agg.cg_iterations += r.cg_iterations;
        agg.residual_evals += r.residual_evals;
        agg.residual = r.residual;
        agg.relative_residual = std::max(agg.relative_residual, r.relative_residual);
        if (k == 1) agg.first_residual = r.first_residual;
        if (!r.converged) agg.converged = 0;
      }
      results[i] = agg;
      status[i] = st;
      if (wall_ms)
        wall_ms[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    cudaThreadExchangeStreamCaptureMode(&mode);
  };
  std::vector<std::thread> pool;
  for (int w = 1; w < workers; ++w) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  for (int i = 0; i < n; ++i)
    if (status[i] != FEM_OK && status[i] != FEM_NOT_CONVERGED) return status[i];
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

int fem_nodal_mises(void* ctx, const double* u, double* mises_out, int32_t average) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  if (!mises_out) return set_err(c, FEM_ERR_INVALID, "mises_out is null");
  if (average != 0 && average != 1) return set_err(c, FEM_ERR_INVALID, "average must be 0 or 1");
  if (!c->materials_set) return set_err(c, FEM_ERR_STATE, "materials not set");
  if (u) {
    ++c->n_launches; launch_gather_d(u, c->u, c->d_perm_node, c->Nn, c->stream);
    CKL();
  }
  double* sig = nullptr;
  CK(cudaMallocAsync(reinterpret_cast<void**>(&sig), sizeof(double) * 9 * c->Nq, c->stream));
  ++c->n_launches; launch_stress(c->mesh(), c->matD, c->model_kind, c->u, c->ep_c, c->epe_c, c->d_perm_elem,
                                 nullptr, sig, c->stream);
  ++c->n_launches; launch_nodal_mises(c->mesh(), c->d_perm_elem, c->d_perm_node, sig, average, mises_out,
                                      c->stream);
  const cudaError_t e = cudaGetLastError();
  cudaFreeAsync(sig, c->stream);
  if (e != cudaSuccess) return set_err(c, FEM_ERR_CUDA, "nodal Mises kernels failed: %s", cudaGetErrorString(e));
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
  MvArgs mv = make_mv(c);
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
  if (precond < FEM_PRECOND_NONE || precond > FEM_PRECOND_LEARNED)
    return set_err(c, FEM_ERR_INVALID, "unknown preconditioner %d", precond);
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
  if (prm.precond < FEM_PRECOND_NONE || prm.precond > FEM_PRECOND_LEARNED)
    return set_err(c, FEM_ERR_INVALID, "unknown preconditioner %d", prm.precond);
  FemSolveResult out;
  std::memset(&out, 0, sizeof(out));
  // Load-step extrapolation (FEM_OPT_EXTRAPOLATE): when the last solve
  // converged and u is still its end state, Newton starts from u_last +
  // du_last (the last step's change repeated) instead of carrying the
  // prescribed-value change by a first linear solve.  Relative convergence
  // is still measured against the residual of the state the reference
  // evaluates first (below), so the stopping test and the converged
  // equilibrium are the same.
  bool extrap_now = false;
  if (c->extrap) {
    const size_t nd = (size_t)c->ndof_pad;
    if (!c->u_last) {
      if ((st = dalloc(c, &c->u_last, nd)) || (st = dalloc(c, &c->du_last, nd)) || (st = dalloc(c, &c->u_start, nd)))
        return st;
      c->extrap_ready = false;
    }
    if (c->extrap_ready) {
      unsigned int* differ = reinterpret_cast<unsigned int*>(c->scalars + 6);
      CK(cudaMemsetAsync(differ, 0, sizeof(unsigned int), c->stream));
      ++c->n_launches; launch_differ(c->u, c->u_last, c->ndof, differ, c->stream);
      CKL();
      unsigned int h_differ = 1u;
      CK(cudaMemcpyAsync(c->h_scalars + 6, differ, sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      std::memcpy(&h_differ, c->h_scalars + 6, sizeof(unsigned int));
      extrap_now = h_differ == 0u;
    }
    CK(cudaMemcpyAsync(c->u_start, c->u, nd * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    c->extrap_ready = false;
  }
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
    out.residual_evals = 1;
  }
  if (extrap_now) {
    if (!has_dc) {
      // the reference's first residual: the previous u under the new loads
      if ((st = eval_residual(c, nullptr, &r2))) return st;
      ref_norm = std::sqrt(r2);
      out.residual_evals = 1;
    }
    ++c->n_launches; launch_extrap(c->u, c->u_last, c->du_last, c->ndof, c->stream);
    CKL();
  } else if (has_dc) {
    if ((st = eval_residual(c, nullptr, &r2))) return st;
    out.residual_evals = 2;
    if (!std::isfinite(ref_norm) || !std::isfinite(r2)) {
      if (res) *res = out;
      return set_err(c, FEM_ERR_NAN, "NaN/Inf residual at iteration 0");
    }
    MvArgs mv = make_mv(c);
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
    ++c->n_launches; launch_u_update(c->u, c->u_base, c->x, 1.0, c->Nn, c->stream);
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
      ++c->n_launches; launch_u_update(c->u, c->u_base, c->x, alpha, c->Nn, c->stream);
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
    CK(cudaMemcpyAsync(c->ep_c, c->ep_t, 6 * c->Nq * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->epe_c, c->epe_t, c->Nq * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  if (c->extrap && converged && (!c->has_j2 || prm.auto_commit)) {
    ++c->n_launches; launch_extrap_record(c->u, c->u_start, c->u_last, c->du_last, c->ndof, c->stream);
    CKL();
    c->extrap_ready = true;
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
  EventPair ev;
  CK(ev.create());
  cudaEvent_t e0 = ev.a, e1 = ev.b;
  const int nn = c->Nn;
  const CGState hs = endless_cg();
  // a nonzero direction: p = 1 on free DOFs
  launch_dinv_identity(c->p, c->fixed, c->Nn, c->stream);
  auto reset_cg = [&]() { return cudaMemcpyAsync(c->cg, &hs, sizeof(hs), cudaMemcpyHostToDevice, c->stream); };
  MvArgs mv = make_mv(c);
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
  ra.stage_d = (c->npe == 8 || c->res_two_phase) ? c->stage_d : nullptr;
  for (int k = 0; k < 4; ++k) {
    CK(reset_cg());
    for (int w = 0; w < 2; ++w) {
      if (k == 0) launch_matvec(mv, c->model_kind, c->stream);
      if (k == 1) launch_residual(ra, c->model_kind, c->stream);
      if (k == 2) launch_cg_update(c->tmpf, c->r, c->p, c->y, c->dinv, nn, c->cg, c->red(), SITE_CGU, c->stream);
      if (k == 3) launch_cg_pupdate(c->tmpf, c->r, c->dinv, nn, c->cg, c->stream);
    }
    CK(reset_cg());
    CK(cudaEventRecord(e0, c->stream));
    for (int r = 0; r < reps; ++r) {
      if (k == 0) launch_matvec(mv, c->model_kind, c->stream);
      if (k == 1) launch_residual(ra, c->model_kind, c->stream);
      if (k == 2) launch_cg_update(c->tmpf, c->r, c->p, c->y, c->dinv, nn, c->cg, c->red(), SITE_CGU, c->stream);
      if (k == 3) launch_cg_pupdate(c->tmpf, c->r, c->dinv, nn, c->cg, c->stream);
    }
    CK(cudaEventRecord(e1, c->stream));
    CKL();
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    ms_out[k] = ms / reps;
  }
  c->tangent_valid = true;
  return FEM_OK;
}

int fem_commit_history(void* ctx) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  CK(cudaMemcpyAsync(c->ep_c, c->ep_t, 6 * c->Nq * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->epe_c, c->epe_t, c->Nq * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

int fem_reset_history(void* ctx) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  CK(cudaMemsetAsync(c->ep_c, 0, 6 * c->Nq * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->epe_c, 0, c->Nq * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->ep_t, 0, 6 * c->Nq * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->epe_t, 0, c->Nq * sizeof(double), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->tangent_valid = false;
  c->extrap_ready = false;
  // back to rest: the coarse operator was built on a deformed, plastic
  // tangent; the next two-level solve assembles a fresh one
  invalidate_coarse(c);
  return FEM_OK;
}

int fem_get_history(void* ctx, double* ep_out, double* epe_out) {
  FemCtx* c = static_cast<FemCtx*>(ctx);
  int st;
  if ((st = check_ctx(c))) return st;
  std::vector<double> ep(6 * c->Nq), epe(c->Nq);
  CK(cudaMemcpyAsync(ep.data(), c->ep_c, ep.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(epe.data(), c->epe_c, epe.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // internal SoA (xx,yy,zz,yz,xz,xy) -> caller (Ne,3,3) / (Ne)
  // HEX8: caller point e * 8 + g (the reference's gp_idx), internal g * Ne + e
  std::vector<double> full(9 * c->Nq), e1(c->Nq);
  for (int e = 0; e < c->Ne; ++e) {
    const int eu = c->perm_elem[e];
    for (int g = 0; g < c->ngp; ++g) {
      const size_t q = (size_t)g * c->Ne + e, qu = (size_t)eu * c->ngp + g;
      double s[6];
      for (int k = 0; k < 6; ++k) s[k] = ep[(size_t)k * c->Nq + q];
      double* F = &full[9 * qu];
      F[0] = s[0]; F[4] = s[1]; F[8] = s[2];
      F[5] = F[7] = s[3];
      F[2] = F[6] = s[4];
      F[1] = F[3] = s[5];
      e1[qu] = epe[q];
    }
  }
  if (ep_out) CK(cudaMemcpyAsync(ep_out, full.data(), full.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (epe_out) CK(cudaMemcpyAsync(epe_out, e1.data(), e1.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return FEM_OK;
}

}  // extern "C"
