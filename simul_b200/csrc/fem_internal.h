// Internal structures shared by the host driver (fem_ctx.cu) and the kernels
// (fem_kernels.cu).  Not part of the public ABI.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

#include "fem_device.cuh"

namespace femb200 {

// Programmatic dependent launch for the kernels of the PCG iteration chain:
// a kernel launched with it may be scheduled as its predecessor's CTAs
// retire, and waits (griddepcontrol.wait) for the predecessor's results
// before it touches memory.  For a kernel launched without it the wait does
// nothing.
__device__ __forceinline__ void chain_enter() {
#if defined(__CUDA_ARCH__)
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

// Lets the next chain kernel be scheduled: called once a kernel's memory
// traffic is issued and only its block reduction is left.
__device__ __forceinline__ void chain_release() {
#if defined(__CUDA_ARCH__)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// Whether launches from this host thread use programmatic dependent launch
// (set around graph capture of the CG iteration chain).
inline bool& chain_pdl() {
  static thread_local bool on = false;
  return on;
}

// Launches a chain kernel (one that starts with chain_enter()), with
// programmatic dependent launch when chain_pdl() is set.
template <typename... KArgs, typename... Args>
inline void launch_chain(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                         Args... args) {
  if (!chain_pdl()) {
    k<<<grid, block, smem, s>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

// Node-block gather tables (device).  Internal node n belongs to block
// n / nb.  Block b lists every element touching one of its nodes: its "home"
// elements (contiguous internal ids, listed first) then the foreign ones.
// node_slots[node_row[n] .. node_row[n+1]) holds (local element index << 2 |
// local slot) sorted by local index: the fixed summation order of node n.
struct MeshDev {
  int n_nodes;
  int n_elems;
  int n_blocks;
  int nb;
  const double* X64;        // [3 Nn]
  const float4* X32;        // [Nn]
  const int4* conn;         // [Ne]
  const uint8_t* mat_id;    // [Ne]
  const float* scale;       // [Ne]
  const int* blk_ptr;       // [n_blocks + 1] into blk_elems
  const int* blk_home;      // [n_blocks] home element count
  const int* blk_elems;     // element ids
  const int* node_row;      // [Nn + 1]
  const uint32_t* node_slots;
  const uint8_t* fixed;     // [Nn] bit d set = DOF d fixed
  int max_slots;            // largest slot-list range of one block (shared memory sizing)
  const int4* spos;         // [Ne] position of each (element, slot) in node_slots order
                            // (HEX8: [2 Ne], slots 0-3 then 4-7 of each element)
  int npe;                  // nodes per element: 4 (TET4) or 8 (HEX8; conn holds 2 int4 per element)
  int slot_shift;           // node_slots entries are local element << slot_shift | slot
};

// HEX8 elements carry 8 Gauss points; per-point arrays (tangent payload, J2
// history) are SoA over points q = g * Ne + e: word k of point q at k * Nq + q.
constexpr int kHexGauss = 8;

// Last-block reduction bookkeeping: one slot per reduction site.
struct Reduce {
  double* partials;         // [n_sites][max_blocks]
  unsigned int* counters;   // [n_sites]
  int max_blocks;
};

// FP32 node vectors (CG r, x, p, y, diag^-1, scratch) hold one float4 per
// node (xyz, 0); FP64 node vectors (u, R, f_ext, prescribed values) 3 doubles.

// Device-resident PCG state (read by every CG kernel, advanced by the last
// block of each reduction so no host round trip is needed per iteration).
struct CGState {
  double rz, pAp, rr, rr0, tol2, alpha, beta, pad;
  int iter, max_iter, done, status;  // done: 0 running, 1 converged, 2 max iters, 3 breakdown,
                                     // 4 learned FPCG handed over (network switched off)
  int zsel;                          // learned FPCG: 1 = this step used the Jacobi (+ coarse) direction
  int n_alt;                         // learned FPCG: steps that used it
  int locked;                        // learned FPCG: network switched off for the rest of the solve
  int trips;                         // whole-solve graph: trips through the loop body
};

struct ResArgs {
  MeshDev m;
  const DevMat<double>* matD;
  const double* u;          // [3 Nn] internal order
  const double* f_ext;      // [3 Nn]
  double* R;                // [3 Nn] residual f_ext + f, fixed DOFs zeroed
  double* fneg;             // [3 Nn] optional: negative internal force
  float* payload;           // [kPay][Ne] SoA
  const double* ep_c;       // [6][Ne] committed plastic strain
  const double* epe_c;      // [Ne]
  double* ep_t;             // trial history out
  double* epe_t;
  double* rnorm2;           // [1] ||R||^2 (free DOFs)
  Reduce red;
  int red_site;
  double* stage_d;          // HEX8: [3 * 8 Ne] element slot forces in node_slots order
};

// Element-block matvec tables (MV_ELEM_BLOCK, TET4).  Element block k holds
// elements [k eb, (k + 1) eb) of the internal order; its local nodes are the
// distinct vertices of those elements in ascending order.  A local node all
// of whose elements lie in the block ("interior") gets its product row from
// that block alone; a node shared by several blocks gets one partial row per
// block, stored in block order, and a second, small kernel adds them.
struct EbDev {
  int eb;                   // elements per block (= threads per CTA: one element per thread)
  int n_blk;
  int lmax;                 // most local nodes of one block (shared-memory sizing)
  const int* node_ptr;      // [n_blk + 1] into nodes / ninfo; lrow of block b starts at node_ptr[b] + b
  const int* nodes;         // local node -> internal node
  // local node -> (internal node, partial slot or -1 if interior, the node's
  // first partial, its number of partials)
  const int4* ninfo;
  const uint16_t* lrow;     // [node_ptr[n_blk] + n_blk] local slot range of each local node (L_b + 1 per block)
  const uint2* lconn;       // [Ne] four 16-bit local vertex indices
  const uint2* lspos;       // [Ne] four 16-bit positions of the element's slot vectors in node-major order
  float4* parts;            // per-block partial rows of shared nodes, each node's in block order
  const int4* snode;        // [n_shared] shared nodes: (node, first partial, number of partials, 0)
  int n_shared;
  double* pap_part;         // [n_blk] CG: each block's share of p.Ap
};

// Warp-aggregated two-phase matvec tables (MV_WARP_AGG, TET4).  Warp w
// evaluates elements [32 w, 32 w + 32); the slot vectors of each distinct
// vertex of those elements are added in shared memory (fixed order) into one
// partial row per (warp, vertex), stored node-major with each node's partials
// in warp order, and the two-phase node gather adds a node's partials.
struct WaggDev {
  const uint32_t* lspos;    // [Ne] four 8-bit positions of the element's slot vectors in its warp's
                            // node-major slot order
  const int* wptr;          // [n_warps + 1] into went
  const int2* went;         // per (warp, local node): partial position, slot range start | end << 16
  const int* wnode;         // per (warp, local node): the node
  const uint32_t* lrow;     // [Ne] four 8-bit indices of the element's vertices among its warp's rows
  const int* prow;          // [Nn + 1] each node's partial range
  float4* parts;            // [prow[Nn]] partial rows
};

struct MvArgs {
  MeshDev m;
  const DevMat<float>* matF;
  const float* payload;
  const float* x;           // [Nn] float4 (xyz, 0)
  float* y;
  CGState* cg;              // non-null: CG-fused (early exit, p.Ap, alpha)
  Reduce red;
  int red_site;
  int mask_input;           // 1: fixed DOFs of x read as zero (K_ff x); 0: K_f,all x
  int variant;              // MV_FUSED (node-block), MV_TWO_PHASE (element pass + node gather),
                            // MV_ELEM_BLOCK or MV_WARP_AGG
  float4* stage;            // [4 Ne] slot vectors in node_slots order (two-phase scratch)
  // two-phase inside CG, non-null: x holds the preconditioned residual z and
  // the node gather forms the direction by recurrence, p = z + beta p and
  // q = K z + beta q (q in y, p here), so no separate direction update runs
  float* p_rec;
  EbDev eb;                 // element-block tables (MV_ELEM_BLOCK)
  WaggDev wa;               // warp-aggregation tables (MV_WARP_AGG)
};

// MV_ELEM_BLOCK: one CTA per element block: vertex data staged in shared
// memory, slot vectors summed per local node in shared memory; a second
// kernel adds the partial rows of nodes shared by blocks (fem_elemblock.cu).
// MV_WARP_AGG: the two-phase element pass with each warp's distinct
// vertices loaded once into shared memory and its slot vectors added per
// vertex there, so the node gather reads about a quarter of the partial rows
// (fem_kernels.cu).
// MV_PERSIST: the two-phase pair as persistent grid-stride kernels (one wave
// of CTAs, the next element's streaming inputs prefetched).
enum { MV_FUSED = 0, MV_TWO_PHASE = 1, MV_ELEM_BLOCK = 2, MV_WARP_AGG = 3, MV_PERSIST = 4, MV_N_VARIANTS = 5 };

// smallest element block of the element-block matvec (one element per
// thread; blocks of 256, 512, 768 or 1024 elements)
constexpr int kEbThreads = 256;
// shared memory of one element-block CTA
inline size_t eb_smem_bytes(int eb, int lmax) {
  return 16 * (size_t)(4 * eb) + 32 * (size_t)lmax + ((2 * (size_t)(lmax + 1) + 15) & ~(size_t)15);
}

struct DiagArgs {
  MeshDev m;
  const DevMat<float>* matF;
  const float* payload;
  float* dinv;              // [Nn] float4: 1/diag(K) on free DOFs, 0 elsewhere
  float* boff;              // non-null: nodal 3x3 block inverse, dinv its diagonal, boff (01, 02, 12)
  float4* stage;            // HEX8: [2 * 8 Ne] per slot the 6 block entries (or 3 diagonal entries)
};

// Coarse lattice of the two-level preconditioner (fem_coarse.cu).  Cells
// are the non-empty lattice cells (ascending lattice index); coarse nodes are
// their corners (ascending lattice index); corner q of a cell is the lattice
// offset (q >> 2 & 1, q >> 1 & 1, q & 1).
struct CoarseDev {
  int n_cells;
  int n_cn;                 // coarse nodes
  int n_dof;                // 3 n_cn
  float inv_H;              // 1 / cell edge
  float3 lo;                // lattice origin
  const int3* cell_ijk;     // [n_cells] lattice coordinates
  const int* cell_corner;   // [n_cells * 8] coarse node of each corner
  const int* cell_node_ptr; // [n_cells + 1] into cell_nodes (each node in one cell)
  const int* cell_nodes;
  const int* cell_elem_ptr; // [n_cells + 1] into cell_elems (cell of the centroid)
  const int* cell_elems;
  const int* node_cell;     // [Nn]
  const float4* node_lat;   // [Nn] local coordinates in the node's cell (xyz), the cell (w, int bits)
  const uint4* node_corners;  // [Nn] the cell's 8 corner coarse nodes, 16 bits each (n_cn <= 65535)
  const int* cn_cells;      // [n_cn * 8] cell * 8 + corner, ascending cell, -1 padded
  double* blocks;           // [n_cells][cell_slices][24 * 24] Galerkin block shares of each cell
  int cell_slices;          // block shares per cell (coarse_cell_slices)
  double* Ac;               // [n_dof * n_dof] column-major; factorised / inverted in place
  const float* Ac32;        // non-null: the inverse's lower triangle is here in FP32 instead (FP32 inversion)
  float* Ainv;              // [n_dof * n_dof] FP32 inverse (symmetric), or null
  // BF16 inverse, or null: the lower block triangle of 64 x 64 tiles, tile
  // (I, J), I >= J, at index I (I + 1) / 2 + J, row-major inside the tile,
  // zero beyond n_dof (a diagonal tile holds both of its triangles)
  __nv_bfloat16* Ainv16;
  int nb16;                 // tiles per side: ceil(n_dof / 64)
  float* yslots;            // BF16 path: [nb16][nb16][64] slot (R, K) = Ainv_RK r_c,K
  float* cell_r;            // [n_cells][r_slices][24] restricted residual shares per cell
  int r_slices;             // warps (node slices) per cell in the restriction
  float* rc;                // [64 nb16] coarse residual P^T r (zero beyond n_dof)
  float* yc;                // [64 nb16] coarse correction
};

struct CoarseArgs {
  MeshDev m;
  CoarseDev c;
  const DevMat<float>* matF;
  const float* payload;
  const float* boff;        // non-null: the smoother is the nodal 3x3 block inverse (dinv + these)
};

// Fused CG step (fem_step.cu): the work of one PCG iteration after the
// tangent matvec, as one cooperative kernel whose phases are separated by
// grid-wide barriers.  Two-level: x, r update + ||r||^2 + restriction |
// coarse residual + convergence test | coarse product | z = D^-1 r + P y_c and
// r.z | p = z + beta p.  Jacobi: x, r update + ||r||^2 + r.D^-1 r |
// p = D^-1 r + beta p.
constexpr int kStepThreads = 512;

struct StepArgs {
  MeshDev m;
  CoarseDev c;
  float* x;
  float* r;
  float* p;
  const float* q;           // K p from the matvec
  const float* dinv;
  float* z;                 // two-level: preconditioned residual (scratch)
  CGState* cg;
  double* part;             // two-level: [n_cells * slices] ||r||^2 shares, then [n_chunks] r.z shares;
                            // Jacobi: [2][n_chunks]
  int n_chunks;             // ceil(n_nodes / kStepThreads)
  unsigned int* bar;        // [2] grid barrier: arrivals, generation
};

// CTAs of a cooperative step launch on this device (0: not available);
// kind 0 Jacobi, 1 two-level with an n_dof coarse space.
int step_grid(int kind, int n_dof);
// raises the step kernels' shared-memory limit (before a capture)
void prepare_step_kernels(int kind, int n_dof);
cudaError_t launch_tl_step(const StepArgs& a, cudaStream_t s);
cudaError_t launch_jacobi_step(const StepArgs& a, cudaStream_t s);

// Learned preconditioner (fem_mpnn.cu).  Flat FP32 parameter order:
// W_e [64][16], b_e [64], then per layer W_l [64][128], b_l [64], then
// W_d [3][64], b_d [3].
constexpr int kMpnnHidden = 64;
constexpr int kMpnnIn = 16;
constexpr int kMpnnLayers = 4;
constexpr int kMpnnOffWe = 0;
constexpr int kMpnnOffBe = kMpnnHidden * kMpnnIn;
__host__ __device__ constexpr int kMpnnOffW(int l) {
  return kMpnnOffBe + kMpnnHidden + l * (kMpnnHidden * 2 * kMpnnHidden + kMpnnHidden);
}
__host__ __device__ constexpr int kMpnnOffB(int l) { return kMpnnOffW(l) + kMpnnHidden * 2 * kMpnnHidden; }
constexpr int kMpnnOffWd = kMpnnOffW(kMpnnLayers);
constexpr int kMpnnOffBd = kMpnnOffWd + 3 * kMpnnHidden;
constexpr int kMpnnParams = kMpnnOffBd + 3;

struct MpnnDev {
  int n_nodes;
  const int* adj_ptr;           // [Nn + 1] node graph (nodes sharing an element), ids ascending
  const int* adj_idx;
  const float* deg_inv;         // [Nn] 1 / |N(i)| (0 for isolated nodes)
  const float* cfeat;           // [Nn] log-modulus feature
  const uint8_t* fixed;         // [Nn]
  const float* w;               // [kMpnnParams] FP32 master parameters
  const __nv_bfloat16* We_p;    // packed W_e  [64 x 16]  (K-major canonical)
  const __nv_bfloat16* Wl_p;    // packed W_l  [layers][64 x 128]
  const __nv_bfloat16* WlT_p;   // packed W_l^T [layers][128 x 64]
  __nv_bfloat16* H[kMpnnLayers + 1];  // [Nn][64] hidden states per layer
  uint64_t* mask[kMpnnLayers];  // [Nn] relu masks of the message-passing layers
  double* scal;                 // [0] s = RMS |D^-1/2 r|
  int* err;                     // set when an MMA completion wait gives up
};

// Training buffers of the learned preconditioner's backward pass.
struct MpnnTrain {
  MpnnDev m;
  float* GH;                    // [Nn][64] gradient w.r.t. the current layer output
  float* GHn;                   // [Nn][64] self-path part of the gradient w.r.t. its input
  float* Q;                     // [Nn][64] aggregation-path gradient / deg
  float* gpart;                 // [tiles][kMpnnParams] per-tile gradient shares
};

// Raises a kernel's dynamic shared-memory limit to the device's opt-in maximum
// (minus the kernel's static shared memory), once per (device, kernel).  The
// limit is process-wide state: setting it to what one mesh needs would fail
// the launches of a larger mesh, or of another thread, so it is only ever
// raised to the maximum (fem_smem.cu).
void raise_smem_limit(const void* kernel);
template <typename K>
inline void raise_smem_limit_k(K kernel) {
  raise_smem_limit(reinterpret_cast<const void*>(kernel));
}

// Dense SPD inverse (fem_dense.cu): the lower triangle of Ac^-1 (Ac: n x n
// FP64 column-major, lower triangle read) into out (n x n column-major).  A
// and W are work matrices of N x N, N = n rounded up to dense_tile(fp64);
// *info receives the first non-positive pivot (1-based), 0 if none.
// sched holds the streams and events of its multi-stream schedule; a caller
// that inverts repeatedly keeps one (null: created and released per call).
// row_first (host, n entries, or null for dense): the lowest column of each
// row of Ac's lower triangle that may be nonzero; tiles outside that
// envelope are skipped (bitwise the same result).
struct DenseSched {
  cudaStream_t side = nullptr, rest = nullptr, crit = nullptr;
  std::vector<cudaEvent_t> ev, evr;  // nt + 1 and nt events
  cudaError_t ensure(int nt);
  void release();
};
int dense_tile(bool fp64);
cudaError_t dense_spd_inverse_f32(const double* Ac, int n, float* A, float* W, int* info, float* out,
                                  cudaStream_t s, int* launches, DenseSched* sched,
                                  const int* row_first);
// FP32 Cholesky, then W = L^-1 and W^T W on TF32 tensor-core tiles (tcgen05);
// *info = -1 if a tensor-core completion wait timed out
cudaError_t dense_spd_inverse_tf32(const double* Ac, int n, float* A, float* W, int* info, float* out,
                                   cudaStream_t s, int* launches, DenseSched* sched,
                                  const int* row_first);
cudaError_t dense_spd_inverse_f64(const double* Ac, int n, double* A, double* W, int* info, double* out,
                                  cudaStream_t s, int* launches, DenseSched* sched,
                                  const int* row_first);

// Records a failure for fem_last_error(NULL) (thread-local, fem_ctx.cu) and
// returns `code`.
int set_global_error(int code, const char* fmt, ...);

// launchers (fem_kernels.cu)
void launch_residual(const ResArgs& a, int model, cudaStream_t s);
void launch_matvec(const MvArgs& a, int model, cudaStream_t s);
// sets the shared-memory limits the captured CG graph's kernels need
void prepare_kernels(const MeshDev& m, int model);
void launch_diag(const DiagArgs& a, int model, cudaStream_t s);
// coarse lattice (fem_coarse.cu)
size_t coarse_cell_smem();
// Galerkin block slots per lattice cell (TET4: one per CTA; HEX8: one per warp)
int coarse_cell_slices(int npe);
int coarse_restrict_slices(int n_cells);  // node slices (restriction warps) per lattice cell
// x += alpha p, r -= alpha q and the restriction of the new r into cell_r
// (one kernel; ||r||^2 and the convergence test follow in tl_rz)
void launch_update_restrict(const CoarseArgs& a, float* x, float* r, const float* p, const float* q, CGState* cg,
                            cudaStream_t s);
// r_c from cell_r, then y_c = Ainv r_c
void launch_coarse_solve(const CoarseArgs& a, const CGState* cg, cudaStream_t s);
void prepare_coarse_kernels(int model, int n_dof);
// cell Galerkin blocks + dense Ac (FP64, column-major)
void launch_coarse_assemble(const CoarseArgs& a, int model, cudaStream_t s);
// HEX8 cells' Galerkin block shares (fem_hex8.cu); launch_coarse_assemble calls it
void launch_coarse_cells_hex(const CoarseArgs& a, int model, cudaStream_t s);
// Ainv = FP32 symmetric copy of the lower triangle left in Ac
// fills node_lat from X32, node_cell and cell_ijk
void launch_coarse_node_lat(const MeshDev& m, const CoarseDev& c, float4* out, cudaStream_t s);
// fills node_corners from node_cell and cell_corner
void launch_coarse_node_corners(const MeshDev& m, const CoarseDev& c, uint4* out, cudaStream_t s);
// kernels one coarse product launches (1 FP32, 2 packed BF16)
int coarse_product_kernels(const CoarseDev& c);
void launch_coarse_symmetrize(const CoarseDev& c, cudaStream_t s);
// yc = Ainv P^T r (skipped once cg->done is set, when cg is non-null)
void launch_coarse_apply(const CoarseArgs& a, const float* r, const CGState* cg, cudaStream_t s);
// z = D^-1 r + P yc, rz and beta (init: into p, beta = 0)
void launch_tl_rz(const CoarseArgs& a, bool init, const float* r, const float* dinv, float* z, float* p,
                  CGState* cg, Reduce red, int site, cudaStream_t s);
void launch_tl_pupdate(float* p, const float* z, int n_nodes, const CGState* cg, cudaStream_t s);
// learned flexible PCG: [z += P yc], safeguard against the Jacobi (+ coarse)
// direction zalt, rz and Polak-Ribiere beta (two reduction sites)
void launch_fpcg_dots(const CoarseArgs& a, bool init, bool coarse, const float* r, const float* q,
                      const float* dinv, float* z, float* zalt, float* p, CGState* cg, Reduce red, int site,
                      int site2, cudaStream_t s);
void launch_fpcg_pupdate(float* p, const float* z, const float* zalt, int n_nodes, const CGState* cg, bool init,
                         cudaStream_t s);

// learned preconditioner (fem_mpnn.cu)
void prepare_mpnn_kernels();
void launch_mpnn_pack(const float* w, __nv_bfloat16* We_p, __nv_bfloat16* Wl_p, __nv_bfloat16* WlT_p,
                      cudaStream_t s);
// z = M(r) (skipped once cg->done is set, when cg is non-null)
void launch_mpnn_forward(const MpnnDev& m, const float* r, const float* dinv, float* z, const CGState* cg,
                         Reduce red, int site, cudaStream_t s);

// grad (+)= d<gz, M(r)>/dw after a forward pass on the same r (activations kept)
void launch_mpnn_backward(const MpnnTrain& t, const float* r, const float* dinv, const float* gz, float* grad,
                          int accumulate, cudaStream_t s);
void launch_mpnn_adam(float* w, float* mom, float* var, const float* grad, float gscale, float lr, int step,
                      cudaStream_t s);

// training helpers (fem_coarse.cu)
void launch_coarse_add(const CoarseArgs& a, float* z, cudaStream_t s);
// out[0] += energy loss of (z, r, e) with q = A z; out[1] = 2 / e.r
void launch_train_loss(const float* z, const float* q, const float* r, const float* e, int n, double* out,
                       Reduce red, int site, cudaStream_t s);
void launch_train_grad_z(const float* q, const float* r, const uint8_t* fixed, const double* scale, float* gz,
                         int n, cudaStream_t s);
void launch_jacobi_apply(const float* r, const float* dinv, float* z, int n, cudaStream_t s);

// whole-solve CG graph: clears the WHILE condition once cg->done is set, or
// after cg->max_iter / iters_per_trip + 2 trips (then cg->done = 2)
void launch_cg_loop_cond(cudaGraphConditionalHandle h, CGState* cg, int iters_per_trip, cudaStream_t s);

// PCG vector kernels.  precond_in_update = 1: Jacobi z = D^-1 r is applied
// inside cg_init / cg_update (rz, beta there); 0: an external preconditioner
// kernel computes rz and beta.
void launch_cg_init(const double* b, float* r, float* x, float* p, const float* dinv, int n_nodes,
                    CGState* cg, double rtol, int maxit, Reduce red, int site, cudaStream_t s,
                    int precond_in_update = 1);
void launch_cg_update(float* x, float* r, const float* p, const float* y, const float* dinv,
                      int n_nodes, CGState* cg, Reduce red, int site, cudaStream_t s,
                      int precond_in_update = 1);
void launch_cg_pupdate(float* p, const float* r, const float* dinv, int n_nodes, CGState* cg,
                       cudaStream_t s);
void launch_stress(const MeshDev& m, const DevMat<double>* matD, int model, const double* u,
                   const double* ep_c, const double* epe_c, const int* perm_elem, double* F_out,
                   double* sig_out, cudaStream_t s);
// nodal von Mises from caller-order element stresses (sum, or average)
void launch_nodal_mises(const MeshDev& m, const int* perm_elem, const int* perm_node, const double* sig_user,
                        int average, double* out_user, cudaStream_t s);
void launch_refq(const MeshDev& m, const int* perm_elem, double* dNdX, double* vol,
                 cudaStream_t s);
// HEX8 (fem_hex8.cu): element pass writing slot vectors in node_slots order
// plus a fixed-order node gather, like the two-phase TET4 matvec
void launch_residual_hex(const ResArgs& a, int model, cudaStream_t s);
void launch_matvec_hex(const MvArgs& a, int model, cudaStream_t s);
void launch_diag_hex(const DiagArgs& a, int model, cudaStream_t s);
void launch_stress_hex(const MeshDev& m, const DevMat<double>* matD, int model, const double* u,
                       const double* ep_c, const double* epe_c, const int* perm_elem, double* F_out,
                       double* sig_out, cudaStream_t s);
void launch_refq_hex(const MeshDev& m, const int* perm_elem, double* dNdX, double* vol, cudaStream_t s);
// the node gather of the two-phase matvec (fem_kernels.cu)
void launch_node_gather(const MvArgs& a, cudaStream_t s);
// element-block matvec (fem_elemblock.cu); raise its shared-memory limit first
void launch_matvec_eb(const MvArgs& a, int model, cudaStream_t s);
void prepare_eb_kernels(int model);
// out[n*3+d] (internal) = in[perm[n]*3+d] (caller order) and back
void launch_gather_d(const double* in_user, double* out_int, const int* perm, int n, cudaStream_t s);
void launch_scatter_d(const double* in_int, double* out_user, const int* perm, int n,
                      cudaStream_t s);
void launch_gather_f(const float* in_user, float* out_int, const int* perm, int n, cudaStream_t s);
void launch_scatter_f(const float* in_int, float* out_user, const int* perm, int n, cudaStream_t s);
void launch_scatter_f2d(const float* in_int, double* out_user, const int* perm, int n,
                        cudaStream_t s);
void launch_gather_mask(const uint8_t* in_user, uint8_t* out_int, const int* perm, int n,
                        cudaStream_t s);
void launch_apply_bc(double* u, const double* fixed_vals, const uint8_t* fixed, int n,
                     cudaStream_t s);
// u[3n+d] = u_base[3n+d] + alpha du[4n+d] for n < n_nodes
// float4-per-node vector -> three doubles per node; x += x0 (float4 per node)
void launch_f4_to_d3(const float* in, double* out, int n_nodes, cudaStream_t s);
void launch_f4_add(float* x, const float* x0, int n_nodes, cudaStream_t s);
// load-step extrapolation (fem_newton_solve with FEM_OPT_EXTRAPOLATE)
void launch_extrap(double* u, const double* u_last, const double* du_last, int n, cudaStream_t s);
void launch_differ(const double* a, const double* b, int n, unsigned int* differ, cudaStream_t s);
void launch_extrap_record(const double* u, const double* u_start, double* u_last, double* du_last, int n,
                          cudaStream_t s);
void launch_u_update(double* u, const double* u_base, const float* du, double alpha, int n_nodes,
                     cudaStream_t s);
// out[i] = s in[i], i < n
void launch_scale_d(const double* in, double s, double* out, int n, cudaStream_t st);
// X32[n].w = fixed bits of node n
void launch_x32_mask(float4* X32, const uint8_t* fixed, int n, cudaStream_t s);
void launch_gather_d_masked(const double* in_user, double* out_int, const int* perm,
                            const uint8_t* fixed, int n, cudaStream_t s);
void launch_dinv_identity(float* dinv, const uint8_t* fixed, int n, cudaStream_t s);
// dc = (fixed_vals - u) on fixed DOFs (FP32), 0 elsewhere; *dc2 = ||dc||^2
void launch_bc_delta(const double* u, const double* fixed_vals, const uint8_t* fixed, float* dc,
                     int n, Reduce red, int site, double* dc2, cudaStream_t s);
// out = R - y on free DOFs, 0 on fixed DOFs
void launch_rhs_minus(const double* R, const float* y, const uint8_t* fixed, double* out, int n,
                      cudaStream_t s);

}  // namespace femb200
