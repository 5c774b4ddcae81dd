// Internal structures shared by the host driver (fem_ctx.cu) and the kernels
// (fem_kernels.cu).  Not part of the public ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "fem_device.cuh"

namespace femb200 {

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
};

// Last-block reduction bookkeeping: one slot per reduction site.
struct Reduce {
  double* partials;         // [n_sites][max_blocks]
  unsigned int* counters;   // [n_sites]
  int max_blocks;
};

// Device-resident PCG state (read by every CG kernel, advanced by the last
// block of each reduction so no host round trip is needed per iteration).
struct CGState {
  double rz, pAp, rr, rr0, tol2, alpha, beta, pad;
  int iter, max_iter, done, status;  // done: 0 running, 1 converged, 2 max iters, 3 breakdown
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
};

struct MvArgs {
  MeshDev m;
  const DevMat<float>* matF;
  const float* payload;
  const float* x;           // [3 Nn (padded)]
  float* y;
  CGState* cg;              // non-null: CG-fused (early exit, p.Ap, alpha)
  Reduce red;
  int red_site;
  int mask_input;           // 1: fixed DOFs of x read as zero (K_ff x); 0: K_f,all x
};

struct DiagArgs {
  MeshDev m;
  const DevMat<float>* matF;
  const float* payload;
  float* dinv;              // [3 Nn] 1/diag(K) on free DOFs, 0 elsewhere
};

// Records a failure for fem_last_error(NULL) (thread-local, fem_ctx.cu) and
// returns `code`.
int set_global_error(int code, const char* fmt, ...);

// launchers (fem_kernels.cu)
void launch_residual(const ResArgs& a, int model, cudaStream_t s);
void launch_matvec(const MvArgs& a, int model, cudaStream_t s);
void launch_diag(const DiagArgs& a, int model, cudaStream_t s);
void launch_cg_init(const double* b, float* r, float* x, float* p, const float* dinv, int ndof4,
                    CGState* cg, double rtol, int maxit, Reduce red, int site, cudaStream_t s);
void launch_cg_update(float* x, float* r, const float* p, const float* y, const float* dinv,
                      int ndof4, CGState* cg, Reduce red, int site, cudaStream_t s);
void launch_cg_pupdate(float* p, const float* r, const float* dinv, int ndof4, CGState* cg,
                       cudaStream_t s);
void launch_stress(const MeshDev& m, const DevMat<double>* matD, int model, const double* u,
                   const double* ep_c, const double* epe_c, const int* perm_elem, double* F_out,
                   double* sig_out, cudaStream_t s);
void launch_refq(const MeshDev& m, const int* perm_elem, double* dNdX, double* vol,
                 cudaStream_t s);
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
void launch_u_update(double* u, const double* u_base, const float* du, double alpha, int ndof,
                     cudaStream_t s);
void launch_gather_d_masked(const double* in_user, double* out_int, const int* perm,
                            const uint8_t* fixed, int n, cudaStream_t s);
void launch_dinv_identity(float* dinv, const uint8_t* fixed, int n, cudaStream_t s);
// dc = (fixed_vals - u) on fixed DOFs (FP32), 0 elsewhere; *dc2 = ||dc||^2
void launch_bc_delta(const double* u, const double* fixed_vals, const uint8_t* fixed, float* dc,
                     int n, Reduce red, int site, double* dc2, cudaStream_t s);
// out = R - y on free DOFs, 0 on fixed DOFs
void launch_rhs_minus(const double* R, const float* y, const uint8_t* fixed, double* out, int n,
                      cudaStream_t s);
void launch_d2f_masked(const double* in, float* out, const uint8_t* fixed, int n, cudaStream_t s);

}  // namespace femb200
