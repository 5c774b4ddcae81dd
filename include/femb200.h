/*
 * femb200.h — C ABI of the B200-native TET4 FEM static-solve path.
 *
 * The reference (monostylegc/simul, backend/fea/fem) is Python + Taichi and has
 * no native FFI; each entry point below replaces the Python/Taichi call named in
 * its comment (paths relative to the reference project root).  A Python host
 * binds these with ctypes (simul_b200/_lib.py); any C caller can use them.
 *
 * Conventions
 *  - Every function returns an int status (FEM_OK = 0).  The message of the
 *    last failure on a context is returned by fem_last_error(ctx); failures of
 *    fem_ctx_create are reported by fem_last_error(NULL) (thread-local).
 *  - Mesh set-up arrays (FemMeshDesc, material tables) are HOST pointers.
 *  - All per-call arrays are DEVICE pointers on the context's device, in the
 *    caller's node / element order, row-major (node-major, xyz inner).
 *  - The context owns its scratch memory and CUDA graphs; caller-visible
 *    buffers belong to the caller.  Work is issued on the context's stream;
 *    calls that return host values synchronise that stream.
 *  - One context per stream.  Contexts share no mutable state; calls on one
 *    context must not overlap.
 *  - Device loops carry iteration caps; exhausting one returns FEM_ERR_BUDGET
 *    instead of spinning.
 */
#ifndef FEMB200_H
#define FEMB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; map onto backend/fea/fem/validation.py:18-66 */
enum {
  FEM_OK = 0,
  FEM_ERR_INVALID = 1,      /* FEAValidationError (validation.py:18-41) */
  FEM_ERR_CUDA = 2,         /* CUDA runtime failure */
  FEM_ERR_NAN = 3,          /* FEAConvergenceError(reason="nan_divergence"), static_solver.py:174-182 */
  FEM_NOT_CONVERGED = 4,    /* converged=False in the solve dict */
  FEM_ERR_BUDGET = 5,       /* a capped device loop ran out of iterations */
  FEM_ERR_STATE = 6,        /* call order violated (e.g. matvec before any residual) */
  FEM_CANCELLED = 7         /* progress callback returned 0 (static_solver.py:203-216) */
};

/* constitutive models (backend/fea/fem/material/*.py) */
enum {
  FEM_LINEAR_ELASTIC = 0,        /* linear_elastic.py:22-176 */
  FEM_NEO_HOOKEAN = 1,           /* neo_hookean.py:31-226 */
  FEM_MOONEY_RIVLIN = 2,         /* mooney_rivlin.py:36-294 (volumetric term as written) */
  FEM_J2 = 3,                    /* j2_plasticity.py:33-526, 3D small strain */
  FEM_TRANSVERSE_ISOTROPIC = 4,  /* transverse_isotropic.py:36-399, small strain */
  FEM_FIBRE_MOONEY_RIVLIN = 5    /* hyperelastic fibre-reinforced MR; no reference counterpart */
};

/* preconditioners of fem_pcg / fem_newton_solve.  The reference factorises the
 * assembled tangent instead (static_solver.py:399-462).  TWO_LEVEL adds to
 * Jacobi a Galerkin coarse correction on a lattice of trilinear cells:
 * z = D^-1 r + P (P^T K P)^-1 P^T r. */
enum { FEM_PRECOND_NONE = 0, FEM_PRECOND_JACOBI = 1, FEM_PRECOND_TWO_LEVEL = 2, FEM_PRECOND_LEARNED = 3 };

/* line-search policy of fem_newton_solve */
enum {
  FEM_LS_REFERENCE = 0,  /* halve alpha up to 5x while |R| does not drop; keep the last trial
                            (static_solver.py:235-253) */
  FEM_LS_GUARDED = 1,    /* full step unless the trial residual is non-finite or grows more than
                            1e6x; then halve (up to 5x) */
  FEM_LS_NONE = 2
};

#define FEM_MAX_MATERIALS 16

/* Mesh description: replaces FEMesh(n_nodes, n_elements, TET4 | HEX8) +
 * initialize_from_numpy (core/mesh.py:25-121).  HOST pointers. */
typedef struct {
  int64_t n_nodes;
  int64_t n_elements;
  const double* X;        /* (n_nodes, 3) reference coordinates */
  const int32_t* conn;    /* (n_elements, nodes_per_elem) connectivity */
  int32_t device;         /* CUDA device ordinal */
  int32_t nodes_per_block;/* 0 = default (256); 128 / 256 / 512 accepted */
  void* stream;           /* cudaStream_t; NULL = a context-owned stream */
  int32_t nodes_per_elem; /* 0 or 4: TET4 (one Gauss point); 8: HEX8, vertex order of
                             core/element.py:297-315, 2 x 2 x 2 Gauss points.  HEX8
                             contexts solve with Jacobi / nodal block-Jacobi PCG: a
                             two-level or learned request runs Jacobi-PCG and is counted
                             in fem_coarse_info's jacobi_fallbacks */
} FemMeshDesc;

/* One material of the table: replaces the MaterialBase subclasses'
 * constructors (material/base.py:16-63 and framework/material.py:85-138).
 * Unused fields are ignored for a model.  All moduli are multiplied by the
 * per-element scale given to fem_set_materials (sigma_y is not). */
typedef struct {
  int32_t model;
  double E, nu;                 /* LE / NH / J2 */
  double sigma_y, H;            /* J2: yield stress, linear isotropic hardening */
  double C10, C01, D1;          /* MR and fibre MR (D1 <= 1e-20: no volumetric term) */
  double C_voigt[36];           /* TI: global 6x6, Voigt [11,22,33,23,13,12] */
  double fiber_dir[2][3];       /* fibre MR: unit fibre directions */
  double fiber_E;               /* fibre MR: fibre stiffness (tension only) */
  int32_t n_fibers;             /* fibre MR: 0..2 */
} FemMaterial;

typedef struct {
  int32_t max_iterations;   /* Newton iterations, default 50 (static_solver.py:37) */
  double tol;               /* relative residual vs the first residual of the solve (Q8) */
  int32_t line_search;      /* FEM_LS_* */
  int32_t precond;          /* FEM_PRECOND_* */
  int32_t cg_max_iterations;/* per Newton iteration */
  double cg_rtol_min;       /* lower bound of the inexact-Newton forcing term */
  double cg_rtol_max;       /* upper bound of the forcing term */
  int32_t auto_commit;      /* commit J2 history after a converged solve */
  int32_t verbose;
  /* optional progress callback: return 0 to cancel (static_solver.py:203-216) */
  int32_t (*progress)(void* user, int32_t iteration, double residual, double relative_residual);
  void* progress_user;
} FemSolveParams;

typedef struct {
  int32_t converged;
  int32_t iterations;       /* reference semantics: Newton loop passes (static_solver.py:260-265) */
  double residual;
  double relative_residual;
  int32_t cancelled;
  int32_t cg_iterations;    /* total over the solve */
  int32_t residual_evals;
  double first_residual;
} FemSolveResult;

/* ---- lifecycle ---- */
/* FEMesh.__init__ + initialize_from_numpy + _compute_reference_quantities
 * (core/mesh.py:25-151).  Reorders nodes/elements internally (Morton) and
 * builds the node-block gather tables; callers keep their own order. */
int fem_ctx_create(const FemMeshDesc* desc, void** ctx_out);
int fem_ctx_destroy(void* ctx);
const char* fem_last_error(void* ctx);
/* sizes/statistics: out[0]=n_nodes out[1]=n_elements out[2]=n_blocks
 * out[3]=block element entries (incl. redundant) out[4]=nodes_per_block
 * out[5]=device bytes held */
int fem_ctx_info(void* ctx, int64_t* out6);
/* counters since creation: out[0] kernel launches that did work (library
 * kernels only), out[1] CG iterations, out[2] residual evaluations,
 * out[3] CG graph launches; matvec variant selection: out[4] variant in use
 * (0 fused node-block, 1 two-phase, 2 element-block), out[5] / out[6] timed
 * ns per launch of the fused / two-phase variant (0 if not timed), out[7] 1
 * if the choice was made by timing; out[8] PCG solves run as one whole-solve
 * graph launch (conditional WHILE node), out[9] 1 if such graphs are
 * available; out[10] timed ns of the element-block variant at its best block
 * size, out[11] that size (0: no element-block tables), out[12..15] timed ns
 * at 256, 512, 768 and 1024 elements per block (0 if not timed), out[16]
 * timed ns of the warp-aggregated variant (variant 3 in out[4]), out[17]
 * timed ns of the persistent two-phase variant (variant 4) */
int fem_ctx_stats(void* ctx, int64_t* out18);

/* Option keys of fem_set_option (no reference counterpart: the reference has
 * one matvec formulation, backend/fea/fem/material/nonlinear/base.py:110-145). */
enum {
  /* -1 (default): time the tangent-matvec variants on the first PCG solve
   * and keep the fastest; 0: fused node-block kernel; 1: element pass writing
   * slot vectors in node order plus a node gather; 2 (TET4): element-block
   * kernel that sums each block's slot vectors in shared memory, nodes
   * shared by blocks completed by a second kernel; 3 (TET4): the two-phase
   * pass with each warp's slot vectors added per vertex in shared memory
   * before the node gather; 4 (TET4): the two-phase pair as persistent
   * grid-stride kernels (one wave of CTAs, next element's inputs
   * prefetched) */
  FEM_OPT_MATVEC_VARIANT = 1,
  /* two-level preconditioner: lattice cell edge in mesh lengths (default 8;
   * the cube root of 5x the mean element volume, i.e. the voxel edge of
   * 5-tet voxel meshes); grown automatically past 4096 coarse nodes */
  FEM_OPT_COARSE_CELL = 2,
  /* two-level preconditioner: when the coarse operator is rebuilt.  -1
   * (default): adaptive - rebuilt at the next tangent once a solve needs
   * 1.5x the CG iterations per decade of residual reduction measured right
   * after the last assembly; 0: once per state - at the first two-level
   * solve after a history reset, a materials change or a new constraint
   * pattern, then kept for the whole load path; k >= 1: every k PCG solves.
   * Any mode assembles afresh after such a reset or change. */
  FEM_OPT_COARSE_REUSE = 3,
  /* learned preconditioner: 1 (default) adds the two-level coarse correction
   * to the network's output, 0 uses the network alone */
  FEM_OPT_LEARNED_COARSE = 4,
  /* two-level preconditioner: 1 stores the coarse inverse in BF16 (half the
   * bytes per CG iteration; FP32 products), 0 (default) in FP32 */
  FEM_OPT_COARSE_BF16 = 5,
  /* 1: the CG work after each matvec (update, restriction, coarse product,
   * preconditioner, direction) runs as one cooperative kernel with grid-wide
   * barriers, where the runtime accepts it in a graph; 0 (default): as a
   * chain of kernels.  Jacobi and two-level; batched solves use the chain. */
  FEM_OPT_FUSED_STEP = 6,
  /* 1 (default): a PCG solve runs as one graph launch (a conditional WHILE
   * node); 0: as launches of fixed 12- or 32-iteration graphs with a host
   * check between them (kernel profilers cannot attribute kernels inside
   * conditional graphs) */
  FEM_OPT_WHOLE_SOLVE_GRAPH = 7,
  /* 1 (default): inside the captured CG graphs each kernel of the iteration
   * chain is launched as a programmatic dependent of the previous one (it is
   * scheduled while the previous one drains and waits for its results on the
   * device), where the runtime accepts it; 0: plain stream order */
  FEM_OPT_PDL = 8,
  /* 1 (default): two-level PCG with the two-phase matvec applies the matvec
   * to z and forms the direction in its node gather by recurrence,
   * p = z + beta p and K p = K z + beta K p_old, saving the direction-update
   * kernel; 0: p = z + beta p in its own kernel, then K p */
  FEM_OPT_DIRECTION_RECURRENCE = 9,
  /* two-level preconditioner smoother: 1 (default) the inverse of each
   * node's 3 x 3 diagonal block of K_T (free DOFs), 0 the inverse of the
   * diagonal */
  FEM_OPT_BLOCK_JACOBI = 10,
  /* two-level coarse inverse (the project's dense kernels: blocked Cholesky
   * L L^T, W = L^-1, the lower triangle of W^T W): 0 or 1 (default) in FP64,
   * 2 in FP32 (enough for the FP32 or BF16 copy that is applied), 3 FP32
   * Cholesky with W and W^T W on TF32 tensor-core tiles (tcgen05) */
  FEM_OPT_COARSE_INVERSE = 11,
  /* two-level: at most this many coarse nodes (default 4096, up to 16384);
   * the lattice cell grows by 25 % steps until the lattice fits */
  FEM_OPT_COARSE_MAX_NODES = 12,
  /* element-block matvec: elements per block (one thread each), 256, 512,
   * 768 or 1024; 0 (default) times the four and keeps the fastest */
  FEM_OPT_EB_SIZE = 13,
  /* TET4 FP64 residual: 1 (default) two-phase (one thread per element
   * writing its slot forces in node-slot order, then a node gather), 0 the
   * fused node-block kernel (elements shared by node blocks evaluated in
   * each) */
  FEM_OPT_RESIDUAL_TWO_PHASE = 14,
  /* load-step extrapolation, 0 (default) off, 1 on: a Newton solve that
   * follows a converged one, with u unchanged since, starts from the last
   * solve's end state plus its change of u (the step repeated) instead of
   * carrying the new prescribed values by a first linear solve.  The
   * relative residual is still measured against the reference's first
   * residual (the previous u under the new loads).  A history reset or a
   * non-converged solve starts the sequence again. */
  FEM_OPT_EXTRAPOLATE = 15
};
int fem_set_option(void* ctx, int32_t key, int64_t value);
/* Learned preconditioner (no reference counterpart).  A message-passing
 * network over mesh nodes (4 layers, width 64, BF16 weights on tcgen05 tensor
 * cores, FP32 accumulation) maps a residual r to a correction
 *   z = D^-1 r + s D^-1/2 net(D^-1/2 r / s, fixed bits, log-modulus) (+ coarse)
 * used by flexible PCG (FEM_PRECOND_LEARNED); Jacobi-based PCG reruns the
 * solve when the flexible one breaks down or exhausts its iterations.
 * Parameters: FP32, flat order W_e[64][16], b_e[64], 4 x (W_l[64][128],
 * b_l[64]), W_d[3][64], b_d[3] (34,307 values), host arrays. */
int fem_mpnn_set_weights(void* ctx, const float* w, int64_t n);
int fem_mpnn_get_weights(void* ctx, float* w, int64_t n);
/* z = M(r) at the current tangent (caller order, N x 3 FP32 device arrays) */
int fem_mpnn_forward(void* ctx, const float* r, float* z);
/* out[0] flexible solves that fell back to Jacobi-based PCG, out[1] 1 if
 * weights are set, out[2] flexible PCG steps so far, out[3] of which used the
 * Jacobi (+ coarse) direction because the network's was not a descent
 * direction (r.z_net <= 0.25 r.z_jacobi) */
int fem_learned_stats(void* ctx, int64_t* out4);
/* grad (host, 34,307 FP32) = d<gz, M(r)>/dw at the current tangent; r, gz:
 * caller order, N x 3 FP32 device arrays (network only, no coarse part) */
int fem_mpnn_backward(void* ctx, const float* r, const float* gz, float* grad);

/* Training on (residual, correction) pairs the plain solver produced at this
 * context's current tangent: R, E device arrays [n_pairs][N][3] FP32 in
 * caller order, K_ff E_k ~ R_k.  Loss per pair (the preconditioner's A-norm
 * error, 1 for z = 0): (z.Kz - 2 z.r + e.r) / e.r with z = M(r) (+ coarse
 * when FEM_OPT_LEARNED_COARSE is set).  Adam (beta 0.9 / 0.999), gradients
 * averaged over `batch` pairs, forward and backward on the GPU. */
typedef struct {
  int32_t steps;
  int32_t batch;
  double lr;
  int32_t seed;              /* sample order */
  int32_t reset_optimizer;   /* 1: zero the Adam moments first */
  int32_t (*progress)(void* user, int32_t step, double loss, double unused);
  void* progress_user;
} FemTrainParams;

typedef struct {
  int32_t steps_done;
  double loss_first;         /* mean loss of the first steps (up to 16) */
  double loss_last;          /* mean loss of the last steps */
} FemTrainResult;

int fem_mpnn_train(void* ctx, const float* R, const float* E, int32_t n_pairs, const FemTrainParams* prm,
                   FemTrainResult* res);
/* mean loss over the pairs for the network (loss_net) and for the same
 * preconditioner with the network's output zeroed, i.e. Jacobi (+ coarse)
 * (loss_base) */
int fem_mpnn_eval(void* ctx, const float* R, const float* E, int32_t n_pairs, double* loss_net,
                  double* loss_base);

/* Known-answer check of the tensor-core path the learned preconditioner uses
 * (no reference counterpart): D (128 x N, FP32) = A (128 x K) B^T (B: N x K),
 * BF16 row-major device arrays, one tcgen05 tile; N, K multiples of 16 in
 * [16, 256].  Errors go to fem_last_error(NULL). */
int fem_selftest_umma(const void* A, const void* B, float* D, int32_t N, int32_t K, void* stream);
/* Dense SPD inverse, the kernels the two-level preconditioner forms its
 * coarse inverse with (no reference counterpart: the reference has no coarse
 * space; its direct solve is scipy's spsolve of the assembled tangent,
 * backend/fea/fem/solver/static_solver.py:430-462).  A: n x n column-major
 * device array (FP64, lower
 * triangle read); out: n x n column-major device array receiving the lower
 * triangle of A^-1; precision 64, 32 (FP32 arithmetic) or 19 (FP32
 * Cholesky and W, then W^T W on TF32 tensor-core tiles: tcgen05.mma
 * kind::tf32, operands rounded to a 10-bit mantissa, FP32 sums).  Blocked
 * Cholesky A = L L^T, W = L^-1, A^-1 = W^T W on the project's tile kernels.
 * FEM_ERR_NAN if a pivot is not positive, FEM_ERR_BUDGET if a tensor-core
 * completion wait timed out.  Allocates its work space.
 * Errors: fem_last_error(NULL). */
int fem_dense_spd_inverse(const double* A, int32_t n, int32_t precision, double* out, void* stream);
/* The same for a matrix with an envelope: row_first (host, n entries,
 * 0 <= row_first[r] <= r) is the lowest column of row r that may be
 * nonzero in A's lower triangle.  The Cholesky factor's fill stays inside
 * that envelope, so the factorisation and W's update skip the tiles outside
 * it; the result is bitwise that of fem_dense_spd_inverse (the skipped
 * products would add exact zeros).  The solver's coarse inverse uses it
 * with the lattice envelope of the coarse operator. */
int fem_dense_spd_inverse_banded(const double* A, int32_t n, int32_t precision, const int32_t* row_first,
                                 double* out, void* stream);

/* ---- node-to-node contact between two bodies (backend/fea/framework/contact.py) ----
 * Device arrays in the caller's node order, FP64 current coordinates
 * (reference + displacement, n x 3), surfaces as int32 node lists; forces
 * are ADDED to f_a / f_b (n x 3 FP64, zero them first), bitwise
 * reproducible.  Errors: fem_last_error(NULL). */
/* NodeNodeContact.detect's nearest-neighbour query (contact.py:49-92):
 * for every A-surface node i, nearest[i] = the index into surf_b of its
 * nearest B-surface node (the smaller index on ties), dist[i] its distance. */
int fem_contact_nearest(const double* pos_a, const int32_t* surf_a, int32_t na, const double* pos_b,
                        const int32_t* surf_b, int32_t nb, int32_t* nearest, double* dist, void* stream);
/* detect + compute_forces (contact.py:49-173, no damping): pairs closer
 * than gap_tol get f = penalty (gap_tol - d) (x_a - x_b) / max(d_ab, 1e-15)
 * on A and -f on B (added in pair order, as np.add.at); *n_pairs and *total
 * (= sum |f| over A's components, scene.py:357) on the host. */
int fem_contact_penalty(const double* pos_a, const int32_t* surf_a, int32_t na, const double* pos_b,
                        const int32_t* surf_b, int32_t nb, double gap_tol, double penalty, double* f_a, double* f_b,
                        int32_t* n_pairs, double* total, void* stream);
/* compute_tied_forces (contact.py:224-273): pairs (n_pairs x 2 int32, A
 * node, B node; each A node once), offsets (n_pairs x 3) the initial
 * x_a - x_b; f = -penalty ((x_a - x_b) - offset) on A, -f on B; nb_nodes =
 * B's node count; *total = sum |f| (host). */
int fem_contact_tied(const double* pos_a, const double* pos_b, const int32_t* pairs, const double* offsets,
                     int32_t n_pairs, int32_t nb_nodes, double penalty, double* f_a, double* f_b, double* total,
                     void* stream);
/* two-level preconditioner state: out[0] lattice cells, [1] coarse nodes,
 * [2] coarse DOFs, [3] cell edge, [4] assemblies so far, [5] ms of the last
 * assembly + factorisation (CUDA events), [6] ms of its assembly part,
 * [7] the rebuild policy (FEM_OPT_COARSE_REUSE), [8] refreshes whose
 * operator was not positive definite (the last inverse kept), [9] two-level
 * solves run as Jacobi-PCG because no positive definite coarse operator
 * existed yet */
int fem_coarse_info(void* ctx, double* out10);
/* CG iteration launch structure: out[0] 1 while the fused-step option is on
 * and the runtime accepted it, [1] the captured Jacobi CG graph uses the
 * fused step, [2] the two-level one does, [3] warps per lattice cell in the
 * restriction, [4] the Jacobi CG graph uses programmatic dependent launches,
 * [5] the two-level one does */
int fem_step_info(void* ctx, int64_t* out6);
/* cudaStream_t of the context (as void*) */
void* fem_ctx_stream(void* ctx);

/* ---- set-up ---- */
/* material table + per-element material id (uint8, host, nullable = all 0)
 * and per-element modulus scale (float, host, nullable = all 1).
 * Replaces StaticSolver(material=..., materials={id: mat}) with the element
 * ids of FEMesh.material_id (static_solver.py:32-71, core/mesh.py:78-79),
 * honouring per-element materials in the residual. */
int fem_set_materials(void* ctx, const FemMaterial* table, int32_t n_materials,
                      const uint8_t* elem_material /*host*/, const float* elem_scale /*host*/);
/* Dirichlet mask / values and external forces, device pointers (n_nodes,3);
 * NULL keeps the previous array.  Replaces set_fixed_nodes / set_fixed_dofs /
 * set_nodal_forces (core/mesh.py:329-399). */
int fem_set_bc(void* ctx, const uint8_t* fixed_mask, const double* fixed_values,
               const double* f_ext);
/* u = fixed value on fixed DOFs — apply_boundary_conditions (core/mesh.py:321-327) */
int fem_apply_bc(void* ctx);
int fem_set_displacement(void* ctx, const double* u);
int fem_get_displacement(void* ctx, double* u_out);

/* ---- kernels ---- */
/* dN/dX (n_points,npe,3) and Gauss volumes (n_points) —
 * _compute_reference_quantities (core/mesh.py:123-151).  Either may be NULL.
 * n_points = n_elements (TET4) or 8 n_elements (HEX8, point e * 8 + g). */
int fem_reference_quantities(void* ctx, double* dNdX_out, double* vol_out);
/* F (n_points,3,3) and Cauchy stress (n_points,3,3) at displacement u
 * (NULL = context u) — compute_deformation_gradient (core/mesh.py:293-313)
 * + MaterialBase.compute_stress (e.g. neo_hookean.py:91-129,
 * j2_plasticity.py:159-249; J2 starts from the committed history). */
int fem_compute_stress(void* ctx, const double* u, double* F_out, double* sigma_out);
/* Fused F -> stress -> element forces -> deterministic node gather (FP64).
 * f_out (nullable) receives the negative internal force (the reference's
 * mesh.f), residual_out (nullable) R = f_ext + f with fixed DOFs zeroed;
 * *rnorm (nullable) = ||R||.  Also refreshes the tangent state used by
 * fem_tangent_matvec / fem_pcg.  Replaces compute_deformation_gradient +
 * compute_stress + compute_nodal_forces (neo_hookean.py:131-190 etc.) and the
 * residual of static_solver.py:161-172. */
int fem_element_forces(void* ctx, const double* u, double* f_out, double* residual_out,
                       double* rnorm);
/* Nodal von Mises stress (n_nodes, device) at displacement u (NULL = context
 * u): per node the von Mises stress of every element on it (of the element's
 * Gauss-point mean stress for HEX8), added in a fixed
 * order (no atomics); average = 0 keeps the sum, as compute_mises_stress
 * leaves it (core/mesh.py:459-492, returned by StaticSolver.get_mises_stress,
 * static_solver.py:512-515), average = 1 divides by the element count. */
int fem_nodal_mises(void* ctx, const double* u, double* mises_out, int32_t average);
/* y = K_T x with the consistent tangent at the last fem_element_forces state;
 * fixed DOFs of x are ignored and of y zeroed (FP32).  Matrix-free
 * replacement of _assemble_tangent_stiffness (static_solver.py:349-397,
 * assembly.py:20-287). */
int fem_tangent_matvec(void* ctx, const float* x, float* y);
/* Preconditioned CG on K_T du = r (free DOFs), FP32 vectors, FP64 dots.
 * Replaces _solve_linear_system (static_solver.py:399-462). */
int fem_pcg(void* ctx, int32_t precond, const double* r, double* du, double rtol,
            int32_t max_iterations, int32_t* iterations_out, double* rel_residual_out);
/* One static solve at the current loads — StaticSolver.solve / _solve_newton
 * (static_solver.py:73-99, 135-265), Newton in FP64 with inexact PCG inner
 * solves in FP32 (mixed-precision iterative refinement). */
int fem_newton_solve(void* ctx, const FemSolveParams* params, FemSolveResult* result);
void fem_default_solve_params(FemSolveParams* p);

/* Load stepping (the reference loops solve() with scaled loads, e.g.
 * benchmark_spine_compression.py:413-415): prescribed values and external
 * forces become s x the values last given to fem_set_bc. */
int fem_set_load_scale(void* ctx, double s);

/* Batched solves of independent contexts (no reference counterpart): each
 * context, on its own stream, runs `load_steps` load steps (scale k/steps,
 * fem_set_load_scale + fem_newton_solve) on a pool of n_threads host workers
 * (0: one per context), so the instances' kernels overlap on the GPU.
 * results[i] aggregates instance i (iterations summed, converged if every
 * step converged), status[i] its status, wall_ms[i] (optional) its host wall
 * time.  Contexts must be distinct and must not share a stream with other
 * work.  Progress callbacks are ignored. */
int fem_batch_solve(void** ctxs, int32_t n, const FemSolveParams* prm, int32_t load_steps,
                    FemSolveResult* results, int32_t* status, double* wall_ms, int32_t n_threads);

/* Kernel timing (no reference counterpart; the reference has only wall clocks,
 * framework/_adapters/fem_adapter.py:162-172).  Launches each hot kernel
 * `reps` times back to back on the context stream at the current tangent
 * state and writes the mean CUDA-event milliseconds per launch:
 * ms_out[0] tangent matvec (CG-fused), [1] FP64 residual, [2] CG update,
 * [3] CG direction update.  Clobbers the context's CG scratch vectors. */
int fem_profile_kernels(void* ctx, int32_t reps, double* ms_out);

/* Allocation-free FP64 dot product, *result = sum_i a[i] b[i] (device pointers,
 * issued on `stream`, a cudaStream_t or NULL).  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc (an application whose
 * allocator owns all device memory, a loop that forbids allocation after
 * start-up): the same deterministic scheme as the solver's dots and norms
 * (fixed-order per-block partials, the last block adds them in index order),
 * with its own 4096-element tiles, so it is not bitwise equal to the solver's
 * norms; its partial sums live in a static 16 KB device array instead of
 * context scratch.  n <= 8,388,608 (larger n: FEM_ERR_INVALID).
 * The first call on a device looks up that array's address there; make it
 * before any stream capture.  The address is kept until the process exits: no
 * calls after a cudaDeviceReset.  Calls share the array: calls that overlap on
 * the GPU race and must be serialised.  Errors: fem_last_error(NULL). */
int fem_dot_f64_noalloc(const double* a, const double* b, int64_t n, double* result, void* stream);

/* ---- J2 history (j2_plasticity.py:103-123, 513-520) ---- */
int fem_commit_history(void* ctx);
/* back to rest: zero history; also discards the two-level coarse operator
 * (the next two-level solve assembles one for the new tangent) */
int fem_reset_history(void* ctx);
/* plastic strain (n_points,3,3) and equivalent plastic strain (n_points),
 * committed state; either may be NULL. */
int fem_get_history(void* ctx, double* ep_out, double* epe_out);

#ifdef __cplusplus
}
#endif
#endif /* FEMB200_H */
