"""ctypes binding of ``libfemb200.so`` (declarations in ``include/femb200.h``).

Loading fails loudly: there is no CPU fallback for the solver path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfemb200.so"

FEM_OK = 0
FEM_ERR_INVALID = 1
FEM_ERR_CUDA = 2
FEM_ERR_NAN = 3
FEM_NOT_CONVERGED = 4
FEM_ERR_BUDGET = 5
FEM_ERR_STATE = 6
FEM_CANCELLED = 7

FEM_LINEAR_ELASTIC = 0
FEM_NEO_HOOKEAN = 1
FEM_MOONEY_RIVLIN = 2
FEM_J2 = 3
FEM_TRANSVERSE_ISOTROPIC = 4
FEM_FIBRE_MOONEY_RIVLIN = 5

FEM_PRECOND_NONE = 0
FEM_PRECOND_JACOBI = 1
FEM_PRECOND_TWO_LEVEL = 2
FEM_PRECOND_LEARNED = 3

FEM_LS_REFERENCE = 0
FEM_LS_GUARDED = 1
FEM_LS_NONE = 2

FEM_MAX_MATERIALS = 16

FEM_OPT_MATVEC_VARIANT = 1
FEM_OPT_COARSE_CELL = 2
FEM_OPT_COARSE_REUSE = 3
FEM_OPT_LEARNED_COARSE = 4
FEM_OPT_COARSE_BF16 = 5
FEM_OPT_FUSED_STEP = 6
FEM_OPT_WHOLE_SOLVE_GRAPH = 7
FEM_OPT_PDL = 8
FEM_OPT_DIRECTION_RECURRENCE = 9
FEM_OPT_BLOCK_JACOBI = 10
FEM_OPT_COARSE_INVERSE = 11
FEM_OPT_COARSE_MAX_NODES = 12
FEM_OPT_EB_SIZE = 13
FEM_OPT_RESIDUAL_TWO_PHASE = 14
FEM_OPT_EXTRAPOLATE = 15
MPNN_PARAMS = 34307
MATVEC_VARIANTS = {0: "fused", 1: "two_phase", 2: "element_block", 3: "warp_agg", 4: "persistent"}


class FemMeshDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("n_elements", C.c_int64),
                ("X", C.POINTER(C.c_double)), ("conn", C.POINTER(C.c_int32)),
                ("device", C.c_int32), ("nodes_per_block", C.c_int32),
                ("stream", C.c_void_p), ("nodes_per_elem", C.c_int32)]


class FemMaterial(C.Structure):
    _fields_ = [("model", C.c_int32), ("E", C.c_double), ("nu", C.c_double),
                ("sigma_y", C.c_double), ("H", C.c_double),
                ("C10", C.c_double), ("C01", C.c_double), ("D1", C.c_double),
                ("C_voigt", C.c_double * 36), ("fiber_dir", (C.c_double * 3) * 2),
                ("fiber_E", C.c_double), ("n_fibers", C.c_int32)]


PROGRESS_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_int32, C.c_double, C.c_double)


class FemSolveParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("tol", C.c_double),
                ("line_search", C.c_int32), ("precond", C.c_int32),
                ("cg_max_iterations", C.c_int32), ("cg_rtol_min", C.c_double),
                ("cg_rtol_max", C.c_double), ("auto_commit", C.c_int32),
                ("verbose", C.c_int32), ("progress", PROGRESS_FN),
                ("progress_user", C.c_void_p)]


class FemTrainParams(C.Structure):
    _fields_ = [("steps", C.c_int32), ("batch", C.c_int32), ("lr", C.c_double), ("seed", C.c_int32),
                ("reset_optimizer", C.c_int32), ("progress", PROGRESS_FN), ("progress_user", C.c_void_p)]


class FemTrainResult(C.Structure):
    _fields_ = [("steps_done", C.c_int32), ("loss_first", C.c_double), ("loss_last", C.c_double)]


class FemSolveResult(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32),
                ("residual", C.c_double), ("relative_residual", C.c_double),
                ("cancelled", C.c_int32), ("cg_iterations", C.c_int32),
                ("residual_evals", C.c_int32), ("first_residual", C.c_double)]


# every symbol include/femb200.h declares, with (restype, argtypes)
_VP = C.c_void_p
_DP = C.POINTER(C.c_double)
SIGNATURES = {
    "fem_ctx_create": (C.c_int, [C.POINTER(FemMeshDesc), C.POINTER(C.c_void_p)]),
    "fem_ctx_destroy": (C.c_int, [_VP]),
    "fem_last_error": (C.c_char_p, [_VP]),
    "fem_ctx_info": (C.c_int, [_VP, C.POINTER(C.c_int64)]),
    "fem_ctx_stats": (C.c_int, [_VP, C.POINTER(C.c_int64)]),
    "fem_ctx_stream": (C.c_void_p, [_VP]),
    "fem_set_option": (C.c_int, [_VP, C.c_int32, C.c_int64]),
    "fem_coarse_info": (C.c_int, [_VP, _DP]),
    "fem_step_info": (C.c_int, [_VP, C.POINTER(C.c_int64)]),
    "fem_selftest_umma": (C.c_int, [_VP, _VP, _VP, C.c_int32, C.c_int32, _VP]),
    "fem_dense_spd_inverse": (C.c_int, [_VP, C.c_int32, C.c_int32, _VP, _VP]),
    "fem_dense_spd_inverse_banded": (C.c_int, [_VP, C.c_int32, C.c_int32, C.POINTER(C.c_int32), _VP, _VP]),
    "fem_contact_nearest": (C.c_int, [_VP, _VP, C.c_int32, _VP, _VP, C.c_int32, _VP, _VP, _VP]),
    "fem_contact_penalty": (C.c_int, [_VP, _VP, C.c_int32, _VP, _VP, C.c_int32, C.c_double, C.c_double, _VP, _VP,
                                      C.POINTER(C.c_int32), C.POINTER(C.c_double), _VP]),
    "fem_contact_tied": (C.c_int, [_VP, _VP, _VP, _VP, C.c_int32, C.c_int32, C.c_double, _VP, _VP,
                                   C.POINTER(C.c_double), _VP]),
    "fem_mpnn_set_weights": (C.c_int, [_VP, C.POINTER(C.c_float), C.c_int64]),
    "fem_mpnn_get_weights": (C.c_int, [_VP, C.POINTER(C.c_float), C.c_int64]),
    "fem_mpnn_forward": (C.c_int, [_VP, _VP, _VP]),
    "fem_learned_stats": (C.c_int, [_VP, C.POINTER(C.c_int64)]),
    "fem_mpnn_backward": (C.c_int, [_VP, _VP, _VP, C.POINTER(C.c_float)]),
    "fem_mpnn_train": (C.c_int, [_VP, _VP, _VP, C.c_int32, C.POINTER(FemTrainParams),
                                 C.POINTER(FemTrainResult)]),
    "fem_mpnn_eval": (C.c_int, [_VP, _VP, _VP, C.c_int32, _DP, _DP]),
    "fem_set_load_scale": (C.c_int, [_VP, C.c_double]),
    "fem_batch_solve": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(FemSolveParams), C.c_int32,
                                  C.POINTER(FemSolveResult), C.POINTER(C.c_int32), _DP, C.c_int32]),
    "fem_set_materials": (C.c_int, [_VP, C.POINTER(FemMaterial), C.c_int32, _VP, _VP]),
    "fem_set_bc": (C.c_int, [_VP, _VP, _VP, _VP]),
    "fem_apply_bc": (C.c_int, [_VP]),
    "fem_set_displacement": (C.c_int, [_VP, _VP]),
    "fem_get_displacement": (C.c_int, [_VP, _VP]),
    "fem_reference_quantities": (C.c_int, [_VP, _VP, _VP]),
    "fem_compute_stress": (C.c_int, [_VP, _VP, _VP, _VP]),
    "fem_element_forces": (C.c_int, [_VP, _VP, _VP, _VP, _DP]),
    "fem_tangent_matvec": (C.c_int, [_VP, _VP, _VP]),
    "fem_nodal_mises": (C.c_int, [_VP, _VP, _VP, C.c_int32]),
    "fem_pcg": (C.c_int, [_VP, C.c_int32, _VP, _VP, C.c_double, C.c_int32,
                          C.POINTER(C.c_int32), _DP]),
    "fem_newton_solve": (C.c_int, [_VP, C.POINTER(FemSolveParams), C.POINTER(FemSolveResult)]),
    "fem_default_solve_params": (None, [C.POINTER(FemSolveParams)]),
    "fem_profile_kernels": (C.c_int, [_VP, C.c_int32, _DP]),
    "fem_dot_f64_noalloc": (C.c_int, [_VP, _VP, C.c_int64, _VP, _VP]),
    "fem_commit_history": (C.c_int, [_VP]),
    "fem_reset_history": (C.c_int, [_VP]),
    "fem_get_history": (C.c_int, [_VP, _VP, _VP]),
}

_lib = None


def load() -> C.CDLL:
    """Load the in-tree library once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m simul_b200.build` "
            "(the FEM path has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error(ctx=None) -> str:
    msg = load().fem_last_error(ctx)
    return msg.decode() if msg else ""
