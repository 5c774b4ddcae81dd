"""B200 drop-in for the reference's FEM static-solve API (TET4).

Mirrors, name for name, the pieces of ``backend/fea/fem`` a caller touches:

* ``FEMesh``        ``core/mesh.py:18-492`` (TET4 meshes)
* materials         ``material/{linear_elastic,neo_hookean,mooney_rivlin,
                    j2_plasticity,transverse_isotropic}.py`` — each with
                    ``compute_stress``, ``compute_nodal_forces``,
                    ``get_elasticity_tensor`` and ``is_linear``
                    (``material/base.py:16-63``)
* ``StaticSolver``  ``solver/static_solver.py:25-525`` — same constructor,
                    ``solve()`` signature and result dict.

Every numerical operation runs in ``libfemb200.so`` (hand-written sm_100a
kernels) through the C ABI in ``include/femb200.h``; torch tensors hold the
caller-visible device buffers.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import enum
from typing import Callable, Dict, Optional

import numpy as np
import torch

from . import _lib
from .validation import (FEAConvergenceError, FEAValidationError, logger,
                         validate_bc_indices, validate_elastic_constants, validate_positive)


class ElementType(enum.Enum):
    """Element types (core/element.py:12-33); the B200 path implements TET4
    (one Gauss point) and HEX8 (2 x 2 x 2 Gauss points)."""
    TET4 = "C3D4"
    HEX8 = "C3D8"


def _ptr(t: Optional[torch.Tensor]):
    """Device pointer of a tensor handed to the library.  The library works on
    its context's stream, which is torch's current stream only when that is
    a created (non-default) stream; otherwise (torch's default stream, or a
    context that owns its stream) nothing orders torch's pending writes to
    the tensor before the library reads it, so wait for them here.  The
    library synchronises its stream before returning outputs."""
    if t is None:
        return None
    if t.is_cuda:
        torch.cuda.current_stream(t.device).synchronize()
    return C.c_void_p(t.data_ptr())


def _check(rc: int, ctx=None, what: str = ""):
    if rc in (_lib.FEM_OK, _lib.FEM_NOT_CONVERGED):
        return rc
    msg = _lib.last_error(ctx)
    if rc == _lib.FEM_ERR_INVALID:
        raise FEAValidationError(f"{what}: {msg}")
    if rc == _lib.FEM_ERR_NAN:
        raise FEAConvergenceError(f"{what}: {msg}", reason="nan_divergence")
    raise RuntimeError(f"libfemb200 {what} failed ({rc}): {msg}")


def _require_cuda(device) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("simul_b200 needs a CUDA device (B200); there is no CPU fallback")
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else
                       (device if isinstance(device, int) else torch.device(device).index or 0))
    return dev


class FEMesh:
    """TET4 or HEX8 mesh on one GPU (core/mesh.py:18-86).

    Field tensors (torch, float64, on the mesh's device): ``u``, ``f``,
    ``f_ext``, ``fixed`` (int32 per DOF), ``fixed_value``; per Gauss point
    (point e * n_gauss + g, as the reference's ``gp_idx``) ``F``/``stress``
    after ``compute_stress``; per element ``material_id``.  HEX8 meshes solve
    with Jacobi or nodal block-Jacobi PCG (a two-level or learned request runs
    Jacobi-PCG and counts a fallback in ``coarse_info``).
    """

    def __init__(self, n_nodes: int, n_elements: int, element_type: ElementType = ElementType.TET4,
                 device=None, nodes_per_block: int = 0, own_stream: bool = False):
        et = getattr(element_type, "value", element_type)
        if et not in ("C3D4", "C3D8"):
            raise FEAValidationError(f"element type {element_type} is not supported by the B200 path "
                                     "(TET4, HEX8)", parameter="element_type", value=element_type)
        self.n_nodes = int(n_nodes)
        self.n_elements = int(n_elements)
        self.element_type = ElementType(et)
        self.dim = 3
        self.nodes_per_elem = 4 if et == "C3D4" else 8
        self.n_gauss = 1 if et == "C3D4" else 8
        self.device = _require_cuda(device)
        self.nodes_per_block = nodes_per_block
        # own_stream: the library creates a private non-blocking stream for this
        # mesh (batched solves); callers then synchronise torch work themselves
        self.own_stream = bool(own_stream)
        self._ctx = None
        self._bound_material = None
        z = lambda *s, dt=torch.float64: torch.zeros(*s, dtype=dt, device=self.device)
        self.u = z(self.n_nodes, 3)
        self.f = z(self.n_nodes, 3)
        self.f_ext = z(self.n_nodes, 3)
        self.fixed = z(self.n_nodes, 3, dt=torch.int32)
        self.fixed_value = z(self.n_nodes, 3)
        self.F = z(self.n_elements * self.n_gauss, 3, 3)
        self.stress = z(self.n_elements * self.n_gauss, 3, 3)
        self.material_id = np.zeros(self.n_elements, dtype=np.int32)
        self.X = None
        self.elements = None

    # ---- set-up (core/mesh.py:88-151) ----
    def initialize_from_numpy(self, nodes: np.ndarray, elements: np.ndarray,
                              material_ids: Optional[np.ndarray] = None):
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        elements = np.ascontiguousarray(elements, dtype=np.int32)
        if nodes.shape != (self.n_nodes, 3):
            raise FEAValidationError(f"nodes must be ({self.n_nodes}, 3), got {nodes.shape}",
                                     parameter="nodes")
        if elements.shape != (self.n_elements, self.nodes_per_elem):
            raise FEAValidationError(f"elements must be ({self.n_elements}, {self.nodes_per_elem}), "
                                     f"got {elements.shape}", parameter="elements")
        self.X = nodes
        self.elements = elements
        if material_ids is not None:
            self.material_id = np.asarray(material_ids, dtype=np.int32).copy()
        lib = _lib.load()
        with torch.cuda.device(self.device):
            stream = None if self.own_stream else torch.cuda.current_stream(self.device).cuda_stream
            desc = _lib.FemMeshDesc(self.n_nodes, self.n_elements,
                                    nodes.ctypes.data_as(C.POINTER(C.c_double)),
                                    elements.ctypes.data_as(C.POINTER(C.c_int32)),
                                    self.device.index, int(self.nodes_per_block), C.c_void_p(stream),
                                    self.nodes_per_elem)
            ctx = C.c_void_p()
            _check(lib.fem_ctx_create(C.byref(desc), C.byref(ctx)), None, "fem_ctx_create")
        self._ctx = ctx
        self.u.zero_()
        self.f.zero_()
        self.f_ext.zero_()
        self.fixed.zero_()
        self.fixed_value.zero_()
        self._bc_dirty = True

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and _lib is not None and getattr(_lib, "_lib", None) is not None:
            try:
                _lib._lib.fem_ctx_destroy(ctx)
            except Exception:
                pass
            self._ctx = None

    @property
    def ctx(self):
        if self._ctx is None:
            raise FEAValidationError("mesh not initialised: call initialize_from_numpy first")
        return self._ctx

    def info(self) -> dict:
        out = (C.c_int64 * 6)()
        _check(_lib.load().fem_ctx_info(self.ctx, out), self.ctx, "fem_ctx_info")
        return {"n_nodes": out[0], "n_elements": out[1], "n_blocks": out[2],
                "block_element_entries": out[3], "nodes_per_block": out[4], "device_bytes": out[5]}

    def stats(self) -> dict:
        out = (C.c_int64 * 18)()
        _check(_lib.load().fem_ctx_stats(self.ctx, out), self.ctx, "fem_ctx_stats")
        return {"launches": out[0], "cg_iterations": out[1], "residual_evals": out[2], "cg_graphs": out[3],
                "matvec_variant": _lib.MATVEC_VARIANTS.get(out[4], str(out[4])),
                "matvec_ns": {"fused": out[5], "two_phase": out[6], "element_block": out[10],
                              "warp_agg": out[16], "persistent": out[17]},
                "matvec_tuned": bool(out[7]),
                "whole_solve_graphs": out[8], "whole_solve_graph_available": bool(out[9]),
                "element_block_size": out[11],
                "element_block_ns": {256: out[12], 512: out[13], 768: out[14], 1024: out[15]}}

    def coarse_info(self) -> dict:
        out = (C.c_double * 10)()
        _check(_lib.load().fem_coarse_info(self.ctx, out), self.ctx, "fem_coarse_info")
        return {"cells": int(out[0]), "coarse_nodes": int(out[1]), "coarse_dofs": int(out[2]),
                "cell_edge": out[3], "assemblies": int(out[4]), "last_assembly_ms": out[5],
                "last_assembly_kernels_ms": out[6], "reuse": int(out[7]), "refreshes_kept": int(out[8]),
                "jacobi_fallbacks": int(out[9])}

    def set_coarse_options(self, cell=None, reuse=None, bf16=None, inverse=None, max_nodes=None):
        """Two-level preconditioner: lattice cell edge in mesh lengths, when
        the coarse operator is rebuilt (-1, the default: adaptive; 0: once per
        state - after a history reset, materials or constraint change; k >= 1:
        every k PCG solves), whether the coarse inverse is stored in BF16, and the
        precision its Cholesky, triangular inverse and product run in ("f64",
        "f32", or "tf32": FP32 Cholesky with the triangular inverse and the
        product on TF32 tensor-core tiles; the older names "potri" /
        "trsm_syrk" mean "f64", "trsm_syrk_f32" means "f32" and
        "trsm_syrk_tf32" means "tf32")."""
        lib = _lib.load()
        if max_nodes is not None:
            _check(lib.fem_set_option(self.ctx, _lib.FEM_OPT_COARSE_MAX_NODES, int(max_nodes)), self.ctx,
                   "fem_set_option")
        if inverse is not None:
            code = {"potri": 0, "trsm_syrk": 1, "trsm_syrk_f32": 2, "trsm_syrk_tf32": 3, "f64": 1, "f32": 2,
                    "tf32": 3}[inverse]
            _check(lib.fem_set_option(self.ctx, _lib.FEM_OPT_COARSE_INVERSE, code), self.ctx, "fem_set_option")
        if bf16 is not None:
            _check(lib.fem_set_option(self.ctx, _lib.FEM_OPT_COARSE_BF16, 1 if bf16 else 0), self.ctx,
                   "fem_set_option")
        if cell is not None:
            _check(lib.fem_set_option(self.ctx, _lib.FEM_OPT_COARSE_CELL, int(cell)), self.ctx, "fem_set_option")
        if reuse is not None:
            _check(lib.fem_set_option(self.ctx, _lib.FEM_OPT_COARSE_REUSE, int(reuse)), self.ctx, "fem_set_option")

    def set_fused_step(self, on: bool):
        """Runs the CG work after each matvec as one cooperative kernel (True)
        or as a chain of kernels (False, the default)."""
        _check(_lib.load().fem_set_option(self.ctx, _lib.FEM_OPT_FUSED_STEP, 1 if on else 0), self.ctx,
               "fem_set_option")

    def set_whole_solve_graph(self, on: bool):
        """One graph launch per PCG solve (True, the default) or fixed-size
        iteration graphs with a host check between them (False; kernel
        profilers cannot see inside the conditional graph)."""
        _check(_lib.load().fem_set_option(self.ctx, _lib.FEM_OPT_WHOLE_SOLVE_GRAPH, 1 if on else 0), self.ctx,
               "fem_set_option")

    def set_programmatic_launch(self, on: bool):
        """Programmatic dependent launches between the CG iteration's kernels
        inside the captured graphs (True, the default) or plain stream order."""
        _check(_lib.load().fem_set_option(self.ctx, _lib.FEM_OPT_PDL, 1 if on else 0), self.ctx, "fem_set_option")

    def set_direction_recurrence(self, on: bool):
        """Two-level PCG: form the search direction by recurrence inside the
        matvec's node gather (True, the default) or in its own kernel."""
        _check(_lib.load().fem_set_option(self.ctx, _lib.FEM_OPT_DIRECTION_RECURRENCE, 1 if on else 0), self.ctx,
               "fem_set_option")

    def set_block_smoother(self, on: bool):
        """Two-level preconditioner smoother: nodal 3x3 block inverse (True,
        the default) or the inverse of the diagonal (False)."""
        _check(_lib.load().fem_set_option(self.ctx, _lib.FEM_OPT_BLOCK_JACOBI, 1 if on else 0), self.ctx,
               "fem_set_option")

    def step_info(self) -> dict:
        out = (C.c_int64 * 6)()
        _check(_lib.load().fem_step_info(self.ctx, out), self.ctx, "fem_step_info")
        return {"available": bool(out[0]), "jacobi_graph_fused": bool(out[1]),
                "two_level_graph_fused": bool(out[2]), "restriction_warps_per_cell": int(out[3]),
                "jacobi_graph_pdl": bool(out[4]), "two_level_graph_pdl": bool(out[5])}

    def set_matvec_variant(self, variant, block_size=None):
        """Forces the tangent-matvec variant ("fused", "two_phase",
        "element_block", "warp_agg", "persistent") or restores the timed choice (None); ``block_size``
        fixes the element-block variant's elements per block (256, 512, 768
        or 1024; 0: timed; None: unchanged)."""
        code = {None: -1, "fused": 0, "two_phase": 1, "element_block": 2, "warp_agg": 3, "persistent": 4}[variant]
        lib = _lib.load()
        if block_size is not None:
            _check(lib.fem_set_option(self.ctx, _lib.FEM_OPT_EB_SIZE, int(block_size)), self.ctx, "fem_set_option")
        _check(lib.fem_set_option(self.ctx, _lib.FEM_OPT_MATVEC_VARIANT, code), self.ctx, "fem_set_option")

    def set_extrapolation(self, on: bool):
        """Load-step extrapolation: a solve that follows a converged one (u
        unchanged since) starts from the last end state plus its change of u;
        the convergence test is unchanged."""
        _check(_lib.load().fem_set_option(self.ctx, _lib.FEM_OPT_EXTRAPOLATE, 1 if on else 0), self.ctx,
               "fem_set_option")

    def set_residual_variant(self, variant: str):
        """TET4 FP64 residual: "two_phase" (default; one thread per element,
        then a node gather) or "fused" (node-block kernel)."""
        code = {"two_phase": 1, "fused": 0}[variant]
        _check(_lib.load().fem_set_option(self.ctx, _lib.FEM_OPT_RESIDUAL_TWO_PHASE, code), self.ctx,
               "fem_set_option")

    # ---- boundary conditions (core/mesh.py:321-399) ----
    def set_fixed_nodes(self, node_ids, values=None, dofs=None):
        node_ids = np.asarray(node_ids, dtype=np.int64)
        validate_bc_indices(node_ids, self.n_nodes, "고정 경계조건")
        fixed = np.zeros((self.n_nodes, 3), dtype=np.int32)
        if dofs is None:
            fixed[node_ids, :] = 1
        else:
            for d in dofs:
                fixed[node_ids, d] = 1
        vals = np.zeros((self.n_nodes, 3))
        if values is not None:
            vals[node_ids] = values
        self.fixed.copy_(torch.from_numpy(fixed))
        self.fixed_value.copy_(torch.from_numpy(vals))
        self._bc_dirty = True

    def set_fixed_dofs(self, dof_indices, values=None):
        dof_indices = np.asarray(dof_indices, dtype=np.int64)
        fixed = np.zeros((self.n_nodes, 3), dtype=np.int32)
        vals = np.zeros((self.n_nodes, 3))
        if dof_indices.size:
            if dof_indices.min() < 0 or dof_indices.max() >= 3 * self.n_nodes:
                raise FEAValidationError("DOF index out of range", parameter="dof_indices")
            fixed.reshape(-1)[dof_indices] = 1
            if values is not None:
                vals.reshape(-1)[dof_indices] = np.asarray(values, dtype=np.float64)
        self.fixed.copy_(torch.from_numpy(fixed))
        self.fixed_value.copy_(torch.from_numpy(vals))
        self._bc_dirty = True

    def set_nodal_forces(self, node_ids, forces):
        node_ids = np.asarray(node_ids, dtype=np.int64)
        validate_bc_indices(node_ids, self.n_nodes, "하중 경계조건")
        f = np.zeros((self.n_nodes, 3))
        f[node_ids] = forces
        self.f_ext.copy_(torch.from_numpy(f))
        self._bc_dirty = True

    def _push_bc(self):
        mask = (self.fixed != 0).to(torch.uint8).contiguous()
        if self.own_stream:
            torch.cuda.current_stream(self.device).synchronize()
        _check(_lib.load().fem_set_bc(self.ctx, _ptr(mask), _ptr(self.fixed_value.contiguous()),
                                      _ptr(self.f_ext.contiguous())), self.ctx, "fem_set_bc")
        self._bc_dirty = False

    def apply_boundary_conditions(self):
        """u = fixed_value on fixed DOFs (core/mesh.py:321-327)."""
        m = self.fixed != 0
        self.u[m] = self.fixed_value[m]

    # ---- kinematics / outputs ----
    def _reference_quantities(self):
        nq = self.n_elements * self.n_gauss
        dN = torch.empty(nq, self.nodes_per_elem, 3, dtype=torch.float64, device=self.device)
        vol = torch.empty(nq, dtype=torch.float64, device=self.device)
        _check(_lib.load().fem_reference_quantities(self.ctx, _ptr(dN), _ptr(vol)), self.ctx,
               "fem_reference_quantities")
        return dN, vol

    @property
    def dNdX(self) -> torch.Tensor:
        return self._reference_quantities()[0]

    @property
    def gauss_vol(self) -> torch.Tensor:
        return self._reference_quantities()[1]

    @property
    def elem_vol(self) -> torch.Tensor:
        """Element volume: the sum of its Gauss volumes (core/mesh.py:147-151)."""
        return self._reference_quantities()[1].view(self.n_elements, self.n_gauss).sum(dim=1)

    def compute_deformation_gradient(self):
        """F = I + sum_a u_a (x) dN_a/dX into ``self.F`` (core/mesh.py:293-313)."""
        mat = self._bound_material
        if mat is None:
            # F does not depend on the material; bind a placeholder so the kernel can run
            LinearElastic(1.0, 0.0)._bind(self)
        _check(_lib.load().fem_compute_stress(self.ctx, _ptr(self.u.contiguous()), _ptr(self.F), None),
               self.ctx, "fem_compute_stress")

    def get_displacements(self) -> np.ndarray:
        return self.u.detach().cpu().numpy()

    def get_nodal_forces(self) -> np.ndarray:
        return self.f.detach().cpu().numpy()

    def get_stress(self) -> np.ndarray:
        return self.stress.detach().cpu().numpy()

    def compute_mises_stress(self, average: bool = False):
        """Nodal von Mises stress into ``self.mises`` (core/mesh.py:459-492):
        per node the von Mises stress of every element on it, added in a
        fixed order.  The reference leaves the sum (its averaging step is a
        comment); ``average=True`` divides by the element count."""
        if self._bound_material is None:
            raise FEAValidationError("bind a material first (compute_stress / compute_nodal_forces)",
                                     parameter="material")
        if getattr(self, "mises", None) is None:
            self.mises = torch.zeros(self.n_nodes, dtype=torch.float64, device=self.device)
        _check(_lib.load().fem_nodal_mises(self.ctx, _ptr(self.u.contiguous()), _ptr(self.mises), int(average)),
               self.ctx, "fem_nodal_mises")


# ───────────────────────── materials ─────────────────────────

def _split_modulus(E):
    """Per-element modulus array -> (reference value, per-element scale or None)."""
    E = np.asarray(E, dtype=np.float64)
    if E.ndim == 0:
        return float(E), None
    ref = float(E.flat[0])
    return ref, (E / ref).astype(np.float32)


class MaterialBase:
    """material/base.py:16-63 — stress and forces run on the mesh's GPU."""

    dim = 3
    model = None

    @property
    def is_linear(self) -> bool:
        return False

    def _struct(self) -> _lib.FemMaterial:
        raise NotImplementedError

    def _scale(self):
        return None

    def _bind(self, mesh: FEMesh, table=None, elem_ids=None):
        if table is None:
            table, elem_ids = [self], None
        arr = (_lib.FemMaterial * len(table))(*[m._struct() for m in table])
        scales = [m._scale() for m in table]
        scale = None
        if any(s is not None for s in scales):
            scale = np.ones(mesh.n_elements, dtype=np.float32)
            ids = np.zeros(mesh.n_elements, dtype=np.int64) if elem_ids is None else elem_ids
            for k, s in enumerate(scales):
                if s is not None:
                    if s.shape != (mesh.n_elements,):
                        raise FEAValidationError("per-element modulus array must have one value per element",
                                                 parameter="E", value=s.shape)
                    sel = ids == k
                    scale[sel] = s[sel]
        ids8 = None if elem_ids is None else np.ascontiguousarray(elem_ids, dtype=np.uint8)
        _check(_lib.load().fem_set_materials(
            mesh.ctx, arr, len(table),
            ids8.ctypes.data_as(C.c_void_p) if ids8 is not None else None,
            scale.ctypes.data_as(C.c_void_p) if scale is not None else None), mesh.ctx, "fem_set_materials")
        mesh._bound_material = (tuple(id(m) for m in table),
                                None if elem_ids is None else bytes(ids8))

    def _ensure_bound(self, mesh: FEMesh):
        if mesh._bound_material is None or mesh._bound_material[0] != (id(self),):
            self._bind(mesh)

    def compute_stress(self, mesh: FEMesh):
        """Cauchy stress per Gauss point into ``mesh.stress`` (and F into ``mesh.F``)."""
        self._ensure_bound(mesh)
        _check(_lib.load().fem_compute_stress(mesh.ctx, _ptr(mesh.u.contiguous()), _ptr(mesh.F),
                                              _ptr(mesh.stress)), mesh.ctx, "fem_compute_stress")

    def compute_nodal_forces(self, mesh: FEMesh):
        """Negative internal force into ``mesh.f`` (deterministic gather, no atomics)."""
        self._ensure_bound(mesh)
        if mesh._bc_dirty:
            mesh._push_bc()
        _check(_lib.load().fem_element_forces(mesh.ctx, _ptr(mesh.u.contiguous()), _ptr(mesh.f),
                                              None, None), mesh.ctx, "fem_element_forces")

    def get_elasticity_tensor(self) -> np.ndarray:
        raise NotImplementedError


def _iso_C(lam, mu):
    C6 = np.zeros((6, 6))
    C6[:3, :3] = lam
    C6[[0, 1, 2], [0, 1, 2]] = lam + 2 * mu
    C6[[3, 4, 5], [3, 4, 5]] = mu
    return C6


class LinearElastic(MaterialBase):
    """material/linear_elastic.py:22-176 (3D)."""
    model = _lib.FEM_LINEAR_ELASTIC

    def __init__(self, youngs_modulus, poisson_ratio: float, dim: int = 3, plane_stress: bool = False):
        validate_elastic_constants(youngs_modulus, poisson_ratio, "LinearElastic")
        if dim != 3:
            raise FEAValidationError("the B200 path is 3D only", parameter="dim", value=dim)
        self.E, self._E_scale = _split_modulus(youngs_modulus)
        self.nu = float(poisson_ratio)
        self.mu = self.E / (2 * (1 + self.nu))
        self.lam = self.E * self.nu / ((1 + self.nu) * (1 - 2 * self.nu))

    @property
    def is_linear(self):
        return True

    def _scale(self):
        return self._E_scale

    def _struct(self):
        s = _lib.FemMaterial()
        s.model, s.E, s.nu = self.model, self.E, self.nu
        return s

    def get_elasticity_tensor(self):
        return _iso_C(self.lam, self.mu)

    def __repr__(self):
        return f"LinearElastic(E={self.E:.2e}, ν={self.nu:.3f})"


class NeoHookean(LinearElastic):
    """material/neo_hookean.py:31-226."""
    model = _lib.FEM_NEO_HOOKEAN

    def __init__(self, youngs_modulus, poisson_ratio: float, dim: int = 3):
        validate_elastic_constants(youngs_modulus, poisson_ratio, "NeoHookean")
        super().__init__(youngs_modulus, poisson_ratio, dim)

    @property
    def is_linear(self):
        return False

    def __repr__(self):
        return f"NeoHookean(E={self.E:.2e}, ν={self.nu:.3f})"


class J2Plasticity(LinearElastic):
    """material/j2_plasticity.py:33-526 (3D small strain, isotropic hardening).

    History is committed once per converged solve (``reset_state`` clears it).
    """
    model = _lib.FEM_J2

    def __init__(self, youngs_modulus, poisson_ratio: float, yield_stress: float,
                 hardening_modulus=0.0, dim: int = 3):
        validate_elastic_constants(youngs_modulus, poisson_ratio, "J2Plasticity")
        validate_positive(yield_stress, "yield_stress", "J2Plasticity")
        validate_positive(hardening_modulus, "hardening_modulus", "J2Plasticity", allow_zero=True)
        super().__init__(youngs_modulus, poisson_ratio, dim)
        self.sigma_y0 = float(yield_stress)
        H = np.asarray(hardening_modulus, dtype=np.float64)
        if H.ndim == 0:
            self.H = float(H) if self._E_scale is None else float(H) / 1.0
            if self._E_scale is not None and float(H) != 0.0:
                raise FEAValidationError("with per-element E give H per element too (H/E must be uniform)",
                                         parameter="hardening_modulus")
        else:
            scale = self._E_scale if self._E_scale is not None else np.ones(H.shape, np.float32)
            ratio = H / scale.astype(np.float64)
            if not np.allclose(ratio, ratio.flat[0], rtol=1e-6, atol=0):
                raise FEAValidationError("per-element H must be proportional to per-element E",
                                         parameter="hardening_modulus")
            self.H = float(ratio.flat[0])
        self.K_bulk = self.E / (3.0 * (1.0 - 2.0 * self.nu))
        self._mesh = None

    @property
    def is_linear(self):
        return False

    def _struct(self):
        s = super()._struct()
        s.sigma_y, s.H = self.sigma_y0, self.H
        return s

    def _bind(self, mesh, table=None, elem_ids=None):
        super()._bind(mesh, table, elem_ids)
        self._mesh = mesh

    def reset_state(self):
        if self._mesh is not None:
            _check(_lib.load().fem_reset_history(self._mesh.ctx), self._mesh.ctx, "fem_reset_history")

    def get_plastic_strain(self) -> np.ndarray:
        if self._mesh is None:
            return np.array([])
        nq = self._mesh.n_elements * self._mesh.n_gauss
        epe = torch.empty(nq, dtype=torch.float64, device=self._mesh.device)
        _check(_lib.load().fem_get_history(self._mesh.ctx, None, _ptr(epe)), self._mesh.ctx, "fem_get_history")
        return epe.cpu().numpy()

    def get_plastic_strain_tensor(self) -> np.ndarray:
        if self._mesh is None:
            return np.array([])
        nq = self._mesh.n_elements * self._mesh.n_gauss
        ep = torch.empty(nq, 3, 3, dtype=torch.float64, device=self._mesh.device)
        _check(_lib.load().fem_get_history(self._mesh.ctx, _ptr(ep), None), self._mesh.ctx, "fem_get_history")
        return ep.cpu().numpy()

    def get_yield_status(self) -> np.ndarray:
        epe = self.get_plastic_strain()
        return (epe > 1e-12).astype(np.float64) if epe.size else epe

    def __repr__(self):
        return f"J2Plasticity(E={self.E:.2e}, ν={self.nu:.3f}, σ_y={self.sigma_y0:.2e}, H={self.H:.2e})"


class MooneyRivlin(MaterialBase):
    """material/mooney_rivlin.py:36-294 (volumetric Cauchy term as the reference writes it)."""
    model = _lib.FEM_MOONEY_RIVLIN

    def __init__(self, C10: float, C01: float, D1: float, dim: int = 3):
        if C10 + C01 <= 0 or D1 < 0:
            raise FEAValidationError("Mooney-Rivlin needs C10 + C01 > 0 and D1 >= 0", parameter="C10")
        self.C10_val, self.C01_val, self.D1_val = float(C10), float(C01), float(D1)
        self.mu = 2.0 * (C10 + C01)
        self.nu = 0.3
        if D1 > 0:
            K = 2.0 / D1
            self.nu = (3.0 * K - self.mu) / (6.0 * K + self.mu)
        self.E = 2.0 * self.mu * (1.0 + self.nu)

    @staticmethod
    def from_engineering(E: float, nu: float, beta: float = 0.5, dim: int = 3) -> "MooneyRivlin":
        """mooney_rivlin.py:88-119."""
        mu = E / (2.0 * (1.0 + nu))
        K = E / (3.0 * (1.0 - 2.0 * nu))
        return MooneyRivlin((mu / 2.0) * beta, (mu / 2.0) * (1.0 - beta), 2.0 / K if K > 0 else 0.0)

    def _struct(self):
        s = _lib.FemMaterial()
        s.model = self.model
        s.C10, s.C01, s.D1 = self.C10_val, self.C01_val, self.D1_val
        return s

    def get_elasticity_tensor(self):
        mu = 2.0 * (self.C10_val + self.C01_val)
        lam = (2.0 / self.D1_val - 2.0 * mu / 3.0) if self.D1_val > 0 else mu
        return _iso_C(lam, mu)


class FibreReinforcedMooneyRivlin(MooneyRivlin):
    """Hyperelastic fibre-reinforced Mooney-Rivlin matrix (no reference counterpart).

    Adds, per fibre family a (at most two), the tension-only energy
    psi_f = fiber_E/8 (I4 - 1)^2 for I4 = |F a|^2 > 1, i.e. a fibre stress
    fiber_E * strain along a at small strain.
    """
    model = _lib.FEM_FIBRE_MOONEY_RIVLIN

    def __init__(self, C10, C01, D1, fiber_directions, fiber_E: float):
        super().__init__(C10, C01, D1)
        a = np.asarray(fiber_directions, dtype=np.float64).reshape(-1, 3)
        if a.shape[0] > 2:
            raise FEAValidationError("at most two fibre families", parameter="fiber_directions")
        self.fiber_a = a / np.linalg.norm(a, axis=1, keepdims=True)
        self.fiber_E = float(fiber_E)

    def _struct(self):
        s = super()._struct()
        s.n_fibers = self.fiber_a.shape[0]
        for k in range(self.fiber_a.shape[0]):
            for d in range(3):
                s.fiber_dir[k][d] = self.fiber_a[k, d]
        s.fiber_E = self.fiber_E
        return s


class TransverseIsotropic(MaterialBase):
    """material/transverse_isotropic.py:36-399 (3D, small strain)."""
    model = _lib.FEM_TRANSVERSE_ISOTROPIC

    def __init__(self, E1, E2, nu12, nu23, G12, fiber_direction=None, dim: int = 3,
                 rotation: str = "reference"):
        """``rotation="reference"`` keeps the reference's C_global = T^T C T with the
        stress Bond matrix T (transverse_isotropic.py:110-114), which is not a tensor
        rotation for fibres off the x axis; ``"tensor"`` uses T^-1 C T^-T."""
        if rotation not in ("reference", "tensor"):
            raise FEAValidationError("rotation must be 'reference' or 'tensor'", parameter="rotation")
        for name, v in (("E1", E1), ("E2", E2), ("G12", G12)):
            validate_positive(v, name, "TransverseIsotropic")
        self.E1, self.E2, self.nu12, self.nu23, self.G12 = E1, E2, nu12, nu23, G12
        self.G23 = E2 / (2.0 * (1.0 + nu23))
        self.nu21 = nu12 * E2 / E1
        f = np.array([1.0, 0.0, 0.0]) if fiber_direction is None else np.asarray(fiber_direction[:3], float)
        n = np.linalg.norm(f)
        if n < 1e-12:
            raise ValueError("fiber_direction의 노름이 0에 가깝습니다")
        self._fiber_dir = f / n
        self._C = self._material_C()
        self._T = self._bond_T()
        if rotation == "tensor":
            Ti = np.linalg.inv(self._T)
            self._C_global = Ti @ self._C @ Ti.T
        else:
            self._C_global = self._T.T @ self._C @ self._T

    def _material_C(self):
        """Inverse of the compliance of transverse_isotropic.py:124-173."""
        S = np.zeros((6, 6))
        S[0, 0] = 1.0 / self.E1
        S[1, 1] = S[2, 2] = 1.0 / self.E2
        S[0, 1] = S[1, 0] = S[0, 2] = S[2, 0] = -self.nu12 / self.E1
        S[1, 2] = S[2, 1] = -self.nu23 / self.E2
        S[3, 3] = 1.0 / self.G23
        S[4, 4] = S[5, 5] = 1.0 / self.G12
        return np.linalg.inv(S)

    def _bond_T(self):
        """Stress Bond matrix of transverse_isotropic.py:190-261."""
        f = self._fiber_dir
        if np.allclose(f, [1, 0, 0]):
            return np.eye(6)
        helper = np.array([0, 0, 1.0]) if abs(f[2]) < 0.9 else np.array([1, 0, 0.0])
        e2 = np.cross(f, helper)
        e2 /= np.linalg.norm(e2)
        a = np.array([f, e2, np.cross(f, e2)])
        T = np.zeros((6, 6))
        T[:3, :3] = a ** 2
        for i in range(3):
            T[i, 3:] = 2 * a[i, 1] * a[i, 2], 2 * a[i, 0] * a[i, 2], 2 * a[i, 0] * a[i, 1]
        for row, (p, q) in zip((3, 4, 5), ((1, 2), (0, 2), (0, 1))):
            T[row, :3] = a[p] * a[q]
            T[row, 3] = a[p, 1] * a[q, 2] + a[p, 2] * a[q, 1]
            T[row, 4] = a[p, 0] * a[q, 2] + a[p, 2] * a[q, 0]
            T[row, 5] = a[p, 0] * a[q, 1] + a[p, 1] * a[q, 0]
        return T

    @property
    def is_linear(self):
        return True

    def _struct(self):
        s = _lib.FemMaterial()
        s.model = self.model
        for k, v in enumerate(self._C_global.reshape(-1)):
            s.C_voigt[k] = v
        return s

    def get_elasticity_tensor(self):
        return self._C_global.copy()


# ───────────────────────── solver ─────────────────────────

_LS = {"reference": _lib.FEM_LS_REFERENCE, "guarded": _lib.FEM_LS_GUARDED, "none": _lib.FEM_LS_NONE}
_PC = {"jacobi": _lib.FEM_PRECOND_JACOBI, "none": _lib.FEM_PRECOND_NONE,
       "two_level": _lib.FEM_PRECOND_TWO_LEVEL, "learned": _lib.FEM_PRECOND_LEARNED}


class StaticSolver:
    """solver/static_solver.py:25-525 on the GPU.

    Same constructor and ``solve()`` contract.  Differences, by design:
    the tangent is the exact consistent tangent applied matrix-free and the
    linear solve is two-level PCG (Jacobi smoother plus a Galerkin coarse
    correction on a trilinear lattice; FP32 vectors, FP64 dots) instead of assembled
    initial-C + geometric stiffness with SuperLU; prescribed DOFs are held
    exactly instead of by a 1e30 penalty; per-element materials act on the
    residual too; J2 history is committed once per converged ``solve()``.
    ``linear_solver`` is accepted for compatibility (the B200 path always
    uses PCG).  Extra keyword options: ``line_search`` ("guarded",
    "reference", "none"), ``precond`` ("jacobi", "none", "two_level", "learned"),
    ``cg_max_iterations``, ``cg_rtol_min``, ``cg_rtol_max``.
    """

    def __init__(self, mesh: FEMesh, material: MaterialBase = None, use_newton: bool = True,
                 max_iterations: int = 50, tol: float = 1e-8,
                 materials: Optional[Dict[int, MaterialBase]] = None, linear_solver: str = "auto",
                 line_search: str = "guarded", precond: str = "two_level",
                 cg_max_iterations: int = 20000, cg_rtol_min: float = 1e-5, cg_rtol_max: float = 1e-1):
        self.mesh = mesh
        self.materials = materials
        if materials is not None and material is None:
            material = next(iter(materials.values()))
        if material is None:
            raise FEAValidationError("a material is required", parameter="material")
        self.material = material
        self.use_newton = use_newton and not material.is_linear
        self.max_iterations = int(max_iterations)
        self.tol = float(tol)
        self.linear_solver = linear_solver
        self.n_dof = mesh.n_nodes * 3
        self.dim = 3
        if line_search not in _LS or precond not in _PC:
            raise FEAValidationError("unknown line_search / precond option")
        self.line_search = line_search
        self.precond = precond
        self.cg_max_iterations = int(cg_max_iterations)
        self.cg_rtol_min = float(cg_rtol_min)
        self.cg_rtol_max = float(cg_rtol_max)
        self.last_result = None

    def _bind(self):
        if self.materials is not None:
            keys = sorted(self.materials)
            table = [self.materials[k] for k in keys]
            lut = {k: i for i, k in enumerate(keys)}
            ids = np.array([lut.get(int(m), -1) for m in self.mesh.material_id], dtype=np.int64)
            if np.any(ids < 0):
                raise FEAValidationError("mesh.material_id has ids without a material", parameter="materials")
            table[0]._bind(self.mesh, table, ids)
            for m in table:
                if isinstance(m, J2Plasticity):
                    m._mesh = self.mesh
        else:
            self.material._ensure_bound(self.mesh)
            if isinstance(self.material, J2Plasticity):
                self.material._mesh = self.mesh

    def solve(self, external_force_func: Optional[Callable] = None, verbose: bool = True,
              progress_callback: Optional[Callable] = None) -> Dict:
        if external_force_func is not None:
            external_force_func()
        mesh = self.mesh
        self._bind()
        mesh._push_bc()
        lib = _lib.load()
        _check(lib.fem_set_displacement(mesh.ctx, _ptr(mesh.u.contiguous())), mesh.ctx, "fem_set_displacement")
        prm = _lib.FemSolveParams()
        lib.fem_default_solve_params(C.byref(prm))
        prm.max_iterations = self.max_iterations
        prm.tol = self.tol
        prm.line_search = _LS[self.line_search]
        prm.precond = _PC[self.precond]
        prm.cg_max_iterations = self.cg_max_iterations
        prm.cg_rtol_min = self.cg_rtol_min
        prm.cg_rtol_max = self.cg_rtol_max
        prm.verbose = 0
        cb_keep = None
        if progress_callback is not None:
            def _cb(_user, it, res, rel):
                return 0 if progress_callback({"iteration": int(it), "max_iterations": self.max_iterations,
                                               "residual": float(res), "relative_residual": float(rel)}) is False else 1
            cb_keep = _lib.PROGRESS_FN(_cb)
            prm.progress = cb_keep
        res = _lib.FemSolveResult()
        rc = lib.fem_newton_solve(mesh.ctx, C.byref(prm), C.byref(res))
        _check(lib.fem_get_displacement(mesh.ctx, _ptr(mesh.u)), mesh.ctx, "fem_get_displacement")
        if rc == _lib.FEM_ERR_NAN:
            raise FEAConvergenceError(
                "Newton-Raphson에서 NaN/Inf 잔차가 발생했습니다. 하중이 너무 크거나 재료 상수가 부적절할 수 있습니다.",
                iterations=res.iterations, residual=float("inf"), reason="nan_divergence")
        _check(rc, mesh.ctx, "fem_newton_solve")
        self.last_result = res
        if verbose:
            logger.info("B200 Newton: converged=%s iterations=%d rel=%.3e cg=%d",
                        bool(res.converged), res.iterations, res.relative_residual, res.cg_iterations)
        out = {"converged": bool(res.converged), "iterations": int(res.iterations),
               "residual": float(res.residual), "relative_residual": float(res.relative_residual),
               "cg_iterations": int(res.cg_iterations), "residual_evals": int(res.residual_evals)}
        if res.cancelled:
            out["cancelled"] = True
        return out

    def get_mises_stress(self) -> np.ndarray:
        """Nodal von Mises stress (static_solver.py:512-515, summed as the
        reference leaves it)."""
        self._bind()
        self.mesh.compute_mises_stress()
        return self.mesh.mises.cpu().numpy()

    def get_total_energy(self) -> float:
        raise NotImplementedError("strain energy is not part of the B200 path")


# the reference-facing name of the GPU solver
B200StaticSolver = StaticSolver
