"""Batched solves of many independent meshes on one GPU (fem_batch_solve).

Each instance is an ordinary ``FEMesh`` + material created on its own CUDA
stream; ``solve_batch`` hands all contexts to the library, which runs every
instance's load steps (Newton + PCG, CUDA-graph-captured CG iterations) on a
pool of host workers so the instances' kernels overlap on the device.

No reference counterpart: the reference solves one mesh per ``solve()`` call
(backend/fea/fem/solver/static_solver.py:73-99).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Sequence

import numpy as np
import torch

from . import _lib
from . import fem as B


class BatchInstance:
    """A mesh + material on a private stream, with its loads pushed."""

    def __init__(self, X, conn, material, fixed_mask, fixed_vals=None, f_ext=None, device=0,
                 coarse_cell: int = 8, material_ids=None, coarse_bf16: bool = False, coarse_reuse=None):
        """``material`` is one material, or a dict {id: material} with
        ``material_ids`` giving each element's id (as StaticSolver's
        ``materials=``)."""
        # the library owns a non-blocking stream per instance; torch work on the
        # mesh's tensors is synchronised before every library call below
        self.mesh = B.FEMesh(X.shape[0], conn.shape[0], device=device, own_stream=True)
        self.mesh.initialize_from_numpy(X, conn, material_ids=material_ids)
        idx = np.where(np.asarray(fixed_mask).reshape(-1))[0]
        vals = None if fixed_vals is None else np.asarray(fixed_vals).reshape(-1)[idx]
        self.mesh.set_fixed_dofs(idx, vals)
        if f_ext is not None:
            self.mesh.set_nodal_forces(np.arange(X.shape[0]), f_ext)
        self.material = material
        self.mesh.set_coarse_options(cell=coarse_cell, bf16=coarse_bf16, reuse=coarse_reuse)
        torch.cuda.synchronize(self.mesh.device)
        if isinstance(material, dict):
            # binds the material table through a solver object (no solve)
            B.StaticSolver(self.mesh, materials=material)._bind()
        else:
            material.compute_nodal_forces(self.mesh)   # binds the material, pushes the loads
        torch.cuda.synchronize(self.mesh.device)
        self.mesh._push_bc()
        torch.cuda.synchronize(self.mesh.device)

    @property
    def ctx(self):
        return self.mesh.ctx

    def reset(self):
        """Back to rest: u = 0 and no plastic history."""
        lib = _lib.load()
        self.mesh.u.zero_()
        torch.cuda.synchronize(self.mesh.device)
        B._check(lib.fem_set_displacement(self.ctx, B._ptr(self.mesh.u)), self.ctx,
                 "fem_set_displacement")
        B._check(lib.fem_reset_history(self.ctx), self.ctx, "fem_reset_history")


def solve_batch(instances: Sequence[BatchInstance], load_steps: int = 10, precond: str = "two_level",
                tol: float = 1e-8, max_iterations: int = 50, n_threads: int = 0,
                line_search: str = "guarded") -> Dict:
    """Solves every instance from its current state through ``load_steps``
    load steps; returns per-instance results and host wall times."""
    lib = _lib.load()
    n = len(instances)
    ctxs = (C.c_void_p * n)(*[inst.ctx.value for inst in instances])
    prm = _lib.FemSolveParams()
    lib.fem_default_solve_params(C.byref(prm))
    prm.tol = tol
    prm.max_iterations = max_iterations
    prm.precond = B._PC[precond]
    prm.line_search = B._LS[line_search]
    res = (_lib.FemSolveResult * n)()
    status = (C.c_int32 * n)()
    wall = (C.c_double * n)()
    torch.cuda.synchronize()
    rc = lib.fem_batch_solve(ctxs, n, C.byref(prm), int(load_steps), res, status, wall, int(n_threads))
    if rc not in (_lib.FEM_OK, _lib.FEM_NOT_CONVERGED):
        bad = [i for i in range(n) if status[i] not in (_lib.FEM_OK, _lib.FEM_NOT_CONVERGED)]
        ctx = instances[bad[0]].ctx if bad else None
        B._check(rc, ctx, f"fem_batch_solve (instance {bad[0] if bad else '?'})")
    out: List[Dict] = []
    for i in range(n):
        out.append({"status": int(status[i]), "converged": bool(res[i].converged),
                    "newton_iterations": int(res[i].iterations), "cg_iterations": int(res[i].cg_iterations),
                    "relative_residual": float(res[i].relative_residual), "wall_ms": float(wall[i])})
    for inst in instances:
        B._check(lib.fem_get_displacement(inst.ctx, B._ptr(inst.mesh.u)), inst.ctx,
                 "fem_get_displacement")
    return {"instances": out}
