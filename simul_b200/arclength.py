"""Crisfield spherical arc-length solver on the B200 kernels.

Mirrors ``ArcLengthSolver`` of the reference
(backend/fea/fem/solver/arclength_solver.py:37-367): external load
lambda * f_ref, a tangent predictor whose sign follows the previous increment,
Newton correctors with the linearised (Ritto-Correa normal-update) constraint
dlambda = -Delta_u . du_r / (du_f . (Delta_u + du_r) + psi^2 Delta_lambda),
Bergan-Mollestad step adaptation dl *= sqrt(desired / iterations), halving on
failure, and the same result dictionary and equilibrium-path accessor.

The reference assembles an approximate tangent (small-strain C plus the
geometric stiffness) and factorises it; here every linear solve is the GPU's
matrix-free consistent tangent in PCG (``fem_pcg``, two-level by default),
and every residual is the FP64 fused element-force kernel.  Converged points
are equilibrium points of the same residual, so they lie on the same path;
the sequence of arc-length points can differ where the tangents differ.
Prescribed DOFs are held at zero, as in the reference.

The loop itself (``arc_length_path``) only needs two callables - the negative
internal force at a displacement, and a tangent solve - so the same code runs
on the GPU here and on the CPU oracle in the tests.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Dict, List, Optional

import numpy as np
import torch

from . import _lib
from . import fem as B
from .validation import FEAConvergenceError, logger


def arc_length_path(forces: Callable[[torch.Tensor], torch.Tensor],
                    solve: Callable[[torch.Tensor], torch.Tensor],
                    f_ref: torch.Tensor, free: torch.Tensor, *, arc_length: float, max_steps: int,
                    max_iterations: int, tol: float, psi: float, desired_iterations: int,
                    min_arc_length: float, max_arc_length: float, max_load_factor: float,
                    commit: Optional[Callable[[], None]] = None, verbose: bool = False,
                    progress_callback: Optional[Callable] = None) -> Dict:
    """The arc-length iteration (arclength_solver.py:119-348) over flat FP64
    vectors.  ``forces(u)`` returns the negative internal force at u and
    leaves the tangent at u for the next ``solve(b)``, which returns
    K_T^-1 b on the free DOFs (zero elsewhere); ``commit()`` (optional) makes
    a converged step's material history permanent."""
    f_ref_norm = float(torch.linalg.norm(f_ref))   # of the full vector, as the reference
    f_ref = f_ref.clone()
    f_ref[~free] = 0.0
    if f_ref_norm < 1e-30:
        raise FEAConvergenceError("the reference load vector is zero: apply a load first",
                                  iterations=0, residual=0.0, reason="zero_reference_load")
    zero = torch.zeros_like(f_ref)
    lam = 0.0
    u = zero.clone()
    dl = float(arc_length)
    loads: List[float] = [0.0]
    disps: List[torch.Tensor] = [zero.clone()]
    energies: List[float] = [0.0]
    prev_delta_u = zero.clone()
    n_completed = 0
    cancelled = False
    psi_sq = float(psi) ** 2

    for step in range(max_steps):
        # tangent displacement at the last converged state
        f_neg = forces(u)
        du_f = solve(f_ref)
        sign = 1.0 if step == 0 or float(torch.dot(du_f, prev_delta_u)) >= 0.0 else -1.0
        denom = float(torch.dot(du_f, du_f)) + psi_sq
        if denom < 1e-30:
            if verbose:
                logger.warning(f"  step {step}: zero tangent vector - stopping")
            break
        delta_lam = sign * dl / np.sqrt(denom)
        if lam + delta_lam > max_load_factor:
            delta_lam = max_load_factor - lam
        elif lam + delta_lam < -max_load_factor:
            delta_lam = -max_load_factor - lam
        u_trial = u + delta_lam * du_f
        lam_trial = lam + delta_lam

        converged = False
        n_iters = 0
        for it in range(max_iterations):
            n_iters = it + 1
            f_neg = forces(u_trial)
            residual = lam_trial * f_ref + f_neg
            residual[~free] = 0.0
            res_norm = float(torch.linalg.norm(residual))
            ref_force = abs(lam_trial) * f_ref_norm
            if ref_force < 1e-20:
                ref_force = f_ref_norm
            rel = res_norm / ref_force
            if verbose and it % 5 == 0:
                logger.info(f"  step {step}, iteration {it}: |R|={res_norm:.4e}, rel={rel:.4e}, "
                            f"lambda={lam_trial:.6f}")
            if rel < tol:
                converged = True
                break
            if not np.isfinite(res_norm):
                if verbose:
                    logger.warning(f"  step {step}: NaN/Inf residual")
                break
            du_f = solve(f_ref)
            du_r = solve(residual)
            Delta_u = u_trial - u
            Delta_lam = lam_trial - lam
            b_coeff = float(torch.dot(du_f, Delta_u + du_r)) + psi_sq * Delta_lam
            d_lam = 0.0 if abs(b_coeff) < 1e-30 else -float(torch.dot(Delta_u, du_r)) / b_coeff
            u_trial = u_trial + du_r + d_lam * du_f
            lam_trial = lam_trial + d_lam

        if converged:
            prev_delta_u = u_trial - u
            u = u_trial.clone()
            lam = lam_trial
            if commit is not None:
                commit()
            energy = -0.5 * float(torch.dot(u, f_neg))
            loads.append(float(lam))
            disps.append(u.clone())
            energies.append(float(energy))
            n_completed += 1
            if verbose:
                logger.info(f"  step {step} converged: lambda={lam:.6f}, |u|max={float(u.abs().max()):.4e}, "
                            f"{n_iters} iterations")
            if progress_callback is not None:
                go = progress_callback({"step": step, "max_steps": max_steps, "load_factor": float(lam),
                                        "max_load_factor": max_load_factor, "iterations": n_iters,
                                        "energy": float(energy)})
                if go is False:
                    cancelled = True
                    break
            if abs(lam) >= max_load_factor:
                break
            if n_iters > 0:
                dl = float(np.clip(dl * np.sqrt(desired_iterations / max(n_iters, 1)), min_arc_length,
                                   max_arc_length))
        else:
            if verbose:
                logger.warning(f"  step {step} did not converge in {max_iterations} iterations: "
                               f"arc length {dl:.4e} -> {dl * 0.5:.4e}")
            dl *= 0.5
            if dl < min_arc_length:
                if verbose:
                    logger.error("  minimum arc length reached - stopping")
                break
            forces(u)   # back to the last converged state

    return {"converged": n_completed > 0, "n_steps": n_completed, "cancelled": cancelled,
            "load_factors": loads, "displacements": disps, "energies": energies,
            "final_load_factor": loads[-1] if loads else 0.0}


class ArcLengthSolver:
    """Arc-length path following on one GPU mesh (arclength_solver.py:37-91).

    Same constructor arguments as the reference; ``linear_solver`` is
    accepted for the signature (every solve is matrix-free PCG here), and
    ``precond`` / ``cg_rtol`` choose the PCG.  Results hold displacements as
    numpy arrays (n_dof,) like the reference's.
    """

    def __init__(self, mesh: "B.FEMesh", material: "B.MaterialBase", arc_length: float = 0.1,
                 max_steps: int = 100, max_iterations: int = 30, tol: float = 1e-8, psi: float = 1.0,
                 desired_iterations: int = 5, min_arc_length: float = 1e-6, max_arc_length: float = 10.0,
                 max_load_factor: float = 1.0, linear_solver: str = "auto", precond: str = "two_level",
                 cg_rtol: float = 1e-7, cg_max_iterations: int = 20000):
        self.mesh = mesh
        self.material = material
        self.arc_length = arc_length
        self.max_steps = max_steps
        self.max_iterations = max_iterations
        self.tol = tol
        self.psi = psi
        self.desired_iterations = desired_iterations
        self.min_arc_length = min_arc_length
        self.max_arc_length = max_arc_length
        self.max_load_factor = max_load_factor
        self.linear_solver = linear_solver
        self.precond = precond
        self.cg_rtol = cg_rtol
        self.cg_max_iterations = cg_max_iterations
        self.dim = mesh.dim
        self.n_dof = mesh.n_nodes * mesh.dim
        self.load_history: List[float] = []
        self.displacement_history: List[np.ndarray] = []
        self.energy_history: List[float] = []
        self.cg_iterations = 0

    def _forces(self, u: torch.Tensor) -> torch.Tensor:
        self.mesh.u.copy_(u.view(-1, 3))
        self.material.compute_nodal_forces(self.mesh)
        return self.mesh.f.reshape(-1).clone()

    def _solve(self, b: torch.Tensor) -> torch.Tensor:
        lib = _lib.load()
        du = torch.zeros_like(b)
        it, rel = C.c_int32(), C.c_double()
        rc = lib.fem_pcg(self.mesh.ctx, B._PC[self.precond], B._ptr(b), B._ptr(du),
                         float(self.cg_rtol), int(self.cg_max_iterations), C.byref(it), C.byref(rel))
        if rc not in (_lib.FEM_OK, _lib.FEM_NOT_CONVERGED):
            B._check(rc, self.mesh.ctx, "fem_pcg")
        self.cg_iterations += it.value
        du[~self._free] = 0.0
        return du

    def _commit(self):
        B._check(_lib.load().fem_commit_history(self.mesh.ctx), self.mesh.ctx, "fem_commit_history")

    def solve(self, f_ref: Optional[np.ndarray] = None, verbose: bool = True,
              progress_callback: Optional[Callable] = None) -> Dict:
        """Trace lambda from 0 to max_load_factor (arclength_solver.py:94-348)."""
        mesh = self.mesh
        dev = mesh.device
        if f_ref is not None:
            fr = torch.as_tensor(np.asarray(f_ref, dtype=np.float64).reshape(-1), device=dev)
        else:
            fr = mesh.f_ext.reshape(-1).clone()
        self._free = (mesh.fixed.reshape(-1) == 0)
        self.material._ensure_bound(mesh)
        if mesh._bc_dirty:
            mesh._push_bc()
        if verbose:
            logger.info(f"arc-length solver: dl0={self.arc_length:.4e}, psi={self.psi}, "
                        f"lambda_max={self.max_load_factor}, at most {self.max_steps} steps")
        commit = self._commit if isinstance(self.material, B.J2Plasticity) else None
        res = arc_length_path(self._forces, self._solve, fr, self._free, arc_length=self.arc_length,
                              max_steps=self.max_steps, max_iterations=self.max_iterations, tol=self.tol,
                              psi=self.psi, desired_iterations=self.desired_iterations,
                              min_arc_length=self.min_arc_length, max_arc_length=self.max_arc_length,
                              max_load_factor=self.max_load_factor, commit=commit, verbose=verbose,
                              progress_callback=progress_callback)
        self.load_history = list(res["load_factors"])
        self.displacement_history = [d.cpu().numpy() for d in res["displacements"]]
        self.energy_history = list(res["energies"])
        mesh.u.copy_(res["displacements"][-1].view(-1, 3))
        out = dict(res)
        out["displacements"] = [d.copy() for d in self.displacement_history]
        out["cg_iterations"] = self.cg_iterations
        return out

    def get_equilibrium_path(self, node_id: int, dof: int = 0) -> tuple:
        """(displacements, load factors) of one DOF along the path
        (arclength_solver.py:484-504)."""
        k = node_id * self.dim + dof
        return (np.array([u[k] for u in self.displacement_history]), np.array(self.load_history))
