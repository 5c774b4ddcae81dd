"""Time-domain dynamics (Newmark-beta / central difference) on the B200 kernels.

Mirrors ``DynamicSolver`` of the reference
(backend/fea/fem/solver/dynamic_solver.py:21-413): row-sum lumped mass
(density x element volume / nodes per element, per node), Rayleigh damping C = alpha M +
beta K with K the stiffness at rest, the stable-step estimate
dt = 0.8 h / c, Newmark (gamma = 1/2, beta = 1/4) and central-difference
steps, the same ``step`` / ``solve`` / getter API.

Two formulations:
- ``"reference"`` (default) - the reference as written.  Its Newmark step
  solves (K + gamma/(beta dt) C + M/(beta dt^2)) da = f_ext - K u_pred - C
  v_pred and then uses da both as the acceleration and through
  u = u_pred + beta dt^2 da; its central-difference step forms
  a = (f_ext - f - C v) / M with the mesh's negative internal force f
  (dynamic_solver.py:167-243).
- ``"consistent"`` - textbook Newmark, (M + gamma dt C + beta dt^2 K) a =
  f_ext - C v_pred - K u_pred, and central difference with the internal
  force's physical sign, a = (f_ext + f - C v) / M.

K x is the matrix-free tangent at rest (``fem_tangent_matvec`` after an
element-force pass at u = 0; at rest every material's consistent tangent is
its small-strain stiffness, the reference's K).  The implicit solve is CG on
the free DOFs with the mass diagonal as preconditioner (the mass term
dominates at the stable step size); the explicit step's internal force is
the fused FP64 element-force kernel.  Fixed DOFs are held at zero, as in the
reference.  ``get_natural_frequencies`` runs ARPACK in shift-invert mode
with the GPU's PCG as the inverse.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np
import torch

from . import _lib
from . import fem as B


class DynamicSolver:
    def __init__(self, mesh: "B.FEMesh", material: "B.MaterialBase", density: float = 1000.0,
                 method: str = "newmark", dt: Optional[float] = None, rayleigh_alpha: float = 0.0,
                 rayleigh_beta: float = 0.0, linear_solver: str = "auto", formulation: str = "reference",
                 cg_rtol: float = 1e-7, cg_max_iterations: int = 2000):
        if method not in ("newmark", "central_diff"):
            raise B.FEAValidationError(f"unknown method {method}", parameter="method", value=method)
        if formulation not in ("reference", "consistent"):
            raise B.FEAValidationError(f"unknown formulation {formulation}", parameter="formulation",
                                       value=formulation)
        self.mesh = mesh
        self.material = material
        self.density = float(density)
        self.method = method
        self.dim = mesh.dim
        self.n_dof = mesh.n_nodes * mesh.dim
        self.linear_solver = linear_solver
        self.formulation = formulation
        self.rayleigh_alpha = float(rayleigh_alpha)
        self.rayleigh_beta = float(rayleigh_beta)
        self.cg_rtol = float(cg_rtol)
        self.cg_max_iterations = int(cg_max_iterations)
        self.cg_iterations = 0
        dev = mesh.device
        self.material._ensure_bound(mesh)
        if mesh._bc_dirty:
            mesh._push_bc()
        self.M_diag = self._compute_lumped_mass(self.density)
        self._free = (mesh.fixed.reshape(-1) == 0)
        self._tangent_at_rest = False
        if dt is None:
            dt = self._estimate_stable_dt()
        self.dt = float(dt)
        z = lambda: torch.zeros(self.n_dof, dtype=torch.float64, device=dev)
        self.u, self.v, self.a = z(), z(), z()
        self.time = 0.0
        self.step_count = 0
        self.gamma = 0.5
        self.beta = 0.25

    # ---- set-up (dynamic_solver.py:87-148) ----
    def _compute_lumped_mass(self, density: float) -> torch.Tensor:
        vol = self.mesh.elem_vol
        conn = torch.as_tensor(self.mesh.elements, dtype=torch.int64, device=self.mesh.device)
        node_mass = torch.zeros(self.mesh.n_nodes, dtype=torch.float64, device=self.mesh.device)
        npe = self.mesh.nodes_per_elem
        node_mass.index_add_(0, conn.reshape(-1), (density * vol / float(npe)).repeat_interleave(npe))
        return node_mass.repeat_interleave(3)

    def _estimate_stable_dt(self) -> float:
        h = float(self.mesh.elem_vol.mean()) ** (1.0 / 3.0)
        E = float(np.mean(self.material.E))
        nu = float(self.material.nu)
        c = np.sqrt(E * (1 - nu) / (self.density * (1 + nu) * (1 - 2 * nu)))
        return 0.8 * h / c

    def set_initial_velocity(self, v0: np.ndarray):
        self.v = torch.as_tensor(np.asarray(v0, dtype=np.float64).reshape(-1), device=self.mesh.device).clone()

    # ---- operators ----
    def _rest_tangent(self):
        if not self._tangent_at_rest:
            self.mesh.u.zero_()
            self.material.compute_nodal_forces(self.mesh)
            self._tangent_at_rest = True

    def _K(self, x: torch.Tensor) -> torch.Tensor:
        """K x with the stiffness at rest (free rows; fixed rows zero)."""
        self._rest_tangent()
        xf = x.view(-1, 3).to(torch.float32).contiguous()
        y = torch.empty_like(xf)
        B._check(_lib.load().fem_tangent_matvec(self.mesh.ctx, B._ptr(xf), B._ptr(y)),
                 self.mesh.ctx, "fem_tangent_matvec")
        return y.reshape(-1).to(torch.float64)

    def _Cv(self, v: torch.Tensor) -> torch.Tensor:
        out = self.rayleigh_alpha * self.M_diag * v
        if self.rayleigh_beta != 0.0:
            out = out + self.rayleigh_beta * self._K(v)
        return out

    def _solve(self, cK: float, cM: float, b: torch.Tensor) -> torch.Tensor:
        """(cK K + cM M) x = b on the free DOFs by CG, preconditioned by cM M."""
        free = self._free
        b = b.clone()
        b[~free] = 0.0
        x = torch.zeros_like(b)
        dinv = torch.where(free, 1.0 / (cM * self.M_diag), torch.zeros_like(b))
        r = b.clone()
        bn = float(torch.linalg.norm(b))
        if bn == 0.0:
            return x
        z = dinv * r
        p = z.clone()
        rz = float(torch.dot(r, z))
        for it in range(self.cg_max_iterations):
            q = cK * self._K(p) + cM * self.M_diag * p
            q[~free] = 0.0
            alpha = rz / float(torch.dot(p, q))
            x += alpha * p
            r -= alpha * q
            self.cg_iterations += 1
            if float(torch.linalg.norm(r)) <= self.cg_rtol * bn:
                break
            z = dinv * r
            rz_new = float(torch.dot(r, z))
            p = z + (rz_new / rz) * p
            rz = rz_new
        return x

    def _enforce_bc(self):
        free = self._free
        self.v[~free] = 0.0
        self.a[~free] = 0.0
        self.u[~free] = 0.0

    # ---- time stepping (dynamic_solver.py:150-243) ----
    def step(self, f_ext: Optional[np.ndarray] = None) -> Dict:
        if f_ext is None:
            f = self.mesh.f_ext.reshape(-1).clone()
        else:
            f = torch.as_tensor(np.asarray(f_ext, dtype=np.float64).reshape(-1), device=self.mesh.device)
        if self.method == "newmark":
            return self._step_newmark(f)
        return self._step_central_diff(f)

    def _step_newmark(self, f_ext: torch.Tensor) -> Dict:
        dt, g, b = self.dt, self.gamma, self.beta
        u_pred = self.u + dt * self.v + (0.5 - b) * dt ** 2 * self.a
        v_pred = self.v + (1.0 - g) * dt * self.a
        f_eff = f_ext - self._K(u_pred) - self._Cv(v_pred)
        a_R, b_R = self.rayleigh_alpha, self.rayleigh_beta
        if self.formulation == "reference":
            # K_eff = K + g/(b dt) C + 1/(b dt^2) M, the solution used as da
            cK = 1.0 + g / (b * dt) * b_R
            cM = 1.0 / (b * dt ** 2) + g / (b * dt) * a_R
            da = self._solve(cK, cM, f_eff)
            self.a = da
            self.u = u_pred + b * dt ** 2 * da
            self.v = v_pred + g * dt * da
        else:
            # (M + g dt C + b dt^2 K) a = f_ext - C v_pred - K u_pred
            cK = b * dt ** 2 + g * dt * b_R
            cM = 1.0 + g * dt * a_R
            acc = self._solve(cK, cM, f_eff)
            self.a = acc
            self.u = u_pred + b * dt ** 2 * acc
            self.v = v_pred + g * dt * acc
        self._enforce_bc()
        self.mesh.u.copy_(self.u.view(-1, 3))
        self.time += dt
        self.step_count += 1
        return {"kinetic_energy": self.get_kinetic_energy(), "time": self.time}

    def _step_central_diff(self, f_ext: torch.Tensor) -> Dict:
        dt = self.dt
        f_damp = self._Cv(self.v)          # before the force pass: K is the stiffness at rest
        self.mesh.u.copy_(self.u.view(-1, 3))
        self.material.compute_nodal_forces(self.mesh)
        self._tangent_at_rest = False
        f_neg = self.mesh.f.reshape(-1)
        if self.formulation == "reference":
            self.a = (f_ext - f_neg - f_damp) / (self.M_diag + 1e-30)
        else:
            self.a = (f_ext + f_neg - f_damp) / (self.M_diag + 1e-30)
        self.v = self.v + self.a * dt
        self._enforce_bc()
        self.u = self.u + self.v * dt
        self.mesh.u.copy_(self.u.view(-1, 3))
        self.time += dt
        self.step_count += 1
        return {"kinetic_energy": self.get_kinetic_energy(), "time": self.time}

    def solve(self, n_steps: int, f_ext: Optional[np.ndarray] = None, verbose: bool = True,
              print_interval: int = 100) -> Dict:
        """n_steps steps with a constant external force (dynamic_solver.py:320-353)."""
        if verbose:
            print(f"FEM dynamic solver: {self.method} ({self.formulation}), dt={self.dt:.2e}, n_steps={n_steps}")
        info: Dict = {}
        for i in range(n_steps):
            info = self.step(f_ext)
            if verbose and (i + 1) % print_interval == 0:
                print(f"Step {i + 1:6d}: t={info['time']:.4e}, KE={info['kinetic_energy']:.4e}, "
                      f"max_u={float(self.u.abs().max()):.4e}")
        return info

    def get_displacements(self) -> np.ndarray:
        return self.u.view(-1, 3).cpu().numpy()

    def get_velocities(self) -> np.ndarray:
        return self.v.view(-1, 3).cpu().numpy()

    def get_kinetic_energy(self) -> float:
        return 0.5 * float(torch.sum(self.M_diag * self.v ** 2))

    def get_natural_frequencies(self, n_modes: int = 5, precond: str = "two_level", rtol: float = 1e-9) -> np.ndarray:
        """Lowest natural frequencies [Hz] of K phi = omega^2 M phi on the free
        DOFs (dynamic_solver.py:372-413): ARPACK shift-invert at sigma = 0 as
        the reference, with K x the matrix-free stiffness at rest and K^-1 b
        a PCG solve of it on the GPU instead of a sparse factorisation."""
        from scipy import sparse
        from scipy.sparse.linalg import LinearOperator, eigsh
        free = self._free
        idx = torch.nonzero(free).reshape(-1)
        nf = int(idx.numel())
        n_modes = min(int(n_modes), max(nf - 2, 1))
        dev = self.mesh.device
        lib = _lib.load()
        self._rest_tangent()

        def full(xf):
            x = torch.zeros(self.n_dof, dtype=torch.float64, device=dev)
            x[idx] = torch.as_tensor(np.asarray(xf, dtype=np.float64).reshape(-1), device=dev)
            return x

        def k_op(xf):
            return self._K(full(xf))[idx].cpu().numpy()

        def k_inv(bf):
            b = full(bf)
            x = torch.zeros_like(b)
            it, rel = C.c_int32(), C.c_double()
            rc = lib.fem_pcg(self.mesh.ctx, B._PC[precond], B._ptr(b), B._ptr(x),
                             float(rtol), 20000, C.byref(it), C.byref(rel))
            if rc not in (_lib.FEM_OK, _lib.FEM_NOT_CONVERGED):
                B._check(rc, self.mesh.ctx, "fem_pcg")
            self.cg_iterations += it.value
            return x[idx].cpu().numpy()

        K = LinearOperator((nf, nf), matvec=k_op, dtype=np.float64)
        Kinv = LinearOperator((nf, nf), matvec=k_inv, dtype=np.float64)
        M = sparse.diags(self.M_diag[idx].cpu().numpy())
        vals = eigsh(K, k=n_modes, M=M, sigma=0, which="LM", OPinv=Kinv, return_eigenvectors=False)
        return np.sort(np.sqrt(np.abs(vals)) / (2 * np.pi))
