"""CPU oracle of the dynamic solver (test infrastructure only).

Restates backend/fea/fem/solver/dynamic_solver.py in FP64 NumPy / SciPy:
lumped mass (:87-115), stable step (:117-139), Newmark (:167-208) and central
difference (:210-243) steps.  ``formulation="reference"`` follows the
reference as written (its Newmark solve result is used as the acceleration
and scaled by beta dt^2 into u; its central-difference acceleration takes the
mesh's negative internal force with a minus sign); ``"consistent"`` is the
textbook form the GPU solver also offers.  Fixed DOFs are eliminated (the
reference adds a 1e30 penalty, which agrees to ~1e-30 relative).
"""
from __future__ import annotations

import numpy as np
from scipy import sparse
from scipy.sparse.linalg import spsolve

from . import fem_oracle as O


class DynamicOracle:
    def __init__(self, mesh: "O.Mesh", mat: "O.Material", E, nu, fixed_mask, density=1000.0, method="newmark",
                 dt=None, rayleigh_alpha=0.0, rayleigh_beta=0.0, formulation="reference"):
        self.mesh, self.mat = mesh, mat
        self.method, self.formulation = method, formulation
        n = mesh.X.shape[0]
        node_mass = np.zeros(n)
        npe = mesh.conn.shape[1]
        np.add.at(node_mass, np.asarray(mesh.conn, dtype=np.int64).reshape(-1),
                  np.repeat(density * mesh.elem_vol / float(npe), npe))
        self.M = np.repeat(node_mass, 3)
        self.K = O.reference_K_material(mesh, O.isotropic_voigt_C(E, nu)).tocsr()
        self.C = rayleigh_alpha * sparse.diags(self.M) + rayleigh_beta * self.K
        self.free = ~np.asarray(fixed_mask, dtype=bool).reshape(-1)
        if dt is None:
            h = np.mean(mesh.elem_vol) ** (1.0 / 3.0)
            c = np.sqrt(E * (1 - nu) / (density * (1 + nu) * (1 - 2 * nu)))
            dt = 0.8 * h / c
        self.dt = dt
        self.u = np.zeros(3 * n)
        self.v = np.zeros(3 * n)
        self.a = np.zeros(3 * n)
        self.gamma, self.beta = 0.5, 0.25

    def _solve(self, A, b):
        x = np.zeros_like(b)
        f = self.free
        x[f] = spsolve(A.tocsr()[f][:, f].tocsc(), b[f])
        return x

    def _bc(self):
        for w in (self.u, self.v, self.a):
            w[~self.free] = 0.0

    def step(self, f_ext):
        dt, g, b = self.dt, self.gamma, self.beta
        f_ext = np.asarray(f_ext, dtype=np.float64).reshape(-1)
        Ms = sparse.diags(self.M)
        if self.method == "newmark":
            u_pred = self.u + dt * self.v + (0.5 - b) * dt ** 2 * self.a
            v_pred = self.v + (1.0 - g) * dt * self.a
            f_eff = f_ext - self.K @ u_pred - self.C @ v_pred
            if self.formulation == "reference":
                K_eff = self.K + (g / (b * dt)) * self.C + (1.0 / (b * dt ** 2)) * Ms
            else:
                K_eff = Ms + g * dt * self.C + b * dt ** 2 * self.K
            acc = self._solve(K_eff, f_eff)
            self.a = acc
            self.u = u_pred + b * dt ** 2 * acc
            self.v = v_pred + g * dt * acc
        else:
            f_neg = O.internal_state(self.mesh, self.mat, self.u.reshape(-1, 3))[3].reshape(-1)
            f_damp = self.C @ self.v
            sgn = -1.0 if self.formulation == "reference" else 1.0
            self.a = (f_ext + sgn * f_neg - f_damp) / (self.M + 1e-30)
            self.v = self.v + self.a * dt
            self._bc()
            self.u = self.u + self.v * dt
            return
        self._bc()

    def natural_frequencies(self, n_modes=5):
        """dynamic_solver.py:372-413 with the assembled K (fixed DOFs removed)."""
        from scipy.sparse.linalg import eigsh
        f = self.free
        vals, _ = eigsh(self.K[f][:, f].tocsc(), k=n_modes, M=sparse.diags(self.M[f]), sigma=0, which="LM")
        return np.sort(np.sqrt(np.abs(vals)) / (2 * np.pi))

    def energy(self):
        """Kinetic + strain energy of the linear system, 1/2 v'Mv + 1/2 u'Ku."""
        return 0.5 * float(np.sum(self.M * self.v ** 2)) + 0.5 * float(self.u @ (self.K @ self.u))
