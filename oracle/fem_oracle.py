"""FP64 CPU oracle for the TET4 / HEX8 FEM static-solve path (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs may
import it.  The shipped solver (``simul_b200``) never routes through it.

It restates, in NumPy FP64, the arithmetic of the reference's FEM hot path
(monostylegc/simul, ``backend/fea/fem``) for 4-node tetrahedra (one Gauss
point) and 8-node hexahedra (2 x 2 x 2 Gauss points, ``core/mesh.py:182-200,
240-260``; every per-point array is ordered e * 8 + g as the reference's
``gp_idx``):

* reference quantities       ``core/mesh.py:123-151`` (+ ``:153-291`` for TET4)
* deformation gradient       ``core/mesh.py:293-313``
* Dirichlet application      ``core/mesh.py:321-327``
* Neo-Hookean stress/forces  ``material/neo_hookean.py:99-190``
* Mooney-Rivlin              ``material/mooney_rivlin.py:150-250`` (quirk Q4 kept)
* J2 radial return           ``material/j2_plasticity.py:186-249, 366-393``
* transverse isotropic       ``material/transverse_isotropic.py:116-324, 366-393``
* linear elastic             ``material/linear_elastic.py:102-173``
* reference Newton           ``solver/static_solver.py:135-265, 399-510``
* reference tangent          ``solver/assembly.py:92-287``

Two Newton drivers are provided:

``reference_newton``   the reference algorithm as written (initial-C + geometric
                       tangent, 1e30 penalty BCs, direct ``spsolve``, 5-step
                       backtracking, J2 history updated in place on every stress
                       call).  The reference's ILU-CG branch raises ``TypeError``
                       under its pinned SciPy (``cg(tol=)`` was removed) and falls
                       back to ``spsolve`` (``static_solver.py:444, 458-460``), so
                       the restatement calls ``spsolve`` directly.
``consistent_newton``  the same residual with the exact consistent tangent,
                       prescribed DOFs held exactly, per-element moduli honoured
                       and J2 history committed once per converged solve
                       ("fixed" quirks).  This is the FP64 oracle the GPU solver
                       is compared against.

Parity status: PARTIALLY PINNED.  The reference (Python 3.13 + Taichi 1.7.4)
cannot run in this image, and the reference ships no golden vectors.  The
restatement is pinned against every known-answer identity the reference's own
tests hold for this path (unit-tet volume, sum dN = 0, F = I at u = 0, J2
elastic == linear elastic at rtol 1e-10, von Mises cap, transverse-isotropic
isotropic limit at rtol 1e-8, energy balance); everything beyond those
identities (1e-5 / 1e-6 parity) is pinned only by this FP64 restatement.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, Optional

import numpy as np
import scipy.sparse as sp
from scipy.sparse.linalg import spsolve

# dN/dxi for the 4-node tetrahedron, constant (core/mesh.py:226-231).
DN_DXI_TET4 = np.array([[-1.0, -1.0, -1.0],
                        [1.0, 0.0, 0.0],
                        [0.0, 1.0, 0.0],
                        [0.0, 0.0, 1.0]])
TET4_WEIGHT = 1.0 / 6.0  # one-point rule at (1/4, 1/4, 1/4), core/mesh.py:166-168
J_FLOOR = 1e-8           # J_safe clamp, material/neo_hookean.py:119, :176-180
# HEX8 natural node coordinates (core/element.py:297-315); the 2x2x2 Gauss
# points carry the same sign pattern in the same order (core/mesh.py:182-200),
# at the reference's rounded 1/sqrt(3) and weight 1.
HEX8_SIGNS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                       [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)
HEX8_GP = 0.5773502691896257


def hex8_dN_dxi(xi):
    """dN_a/d(xi, eta, zeta) at one natural point (core/mesh.py:240-260), (8,3)."""
    s = HEX8_SIGNS
    f = 1.0 + s * np.asarray(xi, dtype=np.float64)[None, :]
    out = np.empty((8, 3))
    out[:, 0] = 0.125 * s[:, 0] * f[:, 1] * f[:, 2]
    out[:, 1] = 0.125 * f[:, 0] * s[:, 1] * f[:, 2]
    out[:, 2] = 0.125 * f[:, 0] * f[:, 1] * s[:, 2]
    return out


def hex8_N(xi):
    """Trilinear shape functions at one natural point, (8,)."""
    return 0.125 * np.prod(1.0 + HEX8_SIGNS * np.asarray(xi, dtype=np.float64)[None, :], axis=1)
PENALTY = 1e30           # solver/static_solver.py:501


class OracleConvergenceError(RuntimeError):
    """NaN/Inf residual, restating static_solver.py:174-182."""

    def __init__(self, msg, iterations=0, reason="nan_divergence"):
        super().__init__(msg)
        self.iterations = iterations
        self.reason = reason


# ─────────────────────────── geometry / kinematics ───────────────────────────

def reference_quantities(X: np.ndarray, conn: np.ndarray):
    """dN/dX and Gauss volumes — core/mesh.py:123-151.  TET4: (Ne,4,3) and
    (Ne,); HEX8: (Ne*8,8,3) and (Ne*8,), point e * 8 + g.

    J = sum_a X_a (x) dN_a/dxi, dNdX = dNdxi . J^-1, vol = w |det J|.
    """
    Xe = X[conn]                                       # (Ne,npe,3)
    if conn.shape[1] == 8:
        dN, vol = [], []
        for g in range(8):
            d = hex8_dN_dxi(HEX8_GP * HEX8_SIGNS[g])
            J = np.einsum("eai,aj->eij", Xe, d)
            dN.append(np.einsum("aj,ejk->eak", d, np.linalg.inv(J)))
            vol.append(np.abs(np.linalg.det(J)))
        return (np.stack(dN, axis=1).reshape(-1, 8, 3), np.stack(vol, axis=1).reshape(-1))
    J = np.einsum("eai,aj->eij", Xe, DN_DXI_TET4)
    detJ = np.linalg.det(J)
    Jinv = np.linalg.inv(J)
    dNdX = np.einsum("aj,ejk->eak", DN_DXI_TET4, Jinv)
    vol = TET4_WEIGHT * np.abs(detJ)
    return dNdX, vol


def deformation_gradient(u: np.ndarray, conn: np.ndarray, dNdX: np.ndarray):
    """F = I + sum_a u_a (x) dN_a/dX — core/mesh.py:293-313."""
    ue = u[conn]                                       # (Ne,4,3)
    return np.eye(3)[None] + np.einsum("eai,eaj->eij", ue, dNdX)


def _inv_T(F):
    return np.transpose(np.linalg.inv(F), (0, 2, 1))


# ─────────────────────────── materials ───────────────────────────

def lame(E, nu):
    """mu, lambda as in neo_hookean.py:57-58 / linear_elastic.py:51-59."""
    E = np.asarray(E, dtype=np.float64)
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return mu, lam


def isotropic_voigt_C(E, nu):
    """Isotropic 6x6 Voigt C (neo_hookean.py:70-89, linear_elastic.py:72-100)."""
    mu, lam = lame(E, nu)
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[[0, 1, 2], [0, 1, 2]] = lam + 2 * mu
    C[[3, 4, 5], [3, 4, 5]] = mu
    return C


def ti_material_C(E1, E2, nu12, nu23, G12):
    """Material-frame 6x6 stiffness of the transverse-isotropic model.

    Inverse of the compliance built in transverse_isotropic.py:124-173
    (axis 1 = fibre; Voigt [11, 22, 33, 23, 13, 12], engineering shear).
    """
    G23 = E2 / (2.0 * (1.0 + nu23))
    S = np.zeros((6, 6))
    S[0, 0] = 1.0 / E1
    S[1, 1] = S[2, 2] = 1.0 / E2
    S[0, 1] = S[1, 0] = S[0, 2] = S[2, 0] = -nu12 / E1
    S[1, 2] = S[2, 1] = -nu23 / E2
    S[3, 3] = 1.0 / G23
    S[4, 4] = S[5, 5] = 1.0 / G12
    return np.linalg.inv(S)


def ti_bond_T(fiber_direction):
    """6x6 Bond stress-rotation matrix, transverse_isotropic.py:190-261."""
    f = np.asarray(fiber_direction, dtype=np.float64)
    f = f / np.linalg.norm(f)
    if np.allclose(f, [1.0, 0.0, 0.0]):
        return np.eye(6)
    helper = np.array([0.0, 0.0, 1.0]) if abs(f[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
    e2 = np.cross(f, helper)
    e2 /= np.linalg.norm(e2)
    e3 = np.cross(f, e2)
    a = np.array([f, e2, e3])
    T = np.zeros((6, 6))
    T[:3, :3] = a ** 2
    # shear columns (Voigt 23, 13, 12) of the normal rows
    for i in range(3):
        T[i, 3] = 2 * a[i, 1] * a[i, 2]
        T[i, 4] = 2 * a[i, 0] * a[i, 2]
        T[i, 5] = 2 * a[i, 0] * a[i, 1]
    # shear rows: pairs (1,2) -> row 3, (0,2) -> row 4, (0,1) -> row 5
    for row, (p, q) in zip((3, 4, 5), ((1, 2), (0, 2), (0, 1))):
        T[row, 0] = a[p, 0] * a[q, 0]
        T[row, 1] = a[p, 1] * a[q, 1]
        T[row, 2] = a[p, 2] * a[q, 2]
        T[row, 3] = a[p, 1] * a[q, 2] + a[p, 2] * a[q, 1]
        T[row, 4] = a[p, 0] * a[q, 2] + a[p, 2] * a[q, 0]
        T[row, 5] = a[p, 0] * a[q, 1] + a[p, 1] * a[q, 0]
    return T


def ti_global_C(E1, E2, nu12, nu23, G12, fiber_direction=None, rotation="reference"):
    """Global Voigt stiffness of the transverse-isotropic model.

    ``rotation="reference"``: C_global = T^T C_mat T with T the stress Bond
    matrix, exactly as transverse_isotropic.py:110-114 writes it.  That is not
    a tensor rotation (an isotropic C changes under it) — reference quirk Q10.
    ``rotation="tensor"``: C_global = T^-1 C_mat T^-T, the proper rotation.
    """
    C = ti_material_C(E1, E2, nu12, nu23, G12)
    T = np.eye(6) if fiber_direction is None else ti_bond_T(fiber_direction)
    if rotation == "tensor":
        Ti = np.linalg.inv(T)
        return Ti @ C @ Ti.T
    return T.T @ C @ T


def voigt_strain(eps):
    """[e11, e22, e33, 2e23, 2e13, 2e12] (transverse_isotropic.py:308-311)."""
    return np.stack([eps[:, 0, 0], eps[:, 1, 1], eps[:, 2, 2],
                     2 * eps[:, 1, 2], 2 * eps[:, 0, 2], 2 * eps[:, 0, 1]], axis=1)


def voigt_to_tensor(s):
    """Voigt [11,22,33,23,13,12] -> symmetric 3x3 (transverse_isotropic.py:316-320)."""
    out = np.empty((s.shape[0], 3, 3))
    out[:, 0, 0], out[:, 1, 1], out[:, 2, 2] = s[:, 0], s[:, 1], s[:, 2]
    out[:, 1, 2] = out[:, 2, 1] = s[:, 3]
    out[:, 0, 2] = out[:, 2, 0] = s[:, 4]
    out[:, 0, 1] = out[:, 1, 0] = s[:, 5]
    return out


@dataclass
class Material:
    """Per-element constitutive description used by the oracle.

    ``model`` is one of ``neo_hookean``, ``mooney_rivlin``, ``j2``,
    ``linear_elastic``, ``transverse_isotropic``, ``ti_hyper`` (the
    hyperelastic fibre-reinforced Mooney-Rivlin matrix, which the reference
    does not have).  Scalars or per-element arrays are accepted for every
    parameter.
    """
    model: str
    E: object = None
    nu: float = 0.3
    C10: object = None
    C01: object = None
    D1: object = None
    sigma_y: object = None
    H: object = None
    C_voigt: Optional[np.ndarray] = None   # transverse_isotropic: 6x6 global C
    fiber_a: Optional[np.ndarray] = None   # ti_hyper: unit fibre dirs (2,3)
    fiber_E: object = None                 # ti_hyper: fibre stiffness

    def elasticity_tensor(self):
        """Initial Voigt C used by the reference tangent (get_elasticity_tensor)."""
        if self.model in ("neo_hookean", "linear_elastic", "j2"):
            return isotropic_voigt_C(np.mean(self.E) if np.ndim(self.E) else self.E, self.nu)
        if self.model == "transverse_isotropic":
            return self.C_voigt
        if self.model in ("mooney_rivlin", "ti_hyper"):
            # mooney_rivlin.py:130-148: mu = 2(C10+C01), lam = K - 2mu/3
            mu = 2.0 * (self.C10 + self.C01)
            lam = (2.0 / self.D1 - 2.0 * mu / 3.0) if self.D1 > 0 else mu
            C = np.zeros((6, 6))
            C[:3, :3] = lam
            C[[0, 1, 2], [0, 1, 2]] = lam + 2 * mu
            C[[3, 4, 5], [3, 4, 5]] = mu
            return C
        raise ValueError(self.model)

    @property
    def small_strain(self):
        return self.model in ("linear_elastic", "j2", "transverse_isotropic")


@dataclass
class MixedMaterial:
    """Per-element choice among several Materials: element e uses
    ``parts[ids[e]]`` (the reference's ``materials={id: material}`` with
    ``material_id`` per element, static_solver.py:32-71; there every id's
    residual uses the first material's tangent, quirk Q3 — here each element
    uses its own).  Per-element array parameters of a part are indexed by the
    global element number."""
    parts: list
    ids: np.ndarray

    model = "mixed"
    small_strain = False


def _subset(mat: Material, sel, ne):
    """The Material restricted to elements ``sel`` (array parameters sliced)."""
    kw = {}
    for name in ("E", "nu", "C10", "C01", "D1", "sigma_y", "H", "fiber_E"):
        v = getattr(mat, name)
        kw[name] = v[sel] if (v is not None and np.ndim(v) == 1 and np.size(v) == ne) else v
    return Material(mat.model, C_voigt=mat.C_voigt, fiber_a=mat.fiber_a, **kw)


@dataclass
class J2State:
    """J2 history per Gauss point (j2_plasticity.py:103-123)."""
    ep: np.ndarray      # (Ne,3,3) plastic strain
    epe: np.ndarray     # (Ne,) equivalent plastic strain

    @staticmethod
    def zeros(ne):
        return J2State(np.zeros((ne, 3, 3)), np.zeros(ne))

    def copy(self):
        return J2State(self.ep.copy(), self.epe.copy())


def j2_return_map(F, ep, epe, E, nu, sigma_y, H):
    """3D radial return, j2_plasticity.py:186-249 (small strain, Q6).

    Returns sigma, ep_new, epe_new and the consistent-tangent data
    (n, theta, gamma2, plastic mask).
    """
    mu, lam = lame(E, nu)
    mu = np.broadcast_to(mu, (F.shape[0],))
    lam = np.broadcast_to(lam, (F.shape[0],))
    H = np.broadcast_to(np.asarray(H, dtype=np.float64), (F.shape[0],))
    sy = np.broadcast_to(np.asarray(sigma_y, dtype=np.float64), (F.shape[0],))
    I = np.eye(3)[None]
    eps = 0.5 * (F + np.transpose(F, (0, 2, 1))) - I
    ee = eps - ep
    tr = np.trace(ee, axis1=1, axis2=2)
    s_tr = lam[:, None, None] * tr[:, None, None] * I + 2.0 * mu[:, None, None] * ee
    p = np.trace(s_tr, axis1=1, axis2=2) / 3.0
    s = s_tr - p[:, None, None] * I
    snorm = np.sqrt(np.maximum(np.einsum("eij,eij->e", s, s), 1e-30))
    q = math.sqrt(1.5) * snorm
    f = q - (sy + H * epe)
    plastic = f > 0.0
    dg = np.where(plastic, f / (3.0 * mu + H), 0.0)
    n = s / snorm[:, None, None]
    ep_new = ep + (math.sqrt(1.5) * dg)[:, None, None] * n
    epe_new = epe + dg
    factor = np.where(plastic, 1.0 - 3.0 * mu * dg / q, 1.0)
    sigma = np.where(plastic[:, None, None],
                     p[:, None, None] * I + factor[:, None, None] * s, s_tr)
    theta = factor
    gamma2 = np.where(plastic, 6.0 * mu * mu * (1.0 / (3.0 * mu + H) - dg / q), 0.0)
    return sigma, ep_new, epe_new, (n, theta, gamma2, plastic)


def _mixed_cauchy(mat: MixedMaterial, F, j2_state):
    ne = F.shape[0]
    sig = np.zeros((ne, 3, 3))
    st = j2_state if j2_state is not None else J2State.zeros(ne)
    new = st.copy()
    n = np.zeros((ne, 3, 3))
    theta = np.ones(ne)
    gamma2 = np.zeros(ne)
    plastic = np.zeros(ne, dtype=bool)
    has_j2 = False
    for k, part in enumerate(mat.parts):
        m = np.asarray(mat.ids) == k
        if not np.any(m):
            continue
        sub = _subset(part, m, ne)
        if part.model == "j2":
            s, (stk, tk) = cauchy_stress(sub, F[m], J2State(st.ep[m], st.epe[m]))
            new.ep[m], new.epe[m] = stk.ep, stk.epe
            n[m], theta[m], gamma2[m], plastic[m] = tk
            has_j2 = True
        else:
            s, _ = cauchy_stress(sub, F[m])
        sig[m] = s
    return sig, ((new, (n, theta, gamma2, plastic)) if has_j2 else None)


def cauchy_stress(mat: Material, F, j2_state: Optional[J2State] = None):
    """Cauchy stress per element.  Returns (sigma, aux)."""
    if isinstance(mat, MixedMaterial):
        return _mixed_cauchy(mat, F, j2_state)
    I = np.eye(3)[None]
    if mat.model == "neo_hookean":               # neo_hookean.py:99-129
        mu, lam = lame(mat.E, mat.nu)
        mu = np.broadcast_to(mu, (F.shape[0],))[:, None, None]
        lam = np.broadcast_to(lam, (F.shape[0],))[:, None, None]
        J = np.linalg.det(F)
        Js = np.maximum(J, J_FLOOR)
        B = F @ np.transpose(F, (0, 2, 1))
        return (mu * (B - I) + lam * np.log(Js)[:, None, None] * I) / Js[:, None, None], None
    if mat.model in ("mooney_rivlin", "ti_hyper"):  # mooney_rivlin.py:150-190
        J = np.linalg.det(F)
        Js = np.maximum(J, J_FLOOR)
        B = F @ np.transpose(F, (0, 2, 1))
        I1 = np.trace(B, axis1=1, axis2=2)
        sig = (2.0 / Js)[:, None, None] * ((mat.C10 + mat.C01 * I1)[:, None, None] * B - mat.C01 * (B @ B))
        if mat.D1 > 1e-20:
            sig = sig + ((2.0 * Js / mat.D1) * (Js - 1.0))[:, None, None] * I
        if mat.model == "ti_hyper":
            sig = sig + _fiber_cauchy(mat, F, Js)
        return sig, None
    eps = 0.5 * (F + np.transpose(F, (0, 2, 1))) - I
    if mat.model == "linear_elastic":            # linear_elastic.py:102-128
        mu, lam = lame(mat.E, mat.nu)
        mu = np.broadcast_to(mu, (F.shape[0],))[:, None, None]
        lam = np.broadcast_to(lam, (F.shape[0],))[:, None, None]
        tr = np.trace(eps, axis1=1, axis2=2)[:, None, None]
        return lam * tr * I + 2.0 * mu * eps, None
    if mat.model == "transverse_isotropic":      # transverse_isotropic.py:291-324
        return voigt_to_tensor(voigt_strain(eps) @ mat.C_voigt.T), None
    if mat.model == "j2":
        st = j2_state if j2_state is not None else J2State.zeros(F.shape[0])
        sig, ep_new, epe_new, tang = j2_return_map(F, st.ep, st.epe, mat.E, mat.nu,
                                                    mat.sigma_y, mat.H)
        return sig, (J2State(ep_new, epe_new), tang)
    raise ValueError(mat.model)


def _fiber_terms(mat, F):
    """Fibre family data for ``ti_hyper``: a (k,3), Fa (Ne,k,3), I4 (Ne,k)."""
    a = np.asarray(mat.fiber_a, dtype=np.float64).reshape(-1, 3)
    Fa = np.einsum("eij,kj->eki", F, a)
    I4 = np.einsum("eki,eki->ek", Fa, Fa)
    return a, Fa, I4


def _fiber_first_pk(mat, F):
    """Tension-only fibres: psi_f = (E_f/8)(I4-1)^2 for I4>1, P_f = E_f/2 (I4-1) (Fa)(x)a."""
    a, Fa, I4 = _fiber_terms(mat, F)
    c = np.where(I4 > 1.0, 0.5 * mat.fiber_E * (I4 - 1.0), 0.0)
    return np.einsum("ek,eki,kj->eij", c, Fa, a)


def _fiber_cauchy(mat, F, Js):
    P = _fiber_first_pk(mat, F)
    return (P @ np.transpose(F, (0, 2, 1))) / Js[:, None, None]


def first_piola(mat: Material, F, sigma):
    """Stress measure the force kernels contract with dN.

    Large strain (neo_hookean.py:169-180): P = J_safe sigma F^-T.
    Small strain (linear_elastic.py:142-173, j2_plasticity.py:366-393): sigma.
    """
    if isinstance(mat, MixedMaterial):
        out = np.zeros_like(sigma)
        for k, part in enumerate(mat.parts):
            m = np.asarray(mat.ids) == k
            if np.any(m):
                out[m] = first_piola(_subset(part, m, F.shape[0]), F[m], sigma[m])
        return out
    if mat.small_strain:
        return sigma
    Js = np.maximum(np.linalg.det(F), J_FLOOR)
    return Js[:, None, None] * sigma @ _inv_T(F)


def element_forces(P, dNdX, vol):
    """Per-element slot forces f_a = -P . dN_a . vol, (Ne,4,3)."""
    return -np.einsum("eij,eaj,e->eai", P, dNdX, vol)


def scatter_forces(fe, conn, n_nodes):
    """Nodal accumulation of the (negative) internal force — the reference's
    ``ti.atomic_add(f[node], f_a)`` (e.g. neo_hookean.py:190)."""
    f = np.zeros((n_nodes, 3))
    np.add.at(f, conn.reshape(-1), fe.reshape(-1, 3))
    return f


# ─────────────────────────── consistent tangents ───────────────────────────

def dP_directional(mat: Material, F, dF, tang=None):
    """Directional derivative dP[F](dF) of the stress measure used in the force."""
    if isinstance(mat, MixedMaterial):
        out = np.zeros_like(dF)
        for k, part in enumerate(mat.parts):
            m = np.asarray(mat.ids) == k
            if not np.any(m):
                continue
            tk = None if (tang is None or part.model != "j2") else tuple(t[m] for t in tang)
            out[m] = dP_directional(_subset(part, m, F.shape[0]), F[m], dF[m], tk)
        return out
    I = np.eye(3)[None]
    Ft = np.transpose(F, (0, 2, 1))
    if mat.model == "neo_hookean":
        mu, lam = lame(mat.E, mat.nu)
        mu = np.broadcast_to(mu, (F.shape[0],))[:, None, None]
        lam = np.broadcast_to(lam, (F.shape[0],))[:, None, None]
        Finv = np.linalg.inv(F)
        FiT = np.transpose(Finv, (0, 2, 1))
        lnJ = np.log(np.maximum(np.linalg.det(F), J_FLOOR))[:, None, None]
        G = Finv @ dF
        trG = np.trace(G, axis1=1, axis2=2)[:, None, None]
        return mu * dF + (mu - lam * lnJ) * np.transpose(G @ Finv, (0, 2, 1)) + lam * trG * FiT
    if mat.model in ("mooney_rivlin", "ti_hyper"):
        C10, C01, D1 = mat.C10, mat.C01, mat.D1
        B = F @ Ft
        I1 = np.trace(B, axis1=1, axis2=2)[:, None, None]
        FdF = np.einsum("eij,eij->e", F, dF)[:, None, None]
        out = 2.0 * (C10 + C01 * I1) * dF + 4.0 * C01 * FdF * F
        out = out - 2.0 * C01 * (dF @ Ft @ F + F @ np.transpose(dF, (0, 2, 1)) @ F + B @ dF)
        if D1 > 1e-20:
            J = np.linalg.det(F)
            Js = np.maximum(J, J_FLOOR)
            Finv = np.linalg.inv(F)
            FiT = np.transpose(Finv, (0, 2, 1))
            G = Finv @ dF
            trG = np.trace(G, axis1=1, axis2=2)
            g = Js ** 2 * (Js - 1.0)
            dg = (3.0 * Js ** 2 - 2.0 * Js) * Js * trG
            out = out + (2.0 / D1) * (dg[:, None, None] * FiT
                                      - g[:, None, None] * np.transpose(G @ Finv, (0, 2, 1)))
        if mat.model == "ti_hyper":
            a, Fa, I4 = _fiber_terms(mat, F)
            dFa = np.einsum("eij,kj->eki", dF, a)
            on = I4 > 1.0
            c = np.where(on, 0.5 * mat.fiber_E * (I4 - 1.0), 0.0)
            dc = np.where(on, mat.fiber_E * np.einsum("eki,eki->ek", Fa, dFa), 0.0)
            out = out + np.einsum("ek,eki,kj->eij", dc, Fa, a) + np.einsum("ek,eki,kj->eij", c, dFa, a)
        return out
    deps = 0.5 * (dF + np.transpose(dF, (0, 2, 1)))
    if mat.model == "linear_elastic":
        mu, lam = lame(mat.E, mat.nu)
        mu = np.broadcast_to(mu, (F.shape[0],))[:, None, None]
        lam = np.broadcast_to(lam, (F.shape[0],))[:, None, None]
        return lam * np.trace(deps, axis1=1, axis2=2)[:, None, None] * I + 2.0 * mu * deps
    if mat.model == "transverse_isotropic":
        return voigt_to_tensor(voigt_strain(deps) @ mat.C_voigt.T)
    if mat.model == "j2":
        n, theta, gamma2, _ = tang
        mu, lam = lame(mat.E, mat.nu)
        mu = np.broadcast_to(mu, (F.shape[0],))
        lam = np.broadcast_to(lam, (F.shape[0],))
        K = lam + 2.0 * mu / 3.0
        tr = np.trace(deps, axis1=1, axis2=2)
        dev = deps - (tr / 3.0)[:, None, None] * I
        nd = np.einsum("eij,eij->e", n, deps)
        return ((K * tr)[:, None, None] * I + (2.0 * mu * theta)[:, None, None] * dev
                - (gamma2 * nd)[:, None, None] * n)
    raise ValueError(mat.model)


def tangent_A(mat, F, tang=None):
    """A[e,i,j,k,l] = dP_ij/dF_kl assembled from 9 directional derivatives."""
    ne = F.shape[0]
    A = np.zeros((ne, 3, 3, 3, 3))
    for k in range(3):
        for l in range(3):
            dF = np.zeros((ne, 3, 3))
            dF[:, k, l] = 1.0
            A[:, :, :, k, l] = dP_directional(mat, F, dF, tang)
    return A


def element_stiffness(A, dNdX, vol):
    """K_e[(a,i),(b,k)] = sum_jl dN_a,j A_ijkl dN_b,l vol, (Ne, 3 npe, 3 npe)."""
    Ke = np.einsum("eaj,eijkl,ebl,e->eaibk", dNdX, A, dNdX, vol)
    nd = 3 * dNdX.shape[1]
    return Ke.reshape(-1, nd, nd)


def assemble(Ke, conn, n_nodes):
    nd = Ke.shape[1]
    dofs = (conn[:, :, None] * 3 + np.arange(3)[None, None, :]).reshape(-1, nd)
    rows = np.repeat(dofs, nd, axis=1).ravel()
    cols = np.tile(dofs, (1, nd)).ravel()
    return sp.coo_matrix((Ke.reshape(-1), (rows, cols)), shape=(3 * n_nodes, 3 * n_nodes)).tocsr()


def solve_tangent(mat, F, tang, mesh, rhs, fixed_mask):
    """Direct FP64 solve of K_ff x_f = rhs_f (x = 0 on fixed DOFs): the exact
    answer the GPU PCG paths approximate."""
    K = assemble(element_stiffness(tangent_A(mesh.qmat(mat), F, tang), mesh.dNdX, mesh.vol),
                 np.asarray(mesh.qconn, dtype=np.int64), mesh.X.shape[0])
    free = ~np.asarray(fixed_mask, dtype=bool).reshape(-1)
    x = np.zeros(K.shape[0])
    x[free] = spsolve(K[free][:, free].tocsc(), np.asarray(rhs, dtype=np.float64).reshape(-1)[free])
    return x.reshape(-1, 3)


def tangent_matvec(mat, F, tang, dNdX, vol, conn, p):
    """Matrix-free y = K_T p, p (Nn,3): the operator the GPU matvec applies."""
    dF = np.einsum("eai,eaj->eij", p[conn], dNdX)
    dP = dP_directional(mat, F, dF, tang)
    fe = np.einsum("eij,eaj,e->eai", dP, dNdX, vol)
    return scatter_forces(fe, conn, p.shape[0])


# ─────────────────────────── mesh container ───────────────────────────

@dataclass
class Mesh:
    X: np.ndarray
    conn: np.ndarray
    dNdX: np.ndarray = field(init=False)
    vol: np.ndarray = field(init=False)

    def __post_init__(self):
        self.X = np.asarray(self.X, dtype=np.float64)
        self.conn = np.asarray(self.conn, dtype=np.int64)
        if self.conn.shape[1] not in (4, 8):
            raise ValueError(f"elements must have 4 (TET4) or 8 (HEX8) nodes, got {self.conn.shape}")
        self.dNdX, self.vol = reference_quantities(self.X, self.conn)
        self.ngp = 1 if self.conn.shape[1] == 4 else 8
        # connectivity per integration point (point q = e * ngp + g)
        self.qconn = self.conn if self.ngp == 1 else np.repeat(self.conn, self.ngp, axis=0)

    @property
    def n_nodes(self):
        return self.X.shape[0]

    @property
    def n_elements(self):
        return self.conn.shape[0]

    @property
    def n_points(self):
        """Integration points (the rows of F, stress and the J2 history)."""
        return self.conn.shape[0] * self.ngp

    @property
    def elem_vol(self):
        return self.vol.reshape(-1, self.ngp).sum(axis=1)

    def qmat(self, mat):
        """``mat`` with per-element arrays repeated for every integration point."""
        if self.ngp == 1:
            return mat
        ne = self.n_elements
        if isinstance(mat, MixedMaterial):
            return MixedMaterial([self.qmat(p) for p in mat.parts], np.repeat(np.asarray(mat.ids), self.ngp))
        kw = {}
        for name in ("E", "nu", "C10", "C01", "D1", "sigma_y", "H", "fiber_E"):
            v = getattr(mat, name)
            kw[name] = np.repeat(v, self.ngp) if (v is not None and np.ndim(v) == 1 and np.size(v) == ne) else v
        return Material(mat.model, C_voigt=mat.C_voigt, fiber_a=mat.fiber_a, **kw)


def internal_state(mesh: Mesh, mat: Material, u, j2_state=None):
    """F, sigma, P (per integration point), negative internal force f (Nn,3), J2 aux."""
    mat = mesh.qmat(mat)
    F = deformation_gradient(u, mesh.qconn, mesh.dNdX)
    sigma, aux = cauchy_stress(mat, F, j2_state)
    P = first_piola(mat, F, sigma)
    f = scatter_forces(element_forces(P, mesh.dNdX, mesh.vol), mesh.qconn, mesh.n_nodes)
    return F, sigma, P, f, aux


def residual(mesh, mat, u, f_ext, fixed_mask, j2_state=None):
    """R = f_ext + f, fixed DOFs zeroed (static_solver.py:161-172)."""
    F, sigma, P, f, aux = internal_state(mesh, mat, u, j2_state)
    R = f_ext + f
    R[fixed_mask] = 0.0
    return R, F, sigma, aux


# ─────────────────────────── reference Newton (quirks as written) ───────────────────────────

def reference_K_material(mesh: Mesh, C):
    """assembly.py:92-169 — ke = vol B^T C B with B rows [xx,yy,zz,xy,yz,xz]."""
    d = mesh.dNdX
    ne, npe = d.shape[0], d.shape[1]
    B = np.zeros((ne, 6, 3 * npe))
    for a in range(npe):
        B[:, 0, 3 * a] = d[:, a, 0]
        B[:, 1, 3 * a + 1] = d[:, a, 1]
        B[:, 2, 3 * a + 2] = d[:, a, 2]
        B[:, 3, 3 * a] = d[:, a, 1]
        B[:, 3, 3 * a + 1] = d[:, a, 0]
        B[:, 4, 3 * a + 1] = d[:, a, 2]
        B[:, 4, 3 * a + 2] = d[:, a, 1]
        B[:, 5, 3 * a] = d[:, a, 2]
        B[:, 5, 3 * a + 2] = d[:, a, 0]
    Ke = np.einsum("e,evi,vw,ewj->eij", mesh.vol, B, C, B)
    return _assemble_filtered(Ke, mesh)


def reference_K_geometric(mesh: Mesh, sigma):
    """assembly.py:220-287 — K_geo[a*3+d, b*3+d] = vol dN_a^T sigma dN_b."""
    kg = np.einsum("e,eai,eij,ebj->eab", mesh.vol, mesh.dNdX, sigma, mesh.dNdX)
    nd = 3 * mesh.dNdX.shape[1]
    Ke = np.zeros((mesh.dNdX.shape[0], nd, nd))
    for dd in range(3):
        Ke[:, dd::3, dd::3] = kg
    return _assemble_filtered(Ke, mesh)


def _assemble_filtered(Ke, mesh):
    conn = getattr(mesh, "qconn", mesh.conn)
    nd = Ke.shape[1]
    dofs = (conn[:, :, None] * 3 + np.arange(3)[None, None, :]).reshape(-1, nd)
    rows = np.repeat(dofs, nd, axis=1).ravel()
    cols = np.tile(dofs, (1, nd)).ravel()
    vals = Ke.reshape(-1)
    m = np.abs(vals) > 1e-20
    n = 3 * mesh.n_nodes
    return sp.coo_matrix((vals[m], (rows[m], cols[m])), shape=(n, n))


def reference_newton(mesh: Mesh, mat: Material, f_ext, fixed_mask, fixed_vals, u0=None,
                     j2_state: Optional[J2State] = None, max_iterations=50, tol=1e-8,
                     materials_C: Optional[Dict[int, np.ndarray]] = None,
                     material_ids: Optional[np.ndarray] = None):
    """StaticSolver._solve_newton as written (static_solver.py:73-99, 135-265).

    fixed_mask/fixed_vals/f_ext are (Nn,3).  ``j2_state`` is mutated in place on
    every stress evaluation (quirk Q1).  Returns (u, info dict).
    """
    u = np.zeros((mesh.n_nodes, 3)) if u0 is None else u0.copy()
    u[fixed_mask] = fixed_vals[fixed_mask]            # apply_boundary_conditions, mesh.py:321-327
    fixed_dofs = np.where(fixed_mask.reshape(-1))[0]
    fext = f_ext.reshape(-1)

    qmat = mesh.qmat(mat)

    def eval_state(uu):
        F = deformation_gradient(uu, mesh.qconn, mesh.dNdX)
        sigma, aux = cauchy_stress(qmat, F, j2_state)
        if aux is not None:                           # Q1: in-place history update
            j2_state.ep[...] = aux[0].ep
            j2_state.epe[...] = aux[0].epe
        P = first_piola(qmat, F, sigma)
        f = scatter_forces(element_forces(P, mesh.dNdX, mesh.vol), mesh.qconn, mesh.n_nodes)
        return sigma, f.reshape(-1)

    ref = None
    res_norm = rel = float("nan")
    converged = False
    it = 0
    for it in range(max_iterations):
        sigma, fneg = eval_state(u)
        R = fext + fneg
        R[fixed_dofs] = 0.0
        res_norm = float(np.linalg.norm(R))
        if not np.isfinite(res_norm):
            raise OracleConvergenceError("NaN/Inf residual", iterations=it)
        if ref is None:
            ref = res_norm if res_norm > 1e-20 else 1.0
        rel = res_norm / ref
        if rel < tol:
            converged = True
            break
        if materials_C is not None:
            K = _multi_material_K(mesh, materials_C, material_ids)
        else:
            K = reference_K_material(mesh, mat.elasticity_tensor())
        K = (K + reference_K_geometric(mesh, sigma)).tocsr()
        # penalty BC (static_solver.py:479-510)
        diag = K.diagonal().copy()
        diag[fixed_dofs] += PENALTY
        K.setdiag(diag)
        rhs = R.copy()
        rhs[fixed_dofs] = PENALTY * fixed_vals.reshape(-1)[fixed_dofs]
        du = spsolve(K.tocsr(), rhs)
        alpha = 1.0
        u_cur = u.reshape(-1).copy()
        for _ls in range(5):                          # Q7: keep the last trial
            u = (u_cur + alpha * du).reshape(-1, 3)
            _, fneg2 = eval_state(u)
            r2 = fext + fneg2
            r2[fixed_dofs] = 0.0
            if np.linalg.norm(r2) < res_norm:
                break
            alpha *= 0.5
    return u, {"converged": converged, "iterations": it + 1,
               "residual": res_norm, "relative_residual": rel}


def _multi_material_K(mesh, C_map, material_ids):
    """Multi-material grouping of assembly.py:127-147 (C per material id)."""
    K = None
    for mid, C in C_map.items():
        sel = material_ids == mid
        if not np.any(sel):
            continue
        sub = Mesh.__new__(Mesh)
        qsel = np.repeat(sel, mesh.ngp)
        sub.X, sub.conn, sub.dNdX, sub.vol = mesh.X, mesh.conn[sel], mesh.dNdX[qsel], mesh.vol[qsel]
        sub.qconn = mesh.qconn[qsel]
        Kp = reference_K_material(sub, C)
        K = Kp if K is None else K + Kp
    return K


# ─────────────────────────── consistent-tangent Newton (FP64 oracle) ───────────────────────────

def consistent_newton(mesh: Mesh, mat: Material, f_ext, fixed_mask, fixed_vals, u0=None,
                      j2_state: Optional[J2State] = None, max_iterations=50, tol=1e-8,
                      line_search=True, commit=True, callback: Optional[Callable] = None,
                      predictor=True):
    """Exact Newton on the same residual, free-DOF direct solves ("fixed" quirks).

    Prescribed DOFs end at ``fixed_vals`` exactly.  With ``predictor`` the
    change of the prescribed values is carried by the first Newton step
    (K_ff du_f = R - K_fc du_c, then u += du): jumping only the boundary
    nodes instead leaves a one-element layer at large strain, which under J2
    yields and stalls Newton.  Convergence is measured, as in the reference
    (static_solver.py:159-218, quirk Q8), relative to the residual at the
    state the reference evaluates first: the previous u with the new
    prescribed values applied.  J2 return maps start from the committed
    ``j2_state``, which is committed once at convergence.  Returns (u, info).
    """
    u = np.zeros((mesh.n_nodes, 3)) if u0 is None else u0.copy()
    free = np.where(~fixed_mask.reshape(-1))[0]
    base = j2_state.copy() if j2_state is not None else None

    qmat = mesh.qmat(mat)

    def evaluate(uu):
        F = deformation_gradient(uu, mesh.qconn, mesh.dNdX)
        sigma, aux = cauchy_stress(qmat, F, base)
        P = first_piola(qmat, F, sigma)
        f = scatter_forces(element_forces(P, mesh.dNdX, mesh.vol), mesh.qconn, mesh.n_nodes)
        R = f_ext + f
        R[fixed_mask] = 0.0
        return R, F, aux

    def tangent(F, aux):
        tang = aux[1] if aux is not None else None
        return assemble(element_stiffness(tangent_A(qmat, F, tang), mesh.dNdX, mesh.vol),
                        mesh.qconn, mesh.n_nodes)

    dc = np.zeros_like(u)
    dc[fixed_mask] = fixed_vals[fixed_mask] - u[fixed_mask]
    it = 0
    if predictor and np.any(dc != 0.0):
        R_old, F, aux = evaluate(u)
        R_ref = evaluate(u + dc)[0]
        K = tangent(F, aux)
        rhs = R_old.reshape(-1) - K @ dc.reshape(-1)
        du = dc.reshape(-1).copy()
        du[free] += spsolve(K[free][:, free].tocsc(), rhs[free])
        u = u + du.reshape(-1, 3)
        res0 = float(np.linalg.norm(R_ref))
        it = 1
    else:
        u[fixed_mask] = fixed_vals[fixed_mask]
        res0 = None
    R, F, aux = evaluate(u)
    res_norm = float(np.linalg.norm(R))
    if res0 is None:
        res0 = res_norm
    ref = res0 if res0 > 1e-20 else 1.0
    rel = res_norm / ref
    converged = rel < tol
    history = [rel]
    while not converged and it < max_iterations:
        if not np.isfinite(res_norm):
            raise OracleConvergenceError("NaN/Inf residual", iterations=it)
        K = tangent(F, aux)
        du = np.zeros(3 * mesh.n_nodes)
        du[free] = spsolve(K[free][:, free].tocsc(), R.reshape(-1)[free])
        alpha = 1.0
        u_cur = u.copy()
        for _ls in range(5 if line_search else 1):
            u = u_cur + alpha * du.reshape(-1, 3)
            R2, F2, aux2 = evaluate(u)
            if np.linalg.norm(R2) < res_norm:
                break
            alpha *= 0.5
        R, F, aux = R2, F2, aux2
        res_norm = float(np.linalg.norm(R))
        rel = res_norm / ref
        history.append(rel)
        it += 1
        if callback is not None:
            callback(it, rel)
        converged = rel < tol
    if not np.isfinite(res_norm):
        raise OracleConvergenceError("NaN/Inf residual", iterations=it)
    if commit and j2_state is not None and aux is not None:
        j2_state.ep[...] = aux[0].ep
        j2_state.epe[...] = aux[0].epe
    return u, {"converged": bool(converged), "iterations": it, "residual": res_norm,
               "relative_residual": rel, "history": history}


def nodal_mises(mesh: Mesh, mat: Material, u, j2_state=None, average=False):
    """core/mesh.py:459-492: per node the von Mises stress of each element on
    it (of the element's Gauss-point mean stress), summed (the reference never
    divides; ``average`` divides by the element count)."""
    F, sigma, P, f, aux = internal_state(mesh, mat, u, j2_state)
    s = sigma.reshape(-1, mesh.ngp, 3, 3).sum(axis=1) / float(mesh.ngp)
    vm = np.sqrt(0.5 * ((s[:, 0, 0] - s[:, 1, 1]) ** 2 + (s[:, 1, 1] - s[:, 2, 2]) ** 2 +
                        (s[:, 2, 2] - s[:, 0, 0]) ** 2 +
                        6.0 * (s[:, 0, 1] ** 2 + s[:, 1, 2] ** 2 + s[:, 0, 2] ** 2)))
    conn = np.asarray(mesh.conn, dtype=np.int64)
    out = np.zeros(mesh.X.shape[0])
    np.add.at(out, conn.reshape(-1), np.repeat(vm, conn.shape[1]))
    if average:
        cnt = np.zeros(mesh.X.shape[0])
        np.add.at(cnt, conn.reshape(-1), 1.0)
        out = out / np.maximum(cnt, 1.0)
    return out


def strain_energy(mesh: Mesh, mat: Material, u):
    """Total strain energy for NH / LE (neo_hookean.py:193-226, energy_balance)."""
    F = deformation_gradient(u, mesh.qconn, mesh.dNdX)
    mat = mesh.qmat(mat)
    mu, lam = lame(mat.E, mat.nu)
    if mat.model == "neo_hookean":
        J = np.maximum(np.linalg.det(F), J_FLOOR)
        I1 = np.einsum("eij,eij->e", F, F)
        psi = 0.5 * mu * (I1 - 3.0) - mu * np.log(J) + 0.5 * lam * np.log(J) ** 2
    elif mat.model == "linear_elastic":
        eps = 0.5 * (F + np.transpose(F, (0, 2, 1))) - np.eye(3)[None]
        tr = np.trace(eps, axis1=1, axis2=2)
        psi = 0.5 * lam * tr ** 2 + mu * np.einsum("eij,eij->e", eps, eps)
    else:
        raise ValueError(mat.model)
    return float(np.sum(psi * mesh.vol))
