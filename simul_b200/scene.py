"""Staggered static contact between FEM bodies on the GPU.

Mirrors the static mode of the reference's ``Scene``
(``backend/fea/framework/scene.py:48-290, 559-632``) for FEM bodies, with
the node-to-node penalty and tied contact of ``framework/contact.py:13-273``:

- ``FEMBody`` plays the part of the FEM adapter
  (``framework/_adapters/fem_adapter.py:122-203``): a ``FEMesh`` with its
  material and ``StaticSolver``, the user loads and a contact-force buffer
  that ``solve()`` adds to them; every solve continues from the body's last
  displacement (the GPU Newton starts from it), so the contact iterations
  after the first are warm-started;
- ``Scene.solve(mode="static")`` runs the reference's loop: the bodies with
  fixed DOFs are solved alone, then every iteration computes the contact
  forces at the current positions (on the GPU, ``fem_contact_penalty`` /
  ``fem_contact_tied``), injects them, re-solves every body and stops when
  the total contact force changes by less than ``contact_tol`` (relative);
- contact parameters left unset are estimated as the reference does: the
  boundary is the nodes on the min / max planes of each axis, the gap
  tolerance 1.5 x the larger mesh spacing, the penalty E_avg / the smaller
  spacing.

Between FEM bodies in a static solve the reference's friction term is zero
(both velocities are zero, ``scene.py:534-537``), so friction coefficients
are accepted and change nothing here either.  The quasi-static and explicit
modes couple explicit particle bodies (peridynamics, SPG), which are not
part of this library.
"""
from __future__ import annotations

import ctypes as C
import enum
import time
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from .fem import FEMesh, StaticSolver
from .validation import FEAValidationError


class ContactType(enum.Enum):
    """framework/contact.py:13-16."""
    PENALTY = "penalty"
    TIED = "tied"


def _ptr(t: torch.Tensor):
    """A tensor handed to the contact kernels: torch's pending writes to it
    finish first (the kernels run on the library's stream)."""
    if t.is_cuda:
        torch.cuda.current_stream(t.device).synchronize()
    return C.c_void_p(t.data_ptr())


def _check(rc: int, what: str):
    if rc != _lib.FEM_OK:
        raise RuntimeError(f"{what} failed ({rc}): {_lib.last_error()}")


def boundary_nodes(X: np.ndarray) -> np.ndarray:
    """Nodes on the min / max plane of each axis, the tolerance half the
    smallest step between distinct coordinates (scene.py:185-206)."""
    out = set()
    for ax in range(X.shape[1]):
        c = X[:, ax]
        u = np.unique(np.round(c, decimals=10))
        tol = np.min(np.diff(u)) * 0.5 if len(u) > 1 else 1e-6
        out.update(np.where(np.abs(c - c.min()) < tol)[0])
        out.update(np.where(np.abs(c - c.max()) < tol)[0])
    return np.array(sorted(out), dtype=np.int64)


class FEMBody:
    """A FEM body of a Scene (the FEM adapter's role).

    ``mesh`` carries the constraints (``set_fixed_nodes`` / ``set_fixed_dofs``)
    and ``f_ext`` the user loads ((n, 3), or None); ``spacing`` is the mesh
    length the automatic contact parameters use (default: the median length
    of the elements' first edges); ``E`` the modulus for the automatic
    penalty (default: the material's ``E``).  ``solver_options`` go to
    ``StaticSolver``."""

    def __init__(self, mesh: FEMesh, material, f_ext: Optional[np.ndarray] = None, spacing: Optional[float] = None,
                 E: Optional[float] = None, **solver_options):
        self.mesh = mesh
        self.material = material
        self.solver = StaticSolver(mesh, material, **solver_options)
        dev = mesh.device
        self._user_f_ext = torch.zeros(mesh.n_nodes, 3, dtype=torch.float64, device=dev)
        if f_ext is not None:
            self._user_f_ext.copy_(torch.as_tensor(np.asarray(f_ext, dtype=np.float64)))
        self._contact_forces = torch.zeros_like(self._user_f_ext)
        self._X = torch.as_tensor(np.asarray(mesh.X, dtype=np.float64), device=dev)
        if spacing is None:
            el = np.asarray(mesh.elements)
            spacing = float(np.median(np.linalg.norm(mesh.X[el[:, 1]] - mesh.X[el[:, 0]], axis=1)))
        self.spacing = float(spacing)
        if E is None:
            E = getattr(material, "E", None)
            E = float(np.max(E)) if E is not None else 0.0
        self.E = float(E)
        self.last_result = None

    @property
    def has_fixed(self) -> bool:
        return bool((self.mesh.fixed != 0).any().item())

    def solve(self, verbose: bool = False) -> dict:
        """fem_adapter.py:156-172: user loads + contact forces, then a Newton
        solve from the current displacement."""
        self.mesh.f_ext.copy_(self._user_f_ext + self._contact_forces)
        self.mesh._bc_dirty = True
        self.last_result = self.solver.solve(verbose=verbose)
        return self.last_result

    def get_current_positions(self) -> torch.Tensor:
        """Reference coordinates + displacement (device, (n, 3) FP64)."""
        return self._X + self.mesh.u

    def get_reference_positions(self) -> np.ndarray:
        return np.asarray(self.mesh.X)

    def inject_contact_forces(self, forces: torch.Tensor):
        self._contact_forces += forces

    def clear_contact_forces(self):
        self._contact_forces.zero_()

    @property
    def contact_forces(self) -> np.ndarray:
        return self._contact_forces.cpu().numpy()


class ContactDefinition:
    """framework/contact.py:19-40 (bodies by index)."""

    def __init__(self, body_idx_a, body_idx_b, method, penalty, gap_tolerance, surface_a, surface_b,
                 static_friction, dynamic_friction):
        self.body_idx_a, self.body_idx_b = body_idx_a, body_idx_b
        self.method = method
        self.penalty, self.gap_tolerance = penalty, gap_tolerance
        self.surface_a, self.surface_b = surface_a, surface_b
        self.static_friction, self.dynamic_friction = static_friction, dynamic_friction
        self._auto_penalty = penalty is None
        self._auto_gap = gap_tolerance is None
        self._tied_pairs = None
        self._tied_ref_offsets = None


class Scene:
    """Multi-body static contact (framework/scene.py:30-632, static mode)."""

    def __init__(self):
        self._bodies: List[FEMBody] = []
        self._contacts: List[ContactDefinition] = []
        self._built = False

    def add(self, body: FEMBody) -> FEMBody:
        if not isinstance(body, FEMBody):
            raise FEAValidationError("Scene bodies are FEMBody objects", parameter="body")
        body._index = len(self._bodies)
        self._bodies.append(body)
        self._built = False
        return body

    def add_contact(self, body_a: FEMBody, body_b: FEMBody, method: ContactType = ContactType.PENALTY,
                    penalty: Optional[float] = None, gap_tolerance: Optional[float] = None,
                    surface_a: Optional[np.ndarray] = None, surface_b: Optional[np.ndarray] = None,
                    static_friction: float = 0.0, dynamic_friction: float = 0.0):
        """scene.py:76-124."""
        if body_a not in self._bodies or body_b not in self._bodies:
            raise FEAValidationError("contact bodies must be added to the Scene first", parameter="body")
        if dynamic_friction == 0.0 and static_friction > 0.0:
            dynamic_friction = static_friction
        self._contacts.append(ContactDefinition(
            body_a._index, body_b._index, method, penalty, gap_tolerance,
            None if surface_a is None else np.asarray(surface_a, dtype=np.int64),
            None if surface_b is None else np.asarray(surface_b, dtype=np.int64),
            static_friction, dynamic_friction))
        self._built = False

    def _build(self):
        """scene.py:126-183: surfaces, gap and penalty estimates, tied pairs."""
        if self._built:
            return
        lib = _lib.load()
        for c in self._contacts:
            a, b = self._bodies[c.body_idx_a], self._bodies[c.body_idx_b]
            if c.surface_a is None:
                c.surface_a = boundary_nodes(a.get_reference_positions())
            if c.surface_b is None:
                c.surface_b = boundary_nodes(b.get_reference_positions())
            if c._auto_gap:
                c.gap_tolerance = max(a.spacing, b.spacing) * 1.5
            if c._auto_penalty:
                Ea, Eb = a.E, b.E
                E_avg = max(Ea, Eb) if (Ea == 0.0 or Eb == 0.0) else (Ea + Eb) / 2
                h = min(a.spacing, b.spacing)
                c.penalty = E_avg / h if h > 0 else 1e6
            dev = a.mesh.device
            c._sa = torch.as_tensor(c.surface_a.astype(np.int32), device=dev)
            c._sb = torch.as_tensor(c.surface_b.astype(np.int32), device=dev)
            if c.method == ContactType.TIED:
                # detect_tied_pairs (contact.py:175-222) at the reference positions
                pa = torch.as_tensor(a.get_reference_positions(), device=dev).contiguous()
                pb = torch.as_tensor(b.get_reference_positions(), device=dev).contiguous()
                na = len(c.surface_a)
                near = torch.empty(na, dtype=torch.int32, device=dev)
                dist = torch.empty(na, dtype=torch.float64, device=dev)
                torch.cuda.synchronize(dev)
                _check(lib.fem_contact_nearest(_ptr(pa), _ptr(c._sa), na, _ptr(pb), _ptr(c._sb), len(c.surface_b),
                                               _ptr(near), _ptr(dist), None), "fem_contact_nearest")
                torch.cuda.synchronize(dev)
                m = dist < c.gap_tolerance
                ia = c._sa.long()[m]
                ib = c._sb.long()[near.long()[m]]
                c._tied_pairs = torch.stack([ia, ib], dim=1).to(torch.int32).contiguous()
                c._tied_ref_offsets = (pa[ia] - pb[ib]).contiguous()
        self._built = True

    def _compute_and_inject_contact(self) -> float:
        """scene.py:291-359 on the GPU kernels."""
        lib = _lib.load()
        for body in self._bodies:
            body.clear_contact_forces()
        total = 0.0
        for c in self._contacts:
            a, b = self._bodies[c.body_idx_a], self._bodies[c.body_idx_b]
            dev = a.mesh.device
            pa = a.get_current_positions().contiguous()
            pb = b.get_current_positions().contiguous()
            fa = torch.zeros_like(pa)
            fb = torch.zeros_like(pb)
            tot = C.c_double(0.0)
            torch.cuda.synchronize(dev)
            if c.method == ContactType.TIED:
                n = 0 if c._tied_pairs is None else int(c._tied_pairs.shape[0])
                if n == 0:
                    continue
                _check(lib.fem_contact_tied(_ptr(pa), _ptr(pb), _ptr(c._tied_pairs), _ptr(c._tied_ref_offsets), n,
                                            b.mesh.n_nodes, c.penalty, _ptr(fa), _ptr(fb), C.byref(tot), None),
                       "fem_contact_tied")
            else:
                npairs = C.c_int32(0)
                _check(lib.fem_contact_penalty(_ptr(pa), _ptr(c._sa), len(c.surface_a), _ptr(pb), _ptr(c._sb),
                                               len(c.surface_b), c.gap_tolerance, c.penalty, _ptr(fa), _ptr(fb),
                                               C.byref(npairs), C.byref(tot), None), "fem_contact_penalty")
                if npairs.value == 0:
                    continue
            a.inject_contact_forces(fa)
            b.inject_contact_forces(fb)
            total += tot.value
        return total

    def solve(self, mode: str = "static", max_contact_iters: int = 50, contact_tol: float = 1e-3,
              verbose: bool = False, **kwargs) -> dict:
        """scene.py:215-289; static mode only (FEM bodies)."""
        if mode != "static":
            raise FEAValidationError(f"mode {mode!r}: the GPU scene solves FEM bodies in static mode",
                                     parameter="mode")
        self._build()
        return self._solve_static(max_contact_iters, contact_tol, verbose)

    def _solve_static(self, max_contact_iters: int, contact_tol: float, verbose: bool) -> dict:
        """scene.py:559-632."""
        t0 = time.time()
        prev = 0.0
        converged = False
        results = [None] * len(self._bodies)
        total = 0.0
        history = []
        it = 0
        for it in range(max_contact_iters):
            if it == 0:
                for body in self._bodies:
                    body.clear_contact_forces()
                for i, body in enumerate(self._bodies):
                    if body.has_fixed:
                        results[i] = body.solve(verbose=verbose)
            total = self._compute_and_inject_contact()
            history.append(total)
            if total == 0:
                converged = True
                break
            for i, body in enumerate(self._bodies):
                results[i] = body.solve(verbose=verbose)
            if it > 0:
                rel = abs(total - prev) / (total + 1e-30)
                if verbose:
                    print(f"  contact iteration {it}: |F_c|={total:.4e}, change={rel:.4e}")
                if rel < contact_tol:
                    converged = True
                    break
            prev = total
        if len(self._contacts) == 0:
            converged = True
        return {"converged": converged, "contact_iterations": it + 1, "total_contact_force": total,
                "elapsed_time": time.time() - t0, "body_results": results, "contact_force_history": history}
