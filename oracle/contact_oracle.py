"""FP64 restatement of the reference's staggered static contact solve.

Test infrastructure only (checker of the GPU contact kernels and of
``simul_b200.scene``); nothing in the product imports it.

Follows, line by line in behaviour:
- node-to-node penalty contact, ``backend/fea/framework/contact.py``:
  ``NodeNodeContact.detect`` (:49-92: nearest B-surface node of every
  A-surface node, pairs closer than the gap tolerance), ``compute_forces``
  (:94-173, without damping: f = penalty (gap_tol - d) (x_a - x_b) / max(d, 1e-15),
  added to A, subtracted from B, in pair order), ``detect_tied_pairs`` /
  ``compute_tied_forces`` (:175-273: f = -penalty ((x_a - x_b) - offset_0));
- the per-contact injection, ``framework/scene.py:291-359``
  (``_compute_and_inject_contact``: forces cleared, every contact's forces
  added to its two bodies, the returned total is sum |forces_a|);
- the staggered loop, ``framework/scene.py:559-632`` (``_solve_static``):
  iteration 0 solves the bodies that have fixed DOFs, then every iteration
  computes and injects the contact forces at the current positions, stops
  if there are none, re-solves every body, and (from iteration 1) stops when
  the relative change of the total contact force is below ``contact_tol``;
- the automatic parameters of ``framework/scene.py:126-213``: the boundary
  of a body is its nodes on the min / max planes of each axis (tolerance
  half the smallest coordinate step), gap tolerance 1.5 x the larger mesh
  spacing, penalty E_avg / the smaller spacing.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np


def detect(pos_a, pos_b, surface_a, surface_b, gap_tol):
    """contact.py:49-92.  Returns pairs (n, 2) of global node ids and distances."""
    from scipy.spatial import cKDTree
    surface_a = np.asarray(surface_a, dtype=np.int64)
    surface_b = np.asarray(surface_b, dtype=np.int64)
    tree = cKDTree(pos_b[surface_b])
    dists, local = tree.query(pos_a[surface_a])
    mask = dists < gap_tol
    if not np.any(mask):
        return np.empty((0, 2), dtype=np.int64), np.empty(0)
    return np.column_stack([surface_a[mask], surface_b[local[mask]]]), dists[mask]


def compute_forces(pos_a, pos_b, pairs, gaps, penalty, gap_tol):
    """contact.py:94-173 without the damping term (the static solve passes none)."""
    fa = np.zeros_like(pos_a)
    fb = np.zeros_like(pos_b)
    if len(pairs) == 0:
        return fa, fb
    ia, ib = pairs[:, 0], pairs[:, 1]
    pen = gap_tol - gaps
    diff = pos_a[ia] - pos_b[ib]
    nrm = np.maximum(np.linalg.norm(diff, axis=1, keepdims=True), 1e-15)
    f = (penalty * pen)[:, None] * (diff / nrm)
    np.add.at(fa, ia, f)
    np.add.at(fb, ib, -f)
    return fa, fb


def detect_tied_pairs(pos_a, pos_b, surface_a, surface_b, gap_tol):
    """contact.py:175-222: nearest pairs within the gap and their initial offsets."""
    pairs, _ = detect(pos_a, pos_b, surface_a, surface_b, gap_tol)
    if len(pairs) == 0:
        return pairs, np.empty((0, pos_a.shape[1]))
    return pairs, pos_a[pairs[:, 0]] - pos_b[pairs[:, 1]]


def compute_tied_forces(pos_a, pos_b, pairs, ref_offsets, penalty):
    """contact.py:224-273: two-sided springs holding the initial offsets."""
    fa = np.zeros_like(pos_a)
    fb = np.zeros_like(pos_b)
    if len(pairs) == 0:
        return fa, fb
    ia, ib = pairs[:, 0], pairs[:, 1]
    f = -penalty * ((pos_a[ia] - pos_b[ib]) - ref_offsets)
    np.add.at(fa, ia, f)
    np.add.at(fb, ib, -f)
    return fa, fb


def boundary_nodes(X: np.ndarray) -> np.ndarray:
    """scene.py:185-206: nodes on the min / max plane of each axis."""
    out = set()
    for ax in range(X.shape[1]):
        c = X[:, ax]
        u = np.unique(np.round(c, decimals=10))
        tol = np.min(np.diff(u)) * 0.5 if len(u) > 1 else 1e-6
        out.update(np.where(np.abs(c - c.min()) < tol)[0])
        out.update(np.where(np.abs(c - c.max()) < tol)[0])
    return np.array(sorted(out), dtype=np.int64)


class Body:
    """One FEM body of the staggered loop: reference coordinates, a solve
    callable (f_ext -> displacement, warm-started from its last state),
    the user loads, and whether it has fixed DOFs."""

    def __init__(self, X, solve: Callable[[np.ndarray], np.ndarray], f_user=None, has_fixed=True):
        self.X = np.asarray(X, dtype=np.float64)
        self._solve = solve
        self.f_user = np.zeros_like(self.X) if f_user is None else np.asarray(f_user, dtype=np.float64)
        self.f_contact = np.zeros_like(self.X)
        self.u = np.zeros_like(self.X)
        self.has_fixed = has_fixed

    def solve(self):
        self.u = self._solve(self.f_user + self.f_contact)

    def positions(self):
        return self.X + self.u


class Contact:
    def __init__(self, a: int, b: int, surface_a, surface_b, penalty: float, gap_tol: float, tied=False):
        self.a, self.b = a, b
        self.surface_a = np.asarray(surface_a, dtype=np.int64)
        self.surface_b = np.asarray(surface_b, dtype=np.int64)
        self.penalty, self.gap_tol, self.tied = float(penalty), float(gap_tol), tied
        self.pairs = None
        self.offsets = None


def inject(bodies: Sequence[Body], contacts: Sequence[Contact]) -> float:
    """scene.py:291-359."""
    for b in bodies:
        b.f_contact[:] = 0.0
    total = 0.0
    for c in contacts:
        pa, pb = bodies[c.a].positions(), bodies[c.b].positions()
        if c.tied:
            if c.pairs is None or len(c.pairs) == 0:
                continue
            fa, fb = compute_tied_forces(pa, pb, c.pairs, c.offsets, c.penalty)
        else:
            pairs, gaps = detect(pa, pb, c.surface_a, c.surface_b, c.gap_tol)
            if len(pairs) == 0:
                continue
            fa, fb = compute_forces(pa, pb, pairs, gaps, c.penalty, c.gap_tol)
        act_a = np.where(np.any(fa != 0, axis=1))[0]
        act_b = np.where(np.any(fb != 0, axis=1))[0]
        bodies[c.a].f_contact[act_a] += fa[act_a]
        bodies[c.b].f_contact[act_b] += fb[act_b]
        total += np.sum(np.abs(fa))
    return total


def solve_static(bodies: List[Body], contacts: List[Contact], max_contact_iters=50, contact_tol=1e-3):
    """scene.py:559-632.  Returns the result dict (without timing) and the
    total contact force of every iteration."""
    for c in contacts:
        if c.tied and c.pairs is None:
            c.pairs, c.offsets = detect_tied_pairs(bodies[c.a].X, bodies[c.b].X, c.surface_a, c.surface_b,
                                                   c.gap_tol)
    prev = 0.0
    converged = False
    total = 0.0
    history = []
    it = 0
    for it in range(max_contact_iters):
        if it == 0:
            for b in bodies:
                b.f_contact[:] = 0.0
            for b in bodies:
                if b.has_fixed:
                    b.solve()
        total = inject(bodies, contacts)
        history.append(total)
        if total == 0:
            converged = True
            break
        for b in bodies:
            b.solve()
        if it > 0:
            rel = abs(total - prev) / (total + 1e-30)
            if rel < contact_tol:
                converged = True
                break
        prev = total
    if len(contacts) == 0:
        converged = True
    return {"converged": converged, "contact_iterations": it + 1, "total_contact_force": total}, history
