"""The arc-length loop (simul_b200.arclength.arc_length_path) on the CPU,
driven by the FP64 oracle's forces and direct tangent solves: the path ends
at (just past) the load factor asked for, every converged point is an
equilibrium point of the oracle's residual, and the last one is the
load-controlled oracle solution at its load factor
(arclength_solver.py:94-348)."""
import numpy as np
import torch

from oracle import fem_oracle as O
from simul_b200 import meshgen
from simul_b200.arclength import arc_length_path


def _bar():
    bar = meshgen.cantilever_bar(nx=6, ny=2, nz=2)
    return bar, O.Mesh(bar.X, bar.conn), O.Material("neo_hookean", E=17e3, nu=0.3)


def _callables(bar, m, mat):
    state = {"u": np.zeros_like(bar.X)}

    def forces(u):
        uu = u.numpy().reshape(-1, 3)
        state["u"] = uu.copy()
        return torch.from_numpy(O.internal_state(m, mat, uu)[3].reshape(-1).copy())

    def solve(b):
        F = O.deformation_gradient(state["u"], bar.conn.astype(np.int64), m.dNdX)
        x = O.solve_tangent(mat, F, None, m, b.numpy().reshape(-1, 3), bar.fixed_mask)
        return torch.from_numpy(x.reshape(-1).copy())

    return forces, solve


def test_arc_length_path_reaches_target_on_the_equilibrium_path():
    bar, m, mat = _bar()
    forces, solve = _callables(bar, m, mat)
    f_ref = torch.from_numpy(bar.f_ext.reshape(-1).copy())
    free = torch.from_numpy(~bar.fixed_mask.reshape(-1))
    res = arc_length_path(forces, solve, f_ref, free, arc_length=2.0, max_steps=60, max_iterations=30,
                          tol=1e-8, psi=1.0, desired_iterations=5, min_arc_length=1e-6, max_arc_length=10.0,
                          max_load_factor=1.0)
    assert res["converged"] and res["n_steps"] >= 2
    lams = np.array(res["load_factors"])
    # the last predictor is clipped to the target; its corrector may move the
    # point slightly along the arc, past it (the reference stops there too)
    assert np.all(np.diff(lams) > 0) and 1.0 <= lams[-1] < 1.01
    for lam, u in zip(lams[1:], res["displacements"][1:]):
        R = O.residual(m, mat, u.numpy().reshape(-1, 3), lam * bar.f_ext, bar.fixed_mask)[0]
        assert np.linalg.norm(R) <= 1e-8 * lam * np.linalg.norm(bar.f_ext)
    u_ref, _ = O.consistent_newton(m, mat, lams[-1] * bar.f_ext, bar.fixed_mask, bar.fixed_vals, tol=1e-12,
                                   line_search=False)
    u_end = res["displacements"][-1].numpy().reshape(-1, 3)
    assert np.linalg.norm(u_end - u_ref) <= 1e-7 * np.linalg.norm(u_ref)
    # energy bookkeeping: U = -1/2 u . f_neg at each converged point, positive
    assert all(e > 0 for e in res["energies"][1:])


def test_arc_length_path_rejects_zero_load():
    bar, m, mat = _bar()
    forces, solve = _callables(bar, m, mat)
    free = torch.from_numpy(~bar.fixed_mask.reshape(-1))
    try:
        arc_length_path(forces, solve, torch.zeros(bar.X.size, dtype=torch.float64), free, arc_length=0.1,
                        max_steps=5, max_iterations=5, tol=1e-8, psi=1.0, desired_iterations=5,
                        min_arc_length=1e-6, max_arc_length=10.0, max_load_factor=1.0)
    except Exception as e:  # FEAConvergenceError(reason="zero_reference_load")
        assert getattr(e, "reason", "") == "zero_reference_load"
    else:
        raise AssertionError("a zero reference load must raise")


def test_arc_length_halves_the_arc_after_a_failed_step():
    """With max_iterations = 1 no corrector converges unless the predictor
    lands on the path; the arc halves until it falls below the minimum."""
    bar, m, mat = _bar()
    forces, solve = _callables(bar, m, mat)
    f_ref = torch.from_numpy(bar.f_ext.reshape(-1).copy())
    free = torch.from_numpy(~bar.fixed_mask.reshape(-1))
    res = arc_length_path(forces, solve, f_ref, free, arc_length=1.0, max_steps=50, max_iterations=1,
                          tol=1e-14, psi=1.0, desired_iterations=5, min_arc_length=1e-3, max_arc_length=10.0,
                          max_load_factor=1.0)
    assert res["n_steps"] == 0 and not res["converged"]
