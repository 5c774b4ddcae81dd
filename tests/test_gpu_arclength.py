"""Arc-length path following on the GPU (simul_b200.arclength.ArcLengthSolver,
arclength_solver.py:37-367): every converged point is an equilibrium point
of the FP64 oracle's residual, the last one matches the oracle's
load-controlled solution at its load factor, and the equilibrium-path
accessor returns the tracked DOF."""
import numpy as np
import pytest

from oracle import fem_oracle as O
from simul_b200 import fem as B
from simul_b200 import meshgen
from simul_b200.arclength import ArcLengthSolver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precond", ["jacobi", "two_level"])
def test_arc_length_points_lie_on_the_oracle_equilibrium_path(cuda, precond):
    bar = meshgen.cantilever_bar(nx=6, ny=2, nz=2)
    mesh = B.FEMesh(bar.n_nodes, bar.n_elements, device=cuda)
    mesh.initialize_from_numpy(bar.X, bar.conn)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    mesh.set_nodal_forces(np.arange(bar.n_nodes), bar.f_ext)
    mesh.set_coarse_options(cell=2)
    mat = B.NeoHookean(17e3, 0.3)
    solver = ArcLengthSolver(mesh, mat, arc_length=2.0, max_steps=60, tol=1e-8, precond=precond, cg_rtol=1e-7)
    res = solver.solve(verbose=False)
    assert res["converged"] and res["n_steps"] >= 2
    lams = np.array(res["load_factors"])
    assert np.all(np.diff(lams) > 0) and 1.0 <= lams[-1] < 1.01
    m = O.Mesh(bar.X, bar.conn)
    om = O.Material("neo_hookean", E=17e3, nu=0.3)
    for lam, u in zip(lams[1:], res["displacements"][1:]):
        R = O.residual(m, om, u.reshape(-1, 3), lam * bar.f_ext, bar.fixed_mask)[0]
        assert np.linalg.norm(R) <= 2e-8 * lam * np.linalg.norm(bar.f_ext)
    u_ref, _ = O.consistent_newton(m, om, lams[-1] * bar.f_ext, bar.fixed_mask, bar.fixed_vals, tol=1e-12,
                                   line_search=False)
    u_end = res["displacements"][-1].reshape(-1, 3)
    assert np.linalg.norm(u_end - u_ref) <= 1e-6 * np.linalg.norm(u_ref)
    tip = int(np.argmax(bar.X[:, 0] + bar.X[:, 2]))
    d, l = solver.get_equilibrium_path(tip, 2)
    assert d.shape == l.shape == (res["n_steps"] + 1,) and d[-1] < 0
    assert res["cg_iterations"] > 0
