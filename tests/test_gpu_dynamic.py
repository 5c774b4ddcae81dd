"""Dynamic solver on the GPU (simul_b200.dynamic.DynamicSolver,
dynamic_solver.py:21-413) against the FP64 dynamic oracle: Newmark and
central difference, the reference-as-written and the textbook formulation,
with Rayleigh damping; displacements and velocities after a few steps agree
to the FP32 matvec's accuracy."""
import numpy as np
import pytest
import torch

from oracle import fem_oracle as O
from oracle.dynamic_oracle import DynamicOracle
from simul_b200 import fem as B
from simul_b200 import meshgen
from simul_b200.dynamic import DynamicSolver

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("method,formulation,steps", [("newmark", "reference", 10), ("newmark", "consistent", 10),
                                                      ("central_diff", "consistent", 20),
                                                      ("central_diff", "reference", 5)])
def test_dynamic_solver_matches_oracle(cuda, method, formulation, steps):
    bar = meshgen.cantilever_bar(nx=6, ny=2, nz=2)
    mesh = B.FEMesh(bar.n_nodes, bar.n_elements, device=cuda)
    mesh.initialize_from_numpy(bar.X, bar.conn)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    mat = B.LinearElastic(1000.0, 0.3)
    ra, rb = (0.5, 1e-4) if method == "newmark" else (0.5, 0.0)
    dyn = DynamicSolver(mesh, mat, density=1e-3, method=method, rayleigh_alpha=ra, rayleigh_beta=rb,
                        formulation=formulation, cg_rtol=1e-8)
    ora = DynamicOracle(O.Mesh(bar.X, bar.conn), O.Material("linear_elastic", E=1000.0, nu=0.3), 1000.0, 0.3,
                        bar.fixed_mask, density=1e-3, method=method, rayleigh_alpha=ra, rayleigh_beta=rb,
                        formulation=formulation)
    assert abs(dyn.dt - ora.dt) <= 1e-12 * ora.dt
    assert _rel(dyn.M_diag.cpu().numpy(), ora.M) < 1e-12
    f = bar.f_ext * 0.01
    for _ in range(steps):
        dyn.step(f)
        ora.step(f)
    assert _rel(dyn.u.cpu().numpy(), ora.u) < 2e-5
    assert _rel(dyn.v.cpu().numpy(), ora.v) < 2e-5
    assert dyn.get_kinetic_energy() > 0.0
    assert np.allclose(dyn.get_displacements(), mesh.get_displacements())


def test_natural_frequencies_match_oracle(cuda):
    bar = meshgen.cantilever_bar(nx=8, ny=2, nz=2)
    mesh = B.FEMesh(bar.n_nodes, bar.n_elements, device=cuda)
    mesh.initialize_from_numpy(bar.X, bar.conn)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    dyn = DynamicSolver(mesh, B.LinearElastic(1000.0, 0.3), density=1e-3)
    got = dyn.get_natural_frequencies(5)
    ora = DynamicOracle(O.Mesh(bar.X, bar.conn), O.Material("linear_elastic", E=1000.0, nu=0.3), 1000.0, 0.3,
                        bar.fixed_mask, density=1e-3)
    want = ora.natural_frequencies(5)
    assert np.all(np.abs(got - want) <= 1e-4 * want), (got, want)
