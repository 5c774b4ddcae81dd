"""Batched solves (fem_batch_solve): independent instances on their own
streams, solved concurrently, give the same displacements as solving each
instance alone (relative L2 < 1e-6; the matvec variant each picks may differ,
so bitwise equality is not required)."""
import numpy as np
import pytest
import torch

from simul_b200 import batch, meshgen
from simul_b200 import fem as B

pytestmark = pytest.mark.gpu


def _instance(n, seed, strain, cuda):
    v = meshgen.vertebral_body(n=n, seed=seed, axial_strain=strain)
    mat = B.J2Plasticity(v.E, 0.3, 100.0, hardening_modulus=0.02 * v.E)
    return v, batch.BatchInstance(v.X, v.conn, mat, v.fixed_mask, v.fixed_vals, device=cuda)


def test_batch_matches_sequential(cuda):
    specs = [(12, 1, 0.01), (14, 2, 0.02), (10, 3, 0.03)]
    insts = [_instance(n, s, e, cuda) for n, s, e in specs]
    out = batch.solve_batch([i for _, i in insts], load_steps=3, precond="two_level", n_threads=0)
    assert all(r["converged"] and r["status"] == 0 for r in out["instances"]), out
    assert all(r["wall_ms"] > 0 for r in out["instances"])
    for (n, s, e), (v, inst) in zip(specs, insts):
        mesh = B.FEMesh(v.n_nodes, v.n_elements, device=cuda)
        mesh.initialize_from_numpy(v.X, v.conn)
        mat = B.J2Plasticity(v.E, 0.3, 100.0, hardening_modulus=0.02 * v.E)
        solver = B.StaticSolver(mesh, mat, tol=1e-8, precond="two_level")
        idx = np.where(v.fixed_mask.reshape(-1))[0]
        for k in range(1, 4):
            mesh.set_fixed_dofs(idx, (v.fixed_vals * k / 3).reshape(-1)[idx])
            assert solver.solve(verbose=False)["converged"]
        u_seq = mesh.get_displacements()
        torch.cuda.synchronize()
        u_bat = inst.mesh.u.cpu().numpy()
        assert np.linalg.norm(u_bat - u_seq) / np.linalg.norm(u_seq) < 1e-6


def test_batch_rejects_duplicates_and_bad_steps(cuda):
    from simul_b200 import _lib
    import ctypes as C
    v, inst = _instance(8, 4, 0.01, cuda)
    lib = _lib.load()
    ctxs = (C.c_void_p * 2)(inst.ctx.value, inst.ctx.value)
    res = (_lib.FemSolveResult * 2)()
    st = (C.c_int32 * 2)()
    assert lib.fem_batch_solve(ctxs, 2, None, 1, res, st, None, 0) == _lib.FEM_ERR_INVALID
    assert "repeats" in _lib.last_error(None)
    ctx1 = (C.c_void_p * 1)(inst.ctx.value)
    assert lib.fem_batch_solve(ctx1, 1, None, 0, res, st, None, 0) == _lib.FEM_ERR_INVALID


def _ms_oracle_materials(ms):
    from oracle import fem_oracle as O
    fib = np.array([[np.cos(np.pi / 6), 0.0, np.sin(np.pi / 6)], [np.cos(np.pi / 6), 0.0, -np.sin(np.pi / 6)]])
    mu = 2.0 * (0.18 + 0.045)
    K = 2.0 * mu * (1.0 + 0.45) / (3.0 * (1.0 - 2.0 * 0.45))
    parts = [O.Material("j2", E=ms.E, nu=0.3, sigma_y=100.0, H=0.02 * ms.E),
             O.Material("ti_hyper", C10=0.18, C01=0.045, D1=2.0 / K, fiber_a=fib, fiber_E=500.0),
             O.Material("linear_elastic", E=110e3, nu=0.3)]
    return O.MixedMaterial(parts, ms.info["material_ids"])


def test_motion_segment_mixed_materials_match_oracle(cuda):
    """J2 bone + fibre-reinforced Mooney-Rivlin disc + elastic screw on one
    mesh, flexion moment: converged displacements within 1e-6 relative L2 of
    the FP64 oracle, with the Jacobi and the two-level preconditioner."""
    from oracle import fem_oracle as O
    from simul_b200 import motion_segment_bench as MSB
    ms = meshgen.motion_segment(n=8)
    top = np.isclose(ms.X[:, 2], ms.X[:, 2].max())
    f = meshgen.top_moment_forces(ms.X, top, "flexion", 750.0)
    m = O.Mesh(ms.X, ms.conn)
    u_ref, info = O.consistent_newton(m, _ms_oracle_materials(ms), f, ms.fixed_mask, ms.fixed_vals,
                                      j2_state=O.J2State.zeros(ms.n_elements), tol=1e-11, line_search=True)
    assert info["converged"]
    for pc in ("jacobi", "two_level"):
        mesh = B.FEMesh(ms.n_nodes, ms.n_elements, device=cuda)
        mesh.initialize_from_numpy(ms.X, ms.conn, material_ids=ms.info["material_ids"])
        mesh.set_fixed_nodes(np.where(ms.fixed_mask[:, 0])[0])
        mesh.set_nodal_forces(np.arange(ms.n_nodes), f)
        res = B.StaticSolver(mesh, materials=MSB.materials(ms.E), tol=1e-10, precond=pc).solve(verbose=False)
        assert res["converged"], (pc, res)
        u = mesh.get_displacements()
        assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) < 1e-6, pc


def test_motion_segment_moment_cases_batch(cuda):
    from simul_b200 import motion_segment_bench as MSB
    ms = meshgen.motion_segment(n=8)
    top = np.isclose(ms.X[:, 2], ms.X[:, 2].max())
    insts = [batch.BatchInstance(ms.X, ms.conn, MSB.materials(ms.E), ms.fixed_mask, None,
                                 meshgen.top_moment_forces(ms.X, top, c, 300.0), device=cuda,
                                 material_ids=ms.info["material_ids"]) for c in MSB.CASES]
    out = batch.solve_batch(insts, load_steps=2, precond="two_level")
    assert all(r["converged"] for r in out["instances"]), out
    torch.cuda.synchronize()
    u = [i.mesh.u.cpu().numpy() for i in insts]
    # flexion and extension are the same couple with opposite sign: the top
    # face moves forward in one and backward in the other (the soft disc makes
    # the response strongly nonlinear, so not exactly opposite)
    uy = [x[top, 1].mean() for x in u]
    assert uy[0] * uy[1] < 0, uy
    assert all(np.abs(x).max() > 0 for x in u)
