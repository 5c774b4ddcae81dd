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
