"""Learned preconditioner on the GPU against the CPU oracle (oracle/mpnn_oracle.py).

Tolerances: the network stores activations in BF16, so the GPU output and the
oracle's BF16-emulating forward differ by accumulation order and by rare
one-ulp BF16 rounding flips: relative L2 error of the network's contribution
z - D^-1 r below 2e-2, and of z itself below 2e-3.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import fem_oracle as O
from oracle import mpnn_oracle as M
from simul_b200 import _lib, meshgen
from simul_b200 import fem as B

pytestmark = pytest.mark.gpu


def _ptr(t):
    # pending torch writes finish before the library reads (B._ptr)
    return B._ptr(t)


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def bar_setup(cuda):
    bar = meshgen.cantilever_bar()
    mesh = B.FEMesh(bar.n_nodes, bar.n_elements, device=cuda)
    mesh.initialize_from_numpy(bar.X, bar.conn)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    mat = B.LinearElastic(17e3, 0.3)
    mat.compute_nodal_forces(mesh)
    return bar, mesh, mat


def _oracle_inputs(bar):
    m = O.Mesh(bar.X, bar.conn)
    mo = O.Material("linear_elastic", E=17e3, nu=0.3)
    F = O.deformation_gradient(np.zeros_like(bar.X), bar.conn.astype(np.int64), m.dNdX)
    A = O.tangent_A(mo, F)
    Ke = O.element_stiffness(A, m.dNdX, m.vol)
    K = O.assemble(Ke, bar.conn.astype(np.int64), bar.n_nodes)
    diag = K.diagonal().reshape(-1, 3)
    fixed = bar.fixed_mask
    dinv = np.where(fixed, 0.0, 1.0 / diag)
    fb = (fixed[:, 0] * 1 + fixed[:, 1] * 2 + fixed[:, 2] * 4).astype(np.int64)
    lam_mu = 17e3 * (1 - 0.3) / ((1 + 0.3) * (1 - 2 * 0.3))
    c = M.log_modulus_feature(bar.conn, bar.n_nodes, np.full(bar.n_elements, lam_mu))
    return dinv, fb, c, M.node_graph(bar.conn, bar.n_nodes)


@pytest.mark.parametrize("seed", [0, 1])
def test_mpnn_forward_matches_oracle(cuda, bar_setup, seed):
    bar, mesh, mat = bar_setup
    lib = _lib.load()
    w = M.init_params(seed=seed, out_scale=0.2).astype(np.float32)
    rc = lib.fem_mpnn_set_weights(mesh.ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size)
    assert rc == 0, _lib.last_error(mesh.ctx)
    rng = np.random.default_rng(10 + seed)
    r = rng.standard_normal((bar.n_nodes, 3))
    r[bar.fixed_mask] = 0.0
    dr = torch.as_tensor(r, dtype=torch.float32, device=cuda)
    dz = torch.empty_like(dr)
    rc = lib.fem_mpnn_forward(mesh.ctx, _ptr(dr), _ptr(dz))
    assert rc == 0, _lib.last_error(mesh.ctx)
    z = dz.cpu().numpy().astype(np.float64)
    dinv, fb, c, graph = _oracle_inputs(bar)
    z_ref = M.forward(w.astype(np.float64), r.astype(np.float32).astype(np.float64), dinv, fb, c, graph)
    jac = dinv * r
    assert np.all(z[bar.fixed_mask] == 0.0)
    assert _rel_l2(z - jac, z_ref - jac) < 2e-2
    assert _rel_l2(z, z_ref) < 2e-3
    # scale equivariance z(a r) = a z(r), exact up to BF16 rounding of r / s
    dz2 = torch.empty_like(dr)
    assert lib.fem_mpnn_forward(mesh.ctx, _ptr(dr * 4.0), _ptr(dz2)) == 0
    assert _rel_l2(dz2.cpu().numpy() / 4.0, z) < 1e-6


def test_mpnn_zero_decoder_is_jacobi(cuda, bar_setup):
    bar, mesh, mat = bar_setup
    lib = _lib.load()
    w = M.init_params(seed=3, out_scale=0.0).astype(np.float32)
    assert lib.fem_mpnn_set_weights(mesh.ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size) == 0
    rng = np.random.default_rng(4)
    r = rng.standard_normal((bar.n_nodes, 3))
    dr = torch.as_tensor(r, dtype=torch.float32, device=cuda)
    dz = torch.empty_like(dr)
    assert lib.fem_mpnn_forward(mesh.ctx, _ptr(dr), _ptr(dz)) == 0
    dinv, *_ = _oracle_inputs(bar)
    assert _rel_l2(dz.cpu().numpy(), dinv * r.astype(np.float32)) < 1e-6


def test_mpnn_weights_roundtrip_and_validation(cuda, bar_setup):
    bar, mesh, mat = bar_setup
    lib = _lib.load()
    w = M.init_params(seed=5, out_scale=0.1).astype(np.float32)
    assert lib.fem_mpnn_set_weights(mesh.ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size) == 0
    back = np.zeros_like(w)
    assert lib.fem_mpnn_get_weights(mesh.ctx, back.ctypes.data_as(C.POINTER(C.c_float)), back.size) == 0
    assert np.array_equal(back, w)
    bad = w.copy()
    bad[7] = np.nan
    assert lib.fem_mpnn_set_weights(mesh.ctx, bad.ctypes.data_as(C.POINTER(C.c_float)), bad.size) \
        == _lib.FEM_ERR_INVALID
    assert lib.fem_mpnn_set_weights(mesh.ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size - 1) \
        == _lib.FEM_ERR_INVALID


def test_learned_fpcg_solves_and_matches_oracle(cuda):
    """Flexible PCG with the network (+ coarse correction): same solution as
    the FP64 direct solve; with a zero decoder it reproduces two-level PCG."""
    from tests.golden import gen_golden as G
    vox = G.vox_mesh()
    mesh = B.FEMesh(vox.n_nodes, vox.n_elements, device=cuda)
    mesh.initialize_from_numpy(vox.X, vox.conn)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    B.LinearElastic(1e3, 0.3).compute_nodal_forces(mesh)
    lib = _lib.load()
    w = M.init_params(seed=2, out_scale=0.05).astype(np.float32)
    assert lib.fem_mpnn_set_weights(mesh.ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size) == 0
    rng = np.random.default_rng(8)
    rhs = rng.standard_normal(vox.X.shape)
    rhs[vox.fixed_mask] = 0.0
    r = torch.as_tensor(rhs, dtype=torch.float64, device=cuda)
    m = O.Mesh(vox.X, vox.conn)
    F = O.deformation_gradient(np.zeros_like(vox.X), vox.conn.astype(np.int64), m.dNdX)
    u_ref = O.solve_tangent(O.Material("linear_elastic", E=1e3, nu=0.3), F, None, m, rhs, vox.fixed_mask)
    for coarse in (1, 0):
        assert lib.fem_set_option(mesh.ctx, _lib.FEM_OPT_LEARNED_COARSE, coarse) == 0
        du = torch.zeros_like(r)
        it = C.c_int32()
        rel = C.c_double()
        rc = lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_LEARNED, _ptr(r), _ptr(du), 1e-7, 5000, C.byref(it),
                         C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        assert rel.value <= 1e-7 and it.value > 0
        assert _rel_l2(du.cpu().numpy(), u_ref) < 1e-5
    st = (C.c_int64 * 4)()
    assert lib.fem_learned_stats(mesh.ctx, st) == 0
    assert st[1] == 1 and st[2] > 0


def test_mpnn_backward_matches_oracle(cuda, bar_setup):
    """GPU gradients (tcgen05 products, BF16 operands) against the oracle's
    BF16-emulating backward; the oracle's own gradient is pinned to finite
    differences in tests/test_oracle_mpnn.py."""
    bar, mesh, mat = bar_setup
    lib = _lib.load()
    w = M.init_params(seed=7, out_scale=0.3).astype(np.float32)
    assert lib.fem_mpnn_set_weights(mesh.ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size) == 0
    rng = np.random.default_rng(21)
    r = rng.standard_normal((bar.n_nodes, 3))
    r[bar.fixed_mask] = 0.0
    gz = rng.standard_normal((bar.n_nodes, 3))
    gz[bar.fixed_mask] = 0.0
    dr = torch.as_tensor(r, dtype=torch.float32, device=cuda)
    dg = torch.as_tensor(gz, dtype=torch.float32, device=cuda)
    grad = np.zeros(M.n_params(), dtype=np.float32)
    rc = lib.fem_mpnn_backward(mesh.ctx, _ptr(dr), _ptr(dg), grad.ctypes.data_as(C.POINTER(C.c_float)))
    assert rc == 0, _lib.last_error(mesh.ctx)
    dinv, fb, c, graph = _oracle_inputs(bar)
    g_ref = M.backward(w.astype(np.float64), r.astype(np.float32).astype(np.float64), dinv, fb, c, graph,
                       gz.astype(np.float32).astype(np.float64))
    assert np.all(np.isfinite(grad))
    assert _rel_l2(grad.astype(np.float64), g_ref) < 2e-2
    o = 0
    for name, shp in M.param_shapes():
        k = int(np.prod(shp))
        ref = g_ref[o:o + k]
        if np.linalg.norm(ref) > 1e-6 * np.linalg.norm(g_ref):
            assert _rel_l2(grad[o:o + k].astype(np.float64), ref) < 5e-2, name
        o += k
    # deterministic: a second call gives the same bits
    grad2 = np.zeros_like(grad)
    assert lib.fem_mpnn_backward(mesh.ctx, _ptr(dr), _ptr(dg), grad2.ctypes.data_as(C.POINTER(C.c_float))) == 0
    assert np.array_equal(grad, grad2)


def test_training_gains_over_jacobi(cuda):
    """Train on pairs the plain solver generates; on held-out pairs the trained
    network's one-step A-norm error beats Jacobi's by more than 10 % (the
    gain), while the CG iteration count is not reduced (the measured loss)."""
    from simul_b200 import learned
    from tests.golden import gen_golden as G
    vox = G.vox_mesh()
    mesh = B.FEMesh(vox.n_nodes, vox.n_elements, device=cuda)
    mesh.initialize_from_numpy(vox.X, vox.conn)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    B.LinearElastic(vox.E, 0.3).compute_nodal_forces(mesh)
    learned.set_coarse(mesh, False)
    learned.set_weights(mesh, learned.init_weights(seed=0))
    rng = np.random.default_rng(0)
    R, E = learned.solver_pairs(mesh, learned.random_rhs(vox.X, vox.fixed_mask, 48, rng))
    Rv, Ev = learned.solver_pairs(mesh, learned.random_rhs(vox.X, vox.fixed_mask, 8, np.random.default_rng(99)))
    before = learned.evaluate(mesh, Rv, Ev)
    assert before["loss_net"] == pytest.approx(before["loss_base"], rel=1e-5)   # zero decoder = Jacobi
    res = learned.train(mesh, R, E, steps=300, batch=8, lr=2e-3)
    assert res["loss_last"] < res["loss_first"]
    after = learned.evaluate(mesh, Rv, Ev)
    assert after["loss_net"] < 0.9 * after["loss_base"], after
    lib = _lib.load()
    its = {}
    for name, pc in (("jacobi", _lib.FEM_PRECOND_JACOBI), ("learned", _lib.FEM_PRECOND_LEARNED)):
        du = torch.zeros(vox.X.shape, dtype=torch.float64, device=cuda)
        r = Rv[0].double().contiguous()
        it = C.c_int32()
        rel = C.c_double()
        rc = lib.fem_pcg(mesh.ctx, pc, _ptr(r), _ptr(du), 1e-8, 20000, C.byref(it), C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        its[name] = it.value
    st = (C.c_int64 * 4)()
    lib.fem_learned_stats(mesh.ctx, st)
    # The flexible solve converges without a rerun.  The one-step gain above
    # does not carry over to Krylov iterations: here the network's directions
    # keep passing the descent test, so it is never switched off, and flexible
    # PCG needs more CG iterations than Jacobi-PCG (measured 575 against 170:
    # descent directions, poor conjugate ones; tests/test_learned_headroom.py
    # bounds what a linear learned form of the two-level method could gain).
    # The bounds record that loss.
    print("CG iterations", its)
    assert st[0] == 0, its
    assert its["learned"] >= its["jacobi"], its
    assert its["learned"] <= 4 * its["jacobi"], its
