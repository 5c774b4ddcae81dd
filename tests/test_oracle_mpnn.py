"""CPU checks of the learned-preconditioner oracle (oracle/mpnn_oracle.py).

The reference has no learned preconditioner, so the oracle is pinned by its
own mathematics: gradients against central finite differences of the FP64
forward (relative error < 1e-5), BF16 rounding against torch's, the identity
"zero decoder == Jacobi", scale equivariance, and flexible PCG converging to
the direct solve.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spl
import torch

from oracle import fem_oracle as O
from oracle import mpnn_oracle as M
from simul_b200 import meshgen


@pytest.fixture(scope="module")
def bar_case():
    bar = meshgen.cantilever_bar()
    rng = np.random.default_rng(0)
    dinv = rng.uniform(0.5, 2.0, (bar.n_nodes, 3))
    fb = np.zeros(bar.n_nodes, dtype=np.int64)
    fb[bar.fixed_mask[:, 0]] = 7
    dinv[fb == 7] = 0.0
    c = rng.standard_normal(bar.n_nodes) * 0.3
    return bar, dinv, fb, c, M.node_graph(bar.conn, bar.n_nodes)


def test_parameter_count_and_flatten_roundtrip():
    assert M.n_params() == 34307
    w = M.init_params(seed=3, out_scale=0.1)
    assert np.array_equal(M.flatten(M.unflatten(w)), w)


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(1).standard_normal(10000) * np.logspace(-20, 20, 10000)
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16(x), ref)


def test_node_graph_symmetric_without_self_loops(bar_case):
    bar, *_, (ptr, idx) = bar_case
    rows = np.repeat(np.arange(bar.n_nodes), np.diff(ptr))
    assert not np.any(rows == idx)
    pairs = set(zip(rows.tolist(), idx.tolist()))
    assert all((b, a) in pairs for a, b in pairs)


def test_gradient_matches_finite_differences(bar_case):
    bar, dinv, fb, c, g = bar_case
    rng = np.random.default_rng(2)
    w = M.init_params(seed=1, out_scale=0.1)
    r = rng.standard_normal((bar.n_nodes, 3))
    r[fb == 7] = 0.0
    gz = rng.standard_normal((bar.n_nodes, 3))
    G = M.backward(w, r, dinv, fb, c, g, gz, bf16_storage=False)
    eps = 1e-6
    idx = rng.choice(w.size, 40, replace=False)
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (np.sum(gz * M.forward(wp, r, dinv, fb, c, g, False))
              - np.sum(gz * M.forward(wm, r, dinv, fb, c, g, False))) / (2 * eps)
        assert abs(G[i] - fd) <= 1e-5 * max(abs(fd), 1e-3), (i, G[i], fd)


def test_zero_decoder_is_jacobi_and_scale_equivariant(bar_case):
    bar, dinv, fb, c, g = bar_case
    r = np.random.default_rng(3).standard_normal((bar.n_nodes, 3))
    z0 = M.forward(M.init_params(seed=0, out_scale=0.0), r, dinv, fb, c, g)
    assert np.allclose(z0, dinv * r, rtol=0, atol=1e-14)
    w = M.init_params(seed=0, out_scale=0.3)
    z1 = M.forward(w, r, dinv, fb, c, g)
    z4 = M.forward(w, 4.0 * r, dinv, fb, c, g)
    assert np.allclose(z4, 4.0 * z1, rtol=1e-12, atol=1e-14)
    assert np.all(M.forward(w, np.zeros_like(r), dinv, fb, c, g) == 0.0)


def test_fpcg_with_network_reaches_direct_solution():
    bar = meshgen.cantilever_bar()
    m = O.Mesh(bar.X, bar.conn)
    mo = O.Material("linear_elastic", E=17e3, nu=0.3)
    F = O.deformation_gradient(np.zeros_like(bar.X), bar.conn.astype(np.int64), m.dNdX)
    K = O.assemble(O.element_stiffness(O.tangent_A(mo, F), m.dNdX, m.vol), bar.conn.astype(np.int64), bar.n_nodes)
    free = ~bar.fixed_mask.reshape(-1)
    Kff = K[free][:, free].tocsr()
    b = np.random.default_rng(4).standard_normal(Kff.shape[0])
    d = Kff.diagonal()
    dinv = np.zeros(3 * bar.n_nodes)
    dinv[free] = 1.0 / d
    fb = (bar.fixed_mask[:, 0] * 7).astype(np.int64)
    g = M.node_graph(bar.conn, bar.n_nodes)
    c = np.zeros(bar.n_nodes)
    # zero decoder: the network path must reproduce Jacobi-PCG exactly (the
    # flexible beta reduces to Fletcher-Reeves for a fixed SPD preconditioner)
    w = M.init_params(seed=5, out_scale=0.0)

    def precond(rf):
        full = np.zeros(3 * bar.n_nodes)
        full[free] = rf
        z = M.forward(w, full.reshape(-1, 3), dinv.reshape(-1, 3), fb, c, g, bf16_storage=False)
        return z.reshape(-1)[free]

    x, it = M.fpcg(lambda p: Kff @ p, precond, b, 1e-10, 2000)
    x_ref = spl.spsolve(Kff.tocsc(), b)
    assert it < 2000
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-8
    xj, itj = M.fpcg(lambda p: Kff @ p, lambda rf: rf / d, b, 1e-10, 2000)
    assert abs(itj - it) <= 0.05 * itj      # same method; rounding moves the count a little


def test_energy_loss_and_adam_step():
    rng = np.random.default_rng(6)
    A = rng.standard_normal((6, 6))
    A = A @ A.T + 6 * np.eye(6)
    e = rng.standard_normal(6)
    r = A @ e
    assert M.energy_loss(e, r, A @ e, e @ r) == pytest.approx(0.0, abs=1e-12)
    assert M.energy_loss(np.zeros(6), r, np.zeros(6), e @ r) == pytest.approx(1.0)
    w, m, v = M.adam_step(np.ones(3), np.array([1.0, -2.0, 0.0]), np.zeros(3), np.zeros(3), 1, 0.1)
    assert np.allclose(w, [0.9, 1.1, 1.0], atol=1e-6)
