"""HEX8 (8-node hexahedron, 2 x 2 x 2 Gauss points) on the GPU against the
FP64 oracle run on the same seeded inputs.

Tolerances as the TET4 parity tests: FP64 geometry 1e-12, FP64 residual and
stress 1e-9 (relative to the field's max), FP32 tangent matvec 2e-5 relative
L2, converged displacements 1e-6 relative L2."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import fem_oracle as O
from simul_b200 import _lib, meshgen
from simul_b200 import fem as B
from tests.golden import gen_golden as G

pytestmark = pytest.mark.gpu


def _rel_max(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _ptr(t):
    # pending torch writes finish before the library reads (B._ptr)
    return B._ptr(t)


def distorted_grid(n=3, seed=0, amp=0.12):
    """n^3 unit-spaced HEX8 grid with interior nodes moved by up to amp."""
    X, conn = meshgen.structured_hex8(n, n, n, (float(n),) * 3)
    rng = np.random.default_rng(seed)
    inner = np.all((X > 0.5) & (X < n - 0.5), axis=1)
    X = X.copy()
    X[inner] += amp * rng.uniform(-1, 1, (int(inner.sum()), 3))
    return X, conn


def hex_mesh(X, conn, cuda):
    mesh = B.FEMesh(X.shape[0], conn.shape[0], B.ElementType.HEX8, device=cuda)
    mesh.initialize_from_numpy(X, conn)
    return mesh


MATS = {
    "nh": (lambda: B.NeoHookean(17e3, 0.3), lambda: O.Material("neo_hookean", E=17e3, nu=0.3)),
    "mr": (lambda: B.MooneyRivlin(0.18, 0.045, 0.5), lambda: O.Material("mooney_rivlin", C10=0.18, C01=0.045, D1=0.5)),
    "fmr": (lambda: B.FibreReinforcedMooneyRivlin(0.18, 0.045, 0.5, G.FIBRES, 500.0),
            lambda: O.Material("ti_hyper", C10=0.18, C01=0.045, D1=0.5, fiber_a=np.asarray(G.FIBRES, dtype=float),
                               fiber_E=500.0)),
    "le": (lambda: B.LinearElastic(1e3, 0.3), lambda: O.Material("linear_elastic", E=1e3, nu=0.3)),
    "ti": (lambda: B.TransverseIsotropic(17e3, 11.5e3, 0.3, 0.35, 3.3e3, fiber_direction=(1.0, 1.0, 0.0)),
           lambda: O.Material("transverse_isotropic",
                              C_voigt=O.ti_global_C(17e3, 11.5e3, 0.3, 0.35, 3.3e3, (1.0, 1.0, 0.0)))),
}


def test_hex8_reference_quantities(cuda):
    X, conn = distorted_grid()
    mesh = hex_mesh(X, conn, cuda)
    m = O.Mesh(X, conn)
    assert _rel_max(mesh.dNdX.cpu().numpy(), m.dNdX) < 1e-12
    assert _rel_max(mesh.gauss_vol.cpu().numpy(), m.vol) < 1e-12
    assert mesh.elem_vol.sum().item() == pytest.approx(27.0, rel=1e-12)
    mesh.compute_deformation_gradient()
    assert np.abs(mesh.F.cpu().numpy() - np.eye(3)).max() < 1e-14


@pytest.mark.parametrize("key", ["nh", "mr", "fmr", "le", "ti"])
def test_hex8_forces_stress_and_tangent(cuda, key):
    X, conn = distorted_grid(seed=1)
    mesh = hex_mesh(X, conn, cuda)
    gpu_mat, ora_mat = MATS[key][0](), MATS[key][1]()
    rng = np.random.default_rng(11)
    u = 0.02 * rng.standard_normal(X.shape)
    mesh.u.copy_(torch.from_numpy(u))
    gpu_mat.compute_nodal_forces(mesh)
    m = O.Mesh(X, conn)
    F, sigma, P, f, aux = O.internal_state(m, ora_mat, u)
    assert _rel_max(mesh.get_nodal_forces(), f) < 1e-9
    gpu_mat.compute_stress(mesh)
    assert _rel_max(mesh.get_stress(), sigma) < 1e-9
    assert _rel_max(mesh.F.cpu().numpy(), F) < 1e-12
    # FP32 tangent against the oracle's directional derivative
    p = rng.standard_normal(X.shape)
    x = torch.as_tensor(p, dtype=torch.float32, device=cuda)
    y = torch.empty_like(x)
    lib = _lib.load()
    assert lib.fem_tangent_matvec(mesh.ctx, _ptr(x), _ptr(y)) == 0, _lib.last_error(mesh.ctx)
    want = O.tangent_matvec(m.qmat(ora_mat), F, None, m.dNdX, m.vol, m.qconn, p)
    assert _rel_l2(y.cpu().numpy().astype(np.float64), want) < 2e-5


def test_hex8_forces_bitwise_deterministic(cuda):
    X, conn = distorted_grid(n=4, seed=2)
    mesh = hex_mesh(X, conn, cuda)
    mat = B.NeoHookean(17e3, 0.3)
    mesh.u.copy_(torch.from_numpy(0.01 * np.random.default_rng(3).standard_normal(X.shape)))
    mat.compute_nodal_forces(mesh)
    a = mesh.get_nodal_forces().copy()
    for _ in range(3):
        mat.compute_nodal_forces(mesh)
        assert np.array_equal(mesh.get_nodal_forces(), a)


def _uniaxial(n=3, strain=-0.01):
    X, conn = meshgen.structured_hex8(n, n, n)
    fixed = np.zeros_like(X, dtype=bool)
    vals = np.zeros_like(X)
    for d in range(3):
        fixed[np.isclose(X[:, d], 0.0), d] = True
    top = np.isclose(X[:, 2], 1.0)
    fixed[top, 2] = True
    vals[top, 2] = strain
    return X, conn, fixed, vals


@pytest.mark.parametrize("block", [False, True])
def test_hex8_uniaxial_compression_is_exact(cuda, block):
    # the homogeneous field is the exact trilinear solution
    X, conn, fixed, vals = _uniaxial()
    mesh = hex_mesh(X, conn, cuda)
    mesh.set_block_smoother(block)
    idx = np.where(fixed.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, vals.reshape(-1)[idx])
    res = B.StaticSolver(mesh, B.LinearElastic(1e3, 0.3), tol=1e-10).solve(verbose=False)
    assert res["converged"], res
    e = -0.01
    exact = np.stack([-0.3 * e * X[:, 0], -0.3 * e * X[:, 1], e * X[:, 2]], axis=1)
    assert np.abs(mesh.get_displacements() - exact).max() < 1e-9


def test_hex8_reference_compression_case(cuda):
    # backend/fea/fem/tests/test_hex8.py:194-256 through the drop-in StaticSolver
    X, conn = meshgen.structured_hex8(2, 2, 2, (2.0, 2.0, 2.0))
    mesh = hex_mesh(X, conn, cuda)
    bottom = np.where(X[:, 2] < 0.1)[0]
    top = np.where(X[:, 2] > 2.0 - 0.1)[0]
    mesh.set_fixed_nodes(bottom)
    forces = np.zeros((top.size, 3))
    forces[:, 2] = -100.0
    mesh.set_nodal_forces(top, forces)
    res = B.StaticSolver(mesh, B.LinearElastic(1e6, 0.3)).solve(verbose=False)
    assert res["converged"], res
    u = mesh.get_displacements()
    assert np.all(u[top, 2] < 0)
    fixed = np.zeros_like(X, dtype=bool)
    fixed[bottom] = True
    f = np.zeros_like(X)
    f[top] = forces
    want, _ = O.consistent_newton(O.Mesh(X, conn), O.Material("linear_elastic", E=1e6, nu=0.3), f, fixed,
                                  np.zeros_like(X), tol=1e-12)
    assert _rel_l2(u, want) < 1e-6


def test_hex8_two_level_pcg_matches_oracle(cuda):
    # the lattice's Galerkin blocks come from the HEX8 element tangents; a
    # learned request runs Jacobi-PCG on HEX8 and counts a fallback
    vb = meshgen.vertebral_body(16, seed=4, element="hex8")
    mesh = hex_mesh(vb.X, vb.conn, cuda)
    idx = np.where(vb.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    mat = B.LinearElastic(vb.E, 0.3)
    mat.compute_nodal_forces(mesh)
    mesh.set_coarse_options(cell=2, reuse=1)
    lib = _lib.load()
    rhs = np.random.default_rng(5).standard_normal(vb.X.shape)
    rhs[vb.fixed_mask] = 0.0
    r = torch.as_tensor(rhs, device=cuda)
    out = {}
    for pc in (_lib.FEM_PRECOND_JACOBI, _lib.FEM_PRECOND_TWO_LEVEL, _lib.FEM_PRECOND_LEARNED):
        du = torch.zeros_like(r)
        it, rel = C.c_int32(), C.c_double()
        rc = lib.fem_pcg(mesh.ctx, pc, _ptr(r), _ptr(du), 1e-8, 20000, C.byref(it), C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        out[pc] = (du.cpu().numpy(), it.value)
    info = mesh.coarse_info()
    assert info["assemblies"] >= 1 and info["coarse_nodes"] > 0
    assert info["jacobi_fallbacks"] == 1
    jac, tl, lrn = out[_lib.FEM_PRECOND_JACOBI], out[_lib.FEM_PRECOND_TWO_LEVEL], out[_lib.FEM_PRECOND_LEARNED]
    assert tl[1] < jac[1], (tl[1], jac[1])
    assert lrn[1] == jac[1] and np.array_equal(lrn[0], jac[0])
    m = O.Mesh(vb.X, vb.conn)
    F = np.broadcast_to(np.eye(3), (m.n_points, 3, 3)).copy()
    want = O.solve_tangent(O.Material("linear_elastic", E=vb.E, nu=0.3), F, None, m, rhs, vb.fixed_mask)
    assert _rel_l2(jac[0], want) < 1e-6
    assert _rel_l2(tl[0], want) < 1e-6


def test_hex8_j2_steps_match_oracle(cuda):
    vb = meshgen.vertebral_body(10, seed=3, element="hex8")
    mesh = hex_mesh(vb.X, vb.conn, cuda)
    mat = B.J2Plasticity(vb.E, 0.3, 100.0, hardening_modulus=0.02 * vb.E)
    solver = B.StaticSolver(mesh, mat, tol=1e-10)
    m = O.Mesh(vb.X, vb.conn)
    om = O.Material("j2", E=vb.E, nu=0.3, sigma_y=100.0, H=0.02 * vb.E)
    state = O.J2State.zeros(m.n_points)
    u_ref = np.zeros_like(vb.X)
    idx = np.where(vb.fixed_mask.reshape(-1))[0]
    for k, frac in enumerate((0.25, 0.5, 0.75)):
        vals = vb.fixed_vals * frac
        mesh.set_fixed_dofs(idx, vals.reshape(-1)[idx])
        res = solver.solve(verbose=False)
        assert res["converged"], res
        u_ref, info = O.consistent_newton(m, om, np.zeros_like(vb.X), vb.fixed_mask, vals, u0=u_ref,
                                          j2_state=state, tol=1e-11)
        assert info["converged"]
        assert _rel_l2(mesh.get_displacements(), u_ref) < 1e-6
        epe = mat.get_plastic_strain()
        assert epe.shape == (m.n_points,)
        assert np.max(np.abs(epe - state.epe)) <= 1e-6 * max(state.epe.max(), 1e-12) + 1e-12
    assert state.epe.max() > 0
    # per-point history layout e * 8 + g and the Gauss-point mean nodal Mises
    assert np.max(np.abs(mat.get_plastic_strain_tensor() - state.ep)) <= 1e-6 * np.abs(state.ep).max() + 1e-12
    got = solver.get_mises_stress()
    want = O.nodal_mises(m, om, mesh.get_displacements(), O.J2State(state.ep.copy(), state.epe.copy()))
    assert np.max(np.abs(got - want)) <= 1e-6 * np.max(np.abs(want))


def test_hex8_invalid_connectivity_raises(cuda):
    X, conn = meshgen.structured_hex8(1, 1, 1)
    mesh = B.FEMesh(X.shape[0], 1, B.ElementType.HEX8, device=cuda)
    bad = conn.copy()
    bad[0, 3] = bad[0, 0]
    with pytest.raises(B.FEAValidationError):
        mesh.initialize_from_numpy(X, bad)
    with pytest.raises(B.FEAValidationError):
        mesh.initialize_from_numpy(X, conn[:, :4])


def test_labelmap_bonded_stack_on_gpu(cuda):
    # a two-label labelmap as one conforming HEX8 mesh, modulus by label:
    # the interface displacement of the series stack (nu = 0, rollers)
    lv = np.zeros((6, 5, 7), dtype=np.int16)
    lv[1:5, 1:4, 0:3] = 1
    lv[1:5, 1:4, 3:5] = 2
    X, conn, lab = meshgen.labelmap_hex8(lv, [1.0, 1.0, 1.0])
    E = np.where(lab == 1, 1000.0, 250.0)
    mesh = hex_mesh(X, conn, cuda)
    fixed = np.zeros_like(X, dtype=bool)
    vals = np.zeros_like(X)
    for d in range(3):
        fixed[np.isclose(X[:, d], X[:, d].min()), d] = True
    top = np.isclose(X[:, 2], X[:, 2].max())
    fixed[top, 2] = True
    vals[top, 2] = -0.05
    idx = np.where(fixed.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, vals.reshape(-1)[idx])
    res = B.StaticSolver(mesh, B.LinearElastic(E, 0.0), tol=1e-10, precond="two_level").solve(verbose=False)
    assert res["converged"], res
    u = mesh.get_displacements()
    iface = np.isclose(X[:, 2], 3.0)
    c1, c2 = 3.0 / 1000.0, 2.0 / 250.0
    assert np.allclose(u[iface, 2], -0.05 * c1 / (c1 + c2), rtol=1e-7)
    want, _ = O.consistent_newton(O.Mesh(X, conn), O.Material("linear_elastic", E=E, nu=0.0), np.zeros_like(X),
                                  fixed, vals, tol=1e-12)
    assert _rel_l2(u, want) < 1e-7


def _hex_beam():
    X, conn = meshgen.structured_hex8(8, 2, 2, (8.0, 1.0, 1.0))
    fixed = np.zeros_like(X, dtype=bool)
    fixed[np.isclose(X[:, 0], 0.0)] = True
    return X, conn, fixed


def test_hex8_dynamics_and_natural_frequencies(cuda):
    # Newmark on a HEX8 cantilever (lumped mass: density x volume / 8 per
    # vertex) and its lowest natural frequencies, against the dynamic oracle
    from oracle.dynamic_oracle import DynamicOracle
    from simul_b200.dynamic import DynamicSolver
    X, conn, fixed = _hex_beam()
    mesh = hex_mesh(X, conn, cuda)
    mesh.set_fixed_nodes(np.where(fixed[:, 0])[0])
    dyn = DynamicSolver(mesh, B.LinearElastic(1000.0, 0.3), density=1e-3, method="newmark",
                        rayleigh_alpha=0.5, rayleigh_beta=1e-4, formulation="consistent", cg_rtol=1e-8)
    ora = DynamicOracle(O.Mesh(X, conn), O.Material("linear_elastic", E=1000.0, nu=0.3), 1000.0, 0.3, fixed,
                        density=1e-3, method="newmark", rayleigh_alpha=0.5, rayleigh_beta=1e-4,
                        formulation="consistent")
    assert abs(dyn.dt - ora.dt) <= 1e-12 * ora.dt
    assert _rel_l2(dyn.M_diag.cpu().numpy(), ora.M) < 1e-12
    f = np.zeros_like(X)
    f[np.isclose(X[:, 0], 8.0), 2] = -0.01
    for _ in range(10):
        dyn.step(f)
        ora.step(f)
    assert _rel_l2(dyn.u.cpu().numpy(), ora.u) < 2e-5
    got = DynamicSolver(mesh, B.LinearElastic(1000.0, 0.3), density=1e-3).get_natural_frequencies(4)
    want = ora.natural_frequencies(4)
    assert np.all(np.abs(got - want) <= 1e-4 * want), (got, want)


def test_hex8_arc_length_path_reaches_the_load(cuda):
    # the arc-length loop over the HEX8 kernels stops once lambda >= 1 (the
    # corrector may carry the last point a little past it, as the reference's
    # loop allows) on the load-controlled equilibrium at that lambda
    from simul_b200.arclength import ArcLengthSolver
    X, conn, fixed = _hex_beam()
    f = np.zeros_like(X)
    f[np.isclose(X[:, 0], 8.0), 2] = -2.0
    mesh = hex_mesh(X, conn, cuda)
    mesh.set_fixed_nodes(np.where(fixed[:, 0])[0])
    mesh.set_nodal_forces(np.arange(X.shape[0]), f)
    mat = B.NeoHookean(1000.0, 0.3)
    res = ArcLengthSolver(mesh, mat, arc_length=0.5, max_steps=60, tol=1e-8, cg_rtol=1e-9).solve(verbose=False)
    lams = np.array(res["load_factors"])
    assert res["converged"] and np.all(np.diff(lams) > 0) and 1.0 <= lams[-1] < 1.1
    want, _ = O.consistent_newton(O.Mesh(X, conn), O.Material("neo_hookean", E=1000.0, nu=0.3), lams[-1] * f,
                                  fixed, np.zeros_like(X), tol=1e-12)
    assert _rel_l2(res["displacements"][-1].reshape(-1, 3), want) < 1e-6
