"""GPU parity of libfemb200 against the FP64 oracle's golden fixtures.

All calls go through the C ABI (directly or via the simul_b200 host mirror).
Tolerances: FP64 residual / stress kernels 1e-9 (relative to the field's max),
FP32 tangent matvec 2e-5 relative L2, converged displacements 1e-6 relative L2.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import fem_oracle as O
from simul_b200 import _lib, meshgen
from simul_b200 import fem as B
from tests.golden import gen_golden as G

pytestmark = pytest.mark.gpu

FIBRES = G.FIBRES


def _rel_max(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make_material(key, E=None):
    if key == "nh":
        return B.NeoHookean(17e3, 0.3)
    if key == "mr":
        return B.MooneyRivlin(0.18, 0.045, 0.5)
    if key == "fmr":
        return B.FibreReinforcedMooneyRivlin(0.18, 0.045, 0.5, FIBRES, 500.0)
    if key == "le":
        return B.LinearElastic(1e3, 0.3)
    if key == "ti":
        return B.TransverseIsotropic(17e3, 11.5e3, 0.3, 0.35, 3.3e3, fiber_direction=(1.0, 1.0, 0.0))
    if key == "j2":
        return B.J2Plasticity(E, 0.3, 100.0, hardening_modulus=0.02 * E)
    raise KeyError(key)


def make_mesh(X, conn, cuda, nb=0):
    mesh = B.FEMesh(X.shape[0], conn.shape[0], device=cuda, nodes_per_block=nb)
    mesh.initialize_from_numpy(X, conn)
    return mesh


def dev(a, cuda, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=cuda)


def ptr(t):
    # pending torch writes finish before the library reads (B._ptr)
    return B._ptr(t)


@pytest.fixture(scope="module")
def bar():
    return meshgen.cantilever_bar()


@pytest.fixture(scope="module")
def vox():
    return G.vox_mesh()


def test_fixture_meshes_unchanged(bar, vox):
    np.testing.assert_allclose(G.mesh_checksum(bar.X, bar.conn), np.load(G.path_of("bar_nh_forces"))["mesh_sum"])
    np.testing.assert_allclose(G.mesh_checksum(vox.X, vox.conn), np.load(G.path_of("vox12_j2_forces"))["mesh_sum"])


def test_reference_quantities(cuda, bar):
    ref = np.load(G.path_of("bar_nh_forces"))
    mesh = make_mesh(bar.X, bar.conn, cuda)
    assert _rel_max(mesh.dNdX.cpu().numpy(), ref["dNdX"]) < 1e-12
    assert _rel_max(mesh.elem_vol.cpu().numpy(), ref["vol"]) < 1e-12
    assert mesh.elem_vol.sum().item() == pytest.approx(10.0, rel=1e-12)


@pytest.mark.parametrize("key", ["nh", "mr", "fmr", "le", "ti"])
@pytest.mark.parametrize("nb", [128, 256, 512])
def test_element_forces_and_stress(cuda, bar, key, nb):
    ref = np.load(G.path_of(f"bar_{key}_forces"))
    mesh = make_mesh(bar.X, bar.conn, cuda, nb)
    mat = make_material(key)
    mesh.u.copy_(dev(ref["u"], cuda))
    mat.compute_nodal_forces(mesh)
    assert _rel_max(mesh.get_nodal_forces(), ref["f"]) < 1e-9
    mat.compute_stress(mesh)
    assert _rel_max(mesh.get_stress(), ref["sigma"]) < 1e-9
    if key == "nh":
        assert _rel_max(mesh.F.cpu().numpy(), ref["F"]) < 1e-12


VARIANTS = ["fused", "two_phase", "element_block", "warp_agg", "persistent"]


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("key", ["nh", "mr", "fmr", "le", "ti"])
def test_tangent_matvec(cuda, bar, key, variant):
    ref = np.load(G.path_of(f"bar_{key}_forces"))
    mesh = make_mesh(bar.X, bar.conn, cuda)
    mesh.set_matvec_variant(variant)
    mat = make_material(key)
    mesh.u.copy_(dev(ref["u"], cuda))
    mat.compute_nodal_forces(mesh)          # refreshes the tangent state
    x = dev(ref["p"], cuda, torch.float32)
    y = torch.empty_like(x)
    lib = _lib.load()
    assert lib.fem_tangent_matvec(mesh.ctx, ptr(x), ptr(y)) == 0, _lib.last_error(mesh.ctx)
    # the matvec ignores fixed DOFs; the fixture has none set on this mesh (no BC pushed)
    assert _rel_l2(y.cpu().numpy().astype(np.float64), ref["y"]) < 2e-5


def test_j2_forces_history_and_tangent(cuda, vox):
    ref = np.load(G.path_of("vox12_j2_forces"))
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mat = make_material("j2", E=vox.E)
    mesh.u.copy_(dev(ref["u"], cuda))
    mat.compute_nodal_forces(mesh)
    assert _rel_max(mesh.get_nodal_forces(), ref["f"]) < 1e-9
    x = dev(ref["p"], cuda, torch.float32)
    y = torch.empty_like(x)
    assert _lib.load().fem_tangent_matvec(mesh.ctx, ptr(x), ptr(y)) == 0
    assert _rel_l2(y.cpu().numpy().astype(np.float64), ref["y"]) < 2e-5
    # trial history of the residual pass, committed explicitly
    assert _lib.load().fem_commit_history(mesh.ctx) == 0
    assert _rel_max(mat.get_plastic_strain(), ref["epe"]) < 1e-9
    assert _rel_max(mat.get_plastic_strain_tensor(), ref["ep"]) < 1e-9
    assert mat.get_yield_status().sum() > 0
    # stress from the committed state at the same u equals sigma after the return map
    mat.compute_stress(mesh)
    s_gpu = mesh.get_stress()
    sig_chk, _ = O.cauchy_stress(O.Material("j2", E=vox.E, nu=0.3, sigma_y=100.0, H=0.02 * vox.E),
                                 O.deformation_gradient(ref["u"], vox.conn.astype(np.int64),
                                                        O.reference_quantities(vox.X, vox.conn)[0]),
                                 O.J2State(ref["ep"], ref["epe"]))
    assert _rel_max(s_gpu, sig_chk) < 1e-8
    mat.reset_state()
    assert np.all(mat.get_plastic_strain() == 0)


@pytest.mark.parametrize("variant", VARIANTS)
def test_forces_bitwise_deterministic(cuda, vox, variant):
    ref = np.load(G.path_of("vox12_j2_forces"))
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mesh.set_matvec_variant(variant)
    mat = make_material("j2", E=vox.E)
    mesh.u.copy_(dev(ref["u"], cuda))
    outs, ys = [], []
    x = dev(ref["p"], cuda, torch.float32)
    for _ in range(3):
        mat.compute_nodal_forces(mesh)
        outs.append(mesh.f.clone())
        y = torch.empty_like(x)
        assert _lib.load().fem_tangent_matvec(mesh.ctx, ptr(x), ptr(y)) == 0
        ys.append(y)
    for o in outs[1:]:
        assert torch.equal(o, outs[0])
    for o in ys[1:]:
        assert torch.equal(o, ys[0])


@pytest.mark.parametrize("block_size", [256, 512, 768, 1024])
def test_element_block_sizes_match_oracle_and_repeat_bitwise(cuda, vox, block_size):
    # every block size gives the oracle's product; small blocks make most
    # nodes shared between blocks (completed by the last contributing block)
    ref = np.load(G.path_of("vox12_j2_forces"))
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mesh.set_matvec_variant("element_block", block_size=block_size)
    mat = make_material("j2", E=vox.E)
    mesh.u.copy_(dev(ref["u"], cuda))
    mat.compute_nodal_forces(mesh)
    x = dev(ref["p"], cuda, torch.float32)
    ys = []
    for _ in range(3):
        y = torch.full_like(x, float("nan"))
        assert _lib.load().fem_tangent_matvec(mesh.ctx, ptr(x), ptr(y)) == 0, _lib.last_error(mesh.ctx)
        ys.append(y)
    assert _rel_l2(ys[0].cpu().numpy().astype(np.float64), ref["y"]) < 2e-5
    for o in ys[1:]:
        assert torch.equal(o, ys[0])
    assert mesh.stats()["element_block_size"] == block_size


def test_element_block_size_option_is_validated(cuda, vox):
    mesh = make_mesh(vox.X, vox.conn, cuda)
    lib = _lib.load()
    assert lib.fem_set_option(mesh.ctx, _lib.FEM_OPT_EB_SIZE, 300) == _lib.FEM_ERR_INVALID
    assert "element block size" in _lib.last_error(mesh.ctx)
    assert lib.fem_set_option(mesh.ctx, _lib.FEM_OPT_EB_SIZE, 0) == 0


def test_pcg_solves_tangent_system(cuda, bar):
    mesh = make_mesh(bar.X, bar.conn, cuda)
    mat = B.LinearElastic(17e3, 0.3)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    mat.compute_nodal_forces(mesh)
    lib = _lib.load()
    r = dev(bar.f_ext, cuda)
    du = torch.zeros_like(r)
    it = C.c_int32()
    rel = C.c_double()
    rc = lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_JACOBI, ptr(r), ptr(du), 1e-6, 5000, C.byref(it), C.byref(rel))
    assert rc == 0, _lib.last_error(mesh.ctx)
    assert 0 < it.value < 5000 and rel.value <= 1e-6
    # FP64 oracle: linear elasticity solved directly
    m = O.Mesh(bar.X, bar.conn)
    u_ref, _ = O.consistent_newton(m, O.Material("linear_elastic", E=17e3, nu=0.3), bar.f_ext,
                                   bar.fixed_mask, bar.fixed_vals, tol=1e-12, line_search=False)
    assert _rel_l2(du.cpu().numpy(), u_ref) < 1e-4
    # unpreconditioned CG converges too (more iterations)
    it2 = C.c_int32()
    rc = lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_NONE, ptr(r), ptr(du), 1e-6, 20000, C.byref(it2), C.byref(rel))
    assert rc == 0 and it2.value > 0


@pytest.mark.parametrize("bf16", [False, True])
def test_two_level_pcg_matches_oracle_with_fewer_iterations(cuda, vox, bf16):
    """Jacobi + trilinear Galerkin coarse correction: same solution as the
    FP64 oracle, fewer CG iterations than Jacobi alone; the coarse inverse
    stored in FP32 or BF16."""
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mat = B.LinearElastic(1e3, 0.3)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    mat.compute_nodal_forces(mesh)
    mesh.set_coarse_options(cell=4, bf16=bf16)   # 3x3x3 cells on this 12^3-voxel body
    lib = _lib.load()
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal(vox.X.shape)
    rhs[vox.fixed_mask] = 0.0
    r = dev(rhs, cuda)
    its = {}
    sols = {}
    for name, pc in (("jacobi", _lib.FEM_PRECOND_JACOBI), ("two_level", _lib.FEM_PRECOND_TWO_LEVEL)):
        du = torch.zeros_like(r)
        it = C.c_int32()
        rel = C.c_double()
        rc = lib.fem_pcg(mesh.ctx, pc, ptr(r), ptr(du), 1e-7, 20000, C.byref(it), C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        assert rel.value <= 1e-7
        its[name] = it.value
        sols[name] = du.cpu().numpy()
    info = mesh.coarse_info()
    assert info["assemblies"] == 1 and info["coarse_dofs"] > 0
    assert its["two_level"] < 0.6 * its["jacobi"], its
    # FP64 oracle: K_ff du = rhs_f by a direct solve of the assembled tangent
    m = O.Mesh(vox.X, vox.conn)
    mo = O.Material("linear_elastic", E=1e3, nu=0.3)
    F = O.deformation_gradient(np.zeros_like(vox.X), vox.conn.astype(np.int64), m.dNdX)
    u_ref = O.solve_tangent(mo, F, None, m, rhs, vox.fixed_mask)
    for name in sols:
        assert _rel_l2(sols[name], u_ref) < 1e-5, name


@pytest.mark.parametrize("cell", [3, 4])
def test_bf16_packed_coarse_inverse_tracks_fp32(cuda, vox, cell):
    """The packed BF16 coarse inverse (lower block triangle of 64 x 64 tiles,
    both products from one read of a tile) preconditions like the FP32 one:
    about as many PCG iterations, same solution.  Both lattices give coarse
    DOF counts (240, 144) that leave the last tile row and column partly
    padding."""
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mat = B.LinearElastic(1e3, 0.3)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    mat.compute_nodal_forces(mesh)
    lib = _lib.load()
    rng = np.random.default_rng(21)
    rhs = rng.standard_normal(vox.X.shape)
    rhs[vox.fixed_mask] = 0.0
    r = dev(rhs, cuda)
    its, sols = {}, {}
    for bf in (False, True):
        mesh.set_coarse_options(cell=cell, bf16=bf)
        for rep in range(2):
            du = torch.zeros_like(r)
            it = C.c_int32()
            rel = C.c_double()
            rc = lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_TWO_LEVEL, ptr(r), ptr(du), 1e-7, 20000, C.byref(it),
                             C.byref(rel))
            assert rc == 0, _lib.last_error(mesh.ctx)
            its[(bf, rep)] = it.value
        sols[bf] = du.cpu().numpy()
    assert mesh.coarse_info()["coarse_dofs"] % 64 != 0
    assert its[(True, 0)] == its[(True, 1)]          # deterministic
    assert its[(True, 0)] <= 1.15 * its[(False, 0)] + 2, its
    assert _rel_l2(sols[True], sols[False]) < 1e-5


@pytest.mark.parametrize("pc", ["jacobi", "two_level"])
def test_programmatic_launch_is_bitwise_neutral(cuda, vox, pc):
    """Programmatic dependent launches between the CG kernels change when a
    kernel is scheduled, not what it computes: the same iterations and the
    bitwise same solution with and without them."""
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mat = B.LinearElastic(1e3, 0.3)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    mat.compute_nodal_forces(mesh)
    mesh.set_coarse_options(cell=4)
    lib = _lib.load()
    rng = np.random.default_rng(31)
    rhs = rng.standard_normal(vox.X.shape)
    rhs[vox.fixed_mask] = 0.0
    r = dev(rhs, cuda)
    code = {"jacobi": _lib.FEM_PRECOND_JACOBI, "two_level": _lib.FEM_PRECOND_TWO_LEVEL}[pc]
    out = {}
    for on in (True, False):
        mesh.set_programmatic_launch(on)
        du = torch.zeros_like(r)
        it = C.c_int32()
        rel = C.c_double()
        rc = lib.fem_pcg(mesh.ctx, code, ptr(r), ptr(du), 1e-7, 20000, C.byref(it), C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        assert mesh.step_info()[f"{pc}_graph_pdl"] == on
        out[on] = (du.cpu().numpy(), it.value)
    assert out[True][1] == out[False][1]
    assert np.array_equal(out[True][0], out[False][0])


def test_direction_recurrence_matches_direction_kernel(cuda, vox):
    """Two-level PCG with the direction formed by recurrence in the matvec's
    node gather (K p = K z + beta K p_old) solves to the same displacement,
    in about the same iterations, as with the direction-update kernel; both
    match the FP64 oracle."""
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mat = B.LinearElastic(1e3, 0.3)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    mat.compute_nodal_forces(mesh)
    mesh.set_coarse_options(cell=4)
    mesh.set_matvec_variant("two_phase")
    lib = _lib.load()
    rng = np.random.default_rng(41)
    rhs = rng.standard_normal(vox.X.shape)
    rhs[vox.fixed_mask] = 0.0
    r = dev(rhs, cuda)
    out = {}
    for on in (True, False):
        mesh.set_direction_recurrence(on)
        du = torch.zeros_like(r)
        it = C.c_int32()
        rel = C.c_double()
        rc = lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_TWO_LEVEL, ptr(r), ptr(du), 1e-7, 20000, C.byref(it),
                         C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        assert rel.value <= 1e-7
        out[on] = (du.cpu().numpy(), it.value)
    assert abs(out[True][1] - out[False][1]) <= max(2, 0.05 * out[False][1]), (out[True][1], out[False][1])
    m = O.Mesh(vox.X, vox.conn)
    F = O.deformation_gradient(np.zeros_like(vox.X), vox.conn.astype(np.int64), m.dNdX)
    u_ref = O.solve_tangent(O.Material("linear_elastic", E=1e3, nu=0.3), F, None, m, rhs, vox.fixed_mask)
    for on in out:
        assert _rel_l2(out[on][0], u_ref) < 1e-5, on


@pytest.mark.parametrize("material", ["le", "j2"])
def test_block_smoother_matches_oracle_with_no_more_iterations(cuda, vox, material):
    """Two-level PCG with the nodal 3x3 block-inverse smoother and with the
    diagonal smoother reach the FP64 oracle's solution; the block smoother
    needs no more iterations.  J2 at a plastic state checks the block of the
    consistent elasto-plastic tangent."""
    mesh = make_mesh(vox.X, vox.conn, cuda)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    if material == "le":
        mat = B.LinearElastic(1e3, 0.3)
        mesh.set_fixed_dofs(idx, np.zeros(idx.size))
        mat.compute_nodal_forces(mesh)
    else:
        ref = np.load(G.path_of("vox12_j2_steps"))
        mat = make_material("j2", E=vox.E)
        lf = float(ref["load_factor"])
        vals = vox.fixed_vals * lf / int(ref["n_total"])
        mesh.set_fixed_dofs(idx, vals.reshape(-1)[idx])
        res = B.StaticSolver(mesh, mat, tol=1e-10, precond="two_level").solve(verbose=False)
        assert res["converged"], res
        mesh.set_fixed_dofs(idx, np.zeros(idx.size))
        mat.compute_nodal_forces(mesh)
    mesh.set_coarse_options(cell=4)
    lib = _lib.load()
    rng = np.random.default_rng(51)
    rhs = rng.standard_normal(vox.X.shape)
    rhs[vox.fixed_mask] = 0.0
    r = dev(rhs, cuda)
    out = {}
    for on in (True, False):
        mesh.set_block_smoother(on)
        du = torch.zeros_like(r)
        it = C.c_int32()
        rel = C.c_double()
        rc = lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_TWO_LEVEL, ptr(r), ptr(du), 1e-8, 20000, C.byref(it),
                         C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        out[on] = (du.cpu().numpy(), it.value)
    assert out[True][1] <= out[False][1], (out[True][1], out[False][1])
    assert _rel_l2(out[True][0], out[False][0]) < 1e-5
    if material == "le":
        m = O.Mesh(vox.X, vox.conn)
        F = O.deformation_gradient(np.zeros_like(vox.X), vox.conn.astype(np.int64), m.dNdX)
        u_ref = O.solve_tangent(O.Material("linear_elastic", E=1e3, nu=0.3), F, None, m, rhs, vox.fixed_mask)
        assert _rel_l2(out[True][0], u_ref) < 1e-6


def test_coarse_inverse_methods_agree(cuda, vox):
    """The coarse inverse formed as W^T W with W = L^-1 (cuBLAS trsm + syrk)
    and by cuSOLVER potri precondition alike: the same solution, iteration
    counts within one."""
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mat = B.LinearElastic(1e3, 0.3)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    mat.compute_nodal_forces(mesh)
    lib = _lib.load()
    rng = np.random.default_rng(61)
    rhs = rng.standard_normal(vox.X.shape)
    rhs[vox.fixed_mask] = 0.0
    r = dev(rhs, cuda)
    out = {}
    for method in ("potri", "trsm_syrk"):
        mesh.set_coarse_options(cell=3, bf16=False, inverse=method, reuse=1)
        du = torch.zeros_like(r)
        it = C.c_int32()
        rel = C.c_double()
        rc = lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_TWO_LEVEL, ptr(r), ptr(du), 1e-8, 20000, C.byref(it),
                         C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        out[method] = (du.cpu().numpy(), it.value)
    assert abs(out["potri"][1] - out["trsm_syrk"][1]) <= 1, out
    assert _rel_l2(out["potri"][0], out["trsm_syrk"][0]) < 1e-6


@pytest.mark.parametrize("inverse", ["trsm_syrk_f32", "trsm_syrk_tf32"])
def test_single_precision_coarse_inverse_tracks_fp64(cuda, vox, inverse):
    """The coarse inverse formed in FP32 (and with TF32 tensor-core trsm /
    syrk) for the BF16 packed copy preconditions like the FP64 one: the same
    solution, iterations within 10 %; the node cap bounds the lattice."""
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mat = B.LinearElastic(1e3, 0.3)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    mat.compute_nodal_forces(mesh)
    lib = _lib.load()
    rng = np.random.default_rng(81)
    rhs = rng.standard_normal(vox.X.shape)
    rhs[vox.fixed_mask] = 0.0
    r = dev(rhs, cuda)
    out = {}
    for method in ("trsm_syrk", inverse):
        mesh.set_coarse_options(cell=3, bf16=True, inverse=method, reuse=1)
        du = torch.zeros_like(r)
        it = C.c_int32()
        rel = C.c_double()
        rc = lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_TWO_LEVEL, ptr(r), ptr(du), 1e-8, 20000, C.byref(it),
                         C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        out[method] = (du.cpu().numpy(), it.value)
    assert out[inverse][1] <= 1.1 * out["trsm_syrk"][1] + 1, out
    assert _rel_l2(out[inverse][0], out["trsm_syrk"][0]) < 1e-6
    mesh.set_coarse_options(cell=1, max_nodes=64)
    du = torch.zeros_like(r)
    it, rel = C.c_int32(), C.c_double()
    assert lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_TWO_LEVEL, ptr(r), ptr(du), 1e-8, 20000, C.byref(it),
                       C.byref(rel)) == 0
    info = mesh.coarse_info()
    assert 0 < info["coarse_nodes"] <= 64 and info["cell_edge"] > 1.0


def test_two_level_without_spd_coarse_operator_falls_back_to_jacobi(cuda):
    """Lattice cells finer than the elements of an anisotropic mesh (1.25 mm
    hexes, ~1 mm cells) give a singular coarse operator: the two-level solve
    runs as Jacobi-PCG, counts the fallback and still reaches the FP64
    oracle's solution."""
    bar = meshgen.cantilever_bar(nx=8, ny=2, nz=2)
    mesh = make_mesh(bar.X, bar.conn, cuda)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    mat = B.LinearElastic(1e3, 0.3)
    mat.compute_nodal_forces(mesh)
    mesh.set_coarse_options(cell=2, reuse=-1)
    rng = np.random.default_rng(71)
    rhs = rng.standard_normal(bar.X.shape)
    rhs[bar.fixed_mask] = 0.0
    r = dev(rhs, cuda)
    du = torch.zeros_like(r)
    it, rel = C.c_int32(), C.c_double()
    rc = _lib.load().fem_pcg(mesh.ctx, _lib.FEM_PRECOND_TWO_LEVEL, ptr(r), ptr(du), 1e-8, 20000, C.byref(it),
                             C.byref(rel))
    assert rc == 0, _lib.last_error(mesh.ctx)
    assert mesh.coarse_info()["jacobi_fallbacks"] >= 1
    m = O.Mesh(bar.X, bar.conn)
    F = O.deformation_gradient(np.zeros_like(bar.X), bar.conn.astype(np.int64), m.dNdX)
    u_ref = O.solve_tangent(O.Material("linear_elastic", E=1e3, nu=0.3), F, None, m, rhs, bar.fixed_mask)
    assert _rel_l2(du.cpu().numpy(), u_ref) < 1e-5


def _pcg_fused_vs_chain(mesh, pc, rhs, cuda, rtol):
    lib = _lib.load()
    mesh.set_block_smoother(False)   # the fused step applies the diagonal smoother
    r = dev(rhs, cuda)
    out = {}
    for fused in (True, False):
        mesh.set_fused_step(fused)
        du = torch.zeros_like(r)
        it = C.c_int32()
        rel = C.c_double()
        rc = lib.fem_pcg(mesh.ctx, pc, ptr(r), ptr(du), rtol, 20000, C.byref(it), C.byref(rel))
        assert rc == 0, _lib.last_error(mesh.ctx)
        assert rel.value <= rtol
        info = mesh.step_info()
        key = "two_level_graph_fused" if pc == _lib.FEM_PRECOND_TWO_LEVEL else "jacobi_graph_fused"
        assert info[key] == fused, info
        out[fused] = (du.cpu().numpy(), it.value)
    return out


@pytest.mark.parametrize("pc", ["jacobi", "two_level"])
def test_fused_step_matches_kernel_chain(cuda, vox, pc):
    """The cooperative fused CG step (one kernel after each matvec, grid-wide
    barriers) and the chain of kernels solve to the same displacement in
    about the same number of iterations; both match the FP64 oracle."""
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mat = B.LinearElastic(1e3, 0.3)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    mat.compute_nodal_forces(mesh)
    mesh.set_coarse_options(cell=4)
    rng = np.random.default_rng(11)
    rhs = rng.standard_normal(vox.X.shape)
    rhs[vox.fixed_mask] = 0.0
    code = {"jacobi": _lib.FEM_PRECOND_JACOBI, "two_level": _lib.FEM_PRECOND_TWO_LEVEL}[pc]
    out = _pcg_fused_vs_chain(mesh, code, rhs, cuda, 1e-7)
    (u_f, it_f), (u_c, it_c) = out[True], out[False]
    assert abs(it_f - it_c) <= max(2, 0.05 * it_c), (it_f, it_c)
    m = O.Mesh(vox.X, vox.conn)
    F = O.deformation_gradient(np.zeros_like(vox.X), vox.conn.astype(np.int64), m.dNdX)
    u_ref = O.solve_tangent(O.Material("linear_elastic", E=1e3, nu=0.3), F, None, m, rhs, vox.fixed_mask)
    assert _rel_l2(u_f, u_ref) < 1e-5
    assert _rel_l2(u_c, u_ref) < 1e-5


def test_fused_step_grid_stride_on_larger_mesh(cuda):
    """A mesh with more nodes than the fused step's grid has threads (every
    vector phase loops): fused and chained two-level PCG agree."""
    v = meshgen.vertebral_body(n=80, seed=3)
    mesh = make_mesh(v.X, v.conn, cuda)
    assert v.n_nodes > 2 * 148 * 512
    mat = B.LinearElastic(1e3, 0.3)
    idx = np.where(v.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, np.zeros(idx.size))
    mat.compute_nodal_forces(mesh)
    rng = np.random.default_rng(12)
    rhs = rng.standard_normal(v.X.shape)
    rhs[v.fixed_mask] = 0.0
    out = _pcg_fused_vs_chain(mesh, _lib.FEM_PRECOND_TWO_LEVEL, rhs, cuda, 1e-6)
    (u_f, it_f), (u_c, it_c) = out[True], out[False]
    assert abs(it_f - it_c) <= max(3, 0.05 * it_c), (it_f, it_c)
    assert _rel_l2(u_f, u_c) < 1e-4


@pytest.mark.parametrize("reuse", [0, 1, -1])
def test_newton_j2_two_level_matches_oracle(cuda, vox, reuse):
    """reuse 0: one coarse operator for the whole load path; 1: rebuilt for
    every PCG solve; -1: adaptive refresh."""
    ref = np.load(G.path_of("vox12_j2_steps"))
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mesh.set_coarse_options(reuse=reuse)
    mat = make_material("j2", E=vox.E)
    lf = float(ref["load_factor"])
    total = int(ref["n_total"])
    solver = B.StaticSolver(mesh, mat, tol=1e-10, precond="two_level")
    for k in range(ref["u_steps"].shape[0]):
        vals = vox.fixed_vals * (k + 1) / total * lf
        idx = np.where(vox.fixed_mask.reshape(-1))[0]
        mesh.set_fixed_dofs(idx, vals.reshape(-1)[idx])
        res = solver.solve(verbose=False)
        assert res["converged"], res
        assert _rel_l2(mesh.get_displacements(), ref["u_steps"][k]) < 1e-6
    n_asm = mesh.coarse_info()["assemblies"]
    assert n_asm >= (ref["u_steps"].shape[0] if reuse == 1 else 1)
    if reuse == 0:
        assert n_asm == 1


@pytest.mark.parametrize("precond", ["jacobi", "two_level"])
def test_newton_bar_matches_oracle(cuda, bar, precond):
    # the plain-method cantilever workload as specified: ten traction load
    # steps, each to 1e-10, every step within 1e-6 of the FP64 oracle (the
    # last steps are the large-rotation ones: tip deflection 5.7 mm on 10 mm)
    ref = np.load(G.path_of("bar_nh_steps"))
    assert ref["u_steps"].shape[0] == 10
    mesh = make_mesh(bar.X, bar.conn, cuda)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    solver = B.StaticSolver(mesh, B.NeoHookean(17e3, 0.3), tol=1e-10, precond=precond)
    for k in range(ref["u_steps"].shape[0]):
        mesh.set_nodal_forces(np.arange(bar.n_nodes), bar.f_ext * (k + 1) / 10.0)
        res = solver.solve(verbose=False)
        assert res["converged"], res
        assert res["relative_residual"] < 1e-10
        assert _rel_l2(mesh.get_displacements(), ref["u_steps"][k]) < 1e-6


def test_newton_bar_with_extrapolation_matches_oracle(cuda, bar):
    # force-controlled steps (no prescribed-value change): the extrapolated
    # start still measures convergence against the previous state's residual
    # under the new load, and every step lands within 1e-6 of the oracle
    ref = np.load(G.path_of("bar_nh_steps"))
    mesh = make_mesh(bar.X, bar.conn, cuda)
    mesh.set_extrapolation(True)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    solver = B.StaticSolver(mesh, B.NeoHookean(17e3, 0.3), tol=1e-10)
    newton = []
    for k in range(ref["u_steps"].shape[0]):
        mesh.set_nodal_forces(np.arange(bar.n_nodes), bar.f_ext * (k + 1) / 10.0)
        res = solver.solve(verbose=False)
        assert res["converged"], res
        assert res["relative_residual"] < 1e-10
        assert _rel_l2(mesh.get_displacements(), ref["u_steps"][k]) < 1e-6
        newton.append(res["iterations"])
    assert sum(newton[1:]) > 0


@pytest.mark.parametrize("variant", VARIANTS)
def test_newton_j2_steps_match_oracle(cuda, vox, variant):
    ref = np.load(G.path_of("vox12_j2_steps"))
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mesh.set_matvec_variant(variant)
    mat = make_material("j2", E=vox.E)
    lf = float(ref["load_factor"])
    total = int(ref["n_total"])
    solver = B.StaticSolver(mesh, mat, tol=1e-10)
    for k in range(ref["u_steps"].shape[0]):
        vals = vox.fixed_vals * (k + 1) / total * lf
        idx = np.where(vox.fixed_mask.reshape(-1))[0]
        mesh.set_fixed_dofs(idx, vals.reshape(-1)[idx])
        res = solver.solve(verbose=False)
        assert res["converged"], res
        assert _rel_l2(mesh.get_displacements(), ref["u_steps"][k]) < 1e-6
        epe_ref = ref["epe_steps"][k]
        assert np.max(np.abs(mat.get_plastic_strain() - epe_ref)) <= 1e-6 * max(epe_ref.max(), 1e-12) + 1e-12
    assert ref["epe_steps"][-1].max() > 0


def test_newton_j2_steps_with_extrapolation_match_oracle(cuda, vox):
    """Load-step extrapolation changes where Newton starts, not what it
    converges to: every step within 1e-6 of the FP64 oracle, and the steps
    after the first start from the extrapolated state (no predictor solve)."""
    ref = np.load(G.path_of("vox12_j2_steps"))
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mesh.set_extrapolation(True)
    mat = make_material("j2", E=vox.E)
    lf = float(ref["load_factor"])
    total = int(ref["n_total"])
    solver = B.StaticSolver(mesh, mat, tol=1e-10)
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    evals = []
    for k in range(ref["u_steps"].shape[0]):
        vals = vox.fixed_vals * (k + 1) / total * lf
        mesh.set_fixed_dofs(idx, vals.reshape(-1)[idx])
        res = solver.solve(verbose=False)
        assert res["converged"], res
        assert _rel_l2(mesh.get_displacements(), ref["u_steps"][k]) < 1e-6
        evals.append(res["residual_evals"])
    # the first step runs the predictor (two residuals before Newton), the
    # extrapolated ones evaluate the reference's first residual only once
    assert ref["u_steps"].shape[0] >= 2


def test_matvec_variants_agree_and_autotuner_times_both(cuda, vox):
    ref = np.load(G.path_of("vox12_j2_forces"))
    mesh = make_mesh(vox.X, vox.conn, cuda)
    mat = make_material("j2", E=vox.E)
    mesh.u.copy_(dev(ref["u"], cuda))
    mat.compute_nodal_forces(mesh)
    x = dev(ref["p"], cuda, torch.float32)
    ys = {}
    for v in VARIANTS:
        mesh.set_matvec_variant(v)
        y = torch.empty_like(x)
        assert _lib.load().fem_tangent_matvec(mesh.ctx, ptr(x), ptr(y)) == 0
        ys[v] = y.cpu().numpy().astype(np.float64)
    # fused and two-phase sum each node's slot vectors in the same order (only
    # FMA contraction may differ); the element-block kernel sums per block,
    # then the blocks' partial rows in block order: FP32 rounding apart
    assert _rel_l2(ys["two_phase"], ys["fused"]) < 1e-6
    assert _rel_l2(ys["element_block"], ys["fused"]) < 1e-6
    assert _rel_l2(ys["warp_agg"], ys["fused"]) < 1e-6
    # the persistent pair evaluates the same elements and sums in the same order
    assert np.array_equal(ys["persistent"], ys["two_phase"])
    # automatic choice: the first PCG solve times every variant (the element
    # block at each candidate size) and keeps the fastest
    mesh.set_matvec_variant(None)
    mesh.u.zero_()
    mat.reset_state()
    idx = np.where(vox.fixed_mask.reshape(-1))[0]
    mesh.set_fixed_dofs(idx, (vox.fixed_vals * 0.01).reshape(-1)[idx])
    res = B.StaticSolver(mesh, mat, tol=1e-8).solve(verbose=False)
    assert res["converged"], res
    st = mesh.stats()
    assert st["matvec_tuned"]
    assert all(v > 0 for v in st["matvec_ns"].values()), st
    assert all(v > 0 for v in st["element_block_ns"].values()), st
    faster = min(st["matvec_ns"], key=st["matvec_ns"].get)
    assert st["matvec_variant"] == faster
    assert st["matvec_ns"]["element_block"] == min(st["element_block_ns"].values())
    if faster == "element_block":
        assert st["element_block_size"] == min(st["element_block_ns"], key=st["element_block_ns"].get)
    # every PCG solve ran as one whole-solve graph launch (conditional WHILE node)
    assert st["whole_solve_graph_available"] and st["whole_solve_graphs"] > 0
    assert _lib.load().fem_set_option(mesh.ctx, _lib.FEM_OPT_MATVEC_VARIANT, 7) == _lib.FEM_ERR_INVALID
    assert "matvec variant" in _lib.last_error(mesh.ctx)


def test_reference_line_search_policy_converges(cuda, bar):
    mesh = make_mesh(bar.X, bar.conn, cuda)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    mesh.set_nodal_forces(np.arange(bar.n_nodes), bar.f_ext / 10.0)
    solver = B.StaticSolver(mesh, B.NeoHookean(17e3, 0.3), tol=1e-10, line_search="reference")
    res = solver.solve(verbose=False)
    ref = np.load(G.path_of("bar_nh_steps"))
    assert res["converged"]
    assert _rel_l2(mesh.get_displacements(), ref["u_steps"][0]) < 1e-6


def test_single_element_and_unit_volume(cuda):
    X = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    conn = np.array([[0, 1, 2, 3]], dtype=np.int32)
    mesh = make_mesh(X, conn, cuda)
    assert mesh.elem_vol.item() == pytest.approx(1.0 / 6.0, rel=1e-14)
    u = np.array([[0.0, 0, 0], [0.01, 0, 0], [0, -0.003, 0], [0.001, 0, 0.002]])
    mesh.u.copy_(dev(u, cuda))
    mat = B.NeoHookean(1e3, 0.3)
    mat.compute_nodal_forces(mesh)
    m = O.Mesh(X, conn)
    f_ref = O.internal_state(m, O.Material("neo_hookean", E=1e3, nu=0.3), u)[3]
    assert _rel_max(mesh.get_nodal_forces(), f_ref) < 1e-12
    # sum of internal forces vanishes (equilibrium of a free element)
    assert np.abs(mesh.get_nodal_forces().sum(axis=0)).max() < 1e-12


def test_inverted_element_orientation_is_handled(cuda):
    # negatively oriented connectivity: volumes via |det J|, forces identical
    X = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    u = np.array([[0.0, 0, 0], [0.01, 0, 0], [0, -0.003, 0], [0.001, 0, 0.002]])
    out = []
    for conn in (np.array([[0, 1, 2, 3]], np.int32), np.array([[0, 2, 1, 3]], np.int32)):
        mesh = make_mesh(X, conn, cuda)
        mesh.u.copy_(dev(u, cuda))
        B.NeoHookean(1e3, 0.3).compute_nodal_forces(mesh)
        out.append(mesh.get_nodal_forces())
    assert _rel_max(out[1], out[0]) < 1e-12


def test_invalid_inputs_raise(cuda):
    X = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    with pytest.raises(B.FEAValidationError):
        make_mesh(X, np.array([[0, 1, 2, 4]], np.int32), cuda)
    with pytest.raises(B.FEAValidationError):
        make_mesh(X, np.array([[0, 1, 1, 3]], np.int32), cuda)
    with pytest.raises(B.FEAValidationError):
        B.NeoHookean(1e3, 0.5)
    with pytest.raises(B.FEAValidationError):
        B.J2Plasticity(1e3, 0.3, -1.0)
    mesh = make_mesh(X, np.array([[0, 1, 2, 3]], np.int32), cuda)
    with pytest.raises(B.FEAValidationError):
        mesh.set_fixed_nodes(np.array([7]))
    lib = _lib.load()
    x = torch.zeros(4, 3, dtype=torch.float32, device=cuda)
    # matvec before any residual evaluation: state error, not a fault
    assert lib.fem_tangent_matvec(mesh.ctx, ptr(x), ptr(x)) == _lib.FEM_ERR_STATE


def test_nan_load_raises_convergence_error(cuda, bar):
    # fault injected on the host: a NaN in the external force
    mesh = make_mesh(bar.X, bar.conn, cuda)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    f = bar.f_ext.copy()
    f[-1, 2] = np.nan
    mesh.set_nodal_forces(np.arange(bar.n_nodes), f)
    solver = B.StaticSolver(mesh, B.NeoHookean(17e3, 0.3))
    with pytest.raises(B.FEAConvergenceError) as ei:
        solver.solve(verbose=False)
    assert ei.value.reason == "nan_divergence"


def test_progress_callback_cancels(cuda, bar):
    mesh = make_mesh(bar.X, bar.conn, cuda)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    mesh.set_nodal_forces(np.arange(bar.n_nodes), bar.f_ext / 10.0)
    seen = []

    def cb(info):
        seen.append(info)
        return info["iteration"] < 1

    res = B.StaticSolver(mesh, B.NeoHookean(17e3, 0.3), tol=1e-10).solve(verbose=False, progress_callback=cb)
    assert res.get("cancelled") and res["iterations"] == 1 and not res["converged"]
    assert [s["iteration"] for s in seen] == [0, 1]


def test_multi_material_table(cuda, bar):
    # two materials by element id: the residual honours both (no first-material quirk)
    ids = (bar.X[bar.conn].mean(axis=1)[:, 0] > 5.0).astype(np.int32)
    mesh = B.FEMesh(bar.n_nodes, bar.n_elements, device=cuda)
    mesh.initialize_from_numpy(bar.X, bar.conn, material_ids=ids)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    mesh.set_nodal_forces(np.arange(bar.n_nodes), bar.f_ext / 100.0)
    solver = B.StaticSolver(mesh, materials={0: B.NeoHookean(17e3, 0.3), 1: B.NeoHookean(4e3, 0.3)}, tol=1e-10)
    res = solver.solve(verbose=False)
    assert res["converged"]
    m = O.Mesh(bar.X, bar.conn)
    E = np.where(ids == 1, 4e3, 17e3)
    u_ref, _ = O.consistent_newton(m, O.Material("neo_hookean", E=E, nu=0.3), bar.f_ext / 100.0,
                                   bar.fixed_mask, bar.fixed_vals, tol=1e-11, line_search=False)
    assert _rel_l2(mesh.get_displacements(), u_ref) < 1e-6
