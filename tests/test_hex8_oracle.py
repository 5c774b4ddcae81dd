"""HEX8 oracle and generators on the CPU: the known answers of the
reference's own HEX8 tests (backend/fea/fem/tests/test_hex8.py) restated for
the oracle, a patch test, exact uniaxial compression, J2 elastic == linear
elastic, and the reference's FEMAdapter / voxel_to_hex numbering."""
import numpy as np
import pytest

from oracle import fem_oracle as O
from simul_b200 import meshgen

UNIT_CUBE = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                      [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)


def test_shape_functions_partition_unity_and_kronecker():
    # test_hex8.py:20-49
    rng = np.random.default_rng(0)
    for xi in rng.uniform(-1, 1, (10, 3)):
        assert np.sum(O.hex8_N(xi)) == pytest.approx(1.0, abs=1e-12)
        assert np.abs(O.hex8_dN_dxi(xi).sum(axis=0)).max() < 1e-12   # test_hex8.py:51-66
    for a in range(8):
        N = O.hex8_N(O.HEX8_SIGNS[a])
        assert np.allclose(N, np.eye(8)[a], atol=1e-12)


def test_gauss_rule_and_cube_volumes():
    # test_hex8.py:72-157: 8 points of weight 1; unit cube 1, 2 x 3 x 4 box 24
    m = O.Mesh(UNIT_CUBE, np.arange(8)[None])
    assert m.vol.shape == (8,) and m.dNdX.shape == (8, 8, 3)
    assert m.elem_vol[0] == pytest.approx(1.0, rel=1e-12)
    assert np.allclose(m.vol, 0.125)
    box = O.Mesh(UNIT_CUBE * np.array([2.0, 3.0, 4.0]), np.arange(8)[None])
    assert box.elem_vol[0] == pytest.approx(24.0, rel=1e-12)


def test_deformation_gradient_identity_and_patch():
    # test_hex8.py:159-188 (F = I at u = 0 at all 8 points), and a linear
    # field reproduced exactly on a distorted element
    rng = np.random.default_rng(1)
    X = UNIT_CUBE + 0.1 * rng.standard_normal((8, 3))
    m = O.Mesh(X, np.arange(8)[None])
    F0 = O.deformation_gradient(np.zeros((8, 3)), m.qconn, m.dNdX)
    assert F0.shape == (8, 3, 3) and np.allclose(F0, np.eye(3), atol=1e-14)
    A = 0.01 * rng.standard_normal((3, 3))
    F = O.deformation_gradient(X @ A.T, m.qconn, m.dNdX)
    assert np.abs(F - (np.eye(3) + A)).max() < 1e-13


def test_structured_grid_numbering_follows_fem_adapter():
    # framework/_adapters/fem_adapter.py:41-70
    X, conn = meshgen.structured_hex8(3, 2, 2, (3.0, 2.0, 2.0))
    assert X.shape == (4 * 3 * 3, 3) and conn.shape == (12, 8)
    nx, ny = 3, 2
    n0 = 1 + 1 * (nx + 1) + 1 * (nx + 1) * (ny + 1)           # element ex=1, ey=1, ez=1
    e = 1 + 1 * nx + 1 * nx * ny
    n4 = n0 + (nx + 1) * (ny + 1)
    assert conn[e].tolist() == [n0, n0 + 1, n0 + nx + 2, n0 + nx + 1, n4, n4 + 1, n4 + nx + 2, n4 + nx + 1]
    assert np.allclose(X[n0], [1.0, 1.0, 1.0])
    m = O.Mesh(X, conn)
    assert m.vol.min() > 0 and m.elem_vol.sum() == pytest.approx(12.0)


def test_voxels_to_hex_mesh_merges_shared_corners():
    # preprocessing/voxel_to_hex.py:11-68: two face-adjacent voxels share 4 nodes
    X, conn = meshgen.voxels_to_hex_mesh(np.array([[0.5, 0.5, 0.5], [1.5, 0.5, 0.5]]), [1.0, 1.0, 1.0])
    assert X.shape == (12, 3) and conn.shape == (2, 8)
    assert len(set(conn[0]) & set(conn[1])) == 4
    # nodes ascend lexicographically in (x, y, z)
    assert np.all(np.diff(X[:, 0]) >= 0)
    for e in range(2):
        assert np.allclose(X[conn[e]], np.array([[0.5, 0.5, 0.5]]) + [e, 0, 0] + 0.5 * O.HEX8_SIGNS)
    empty = meshgen.voxels_to_hex_mesh(np.empty((0, 3)), [1.0, 1.0, 1.0])
    assert empty[0].shape == (0, 3) and empty[1].shape == (0, 8)


def _uniaxial_cube(n=2, strain=-0.01):
    X, conn = meshgen.structured_hex8(n, n, n)
    fixed = np.zeros_like(X, dtype=bool)
    vals = np.zeros_like(X)
    fixed[np.isclose(X[:, 0], 0.0), 0] = True
    fixed[np.isclose(X[:, 1], 0.0), 1] = True
    fixed[np.isclose(X[:, 2], 0.0), 2] = True
    top = np.isclose(X[:, 2], 1.0)
    fixed[top, 2] = True
    vals[top, 2] = strain
    return X, conn, fixed, vals


def test_uniaxial_compression_is_exact():
    # roller supports + prescribed top displacement: the linear-elastic
    # solution is the homogeneous field u = (-nu e x, -nu e y, e z), which
    # trilinear elements reproduce exactly (benchmark_analytical.py:175-343)
    X, conn, fixed, vals = _uniaxial_cube()
    m = O.Mesh(X, conn)
    e = -0.01
    u, info = O.consistent_newton(m, O.Material("linear_elastic", E=1e3, nu=0.3), np.zeros_like(X), fixed,
                                  vals, tol=1e-12)
    assert info["converged"]
    exact = np.stack([-0.3 * e * X[:, 0], -0.3 * e * X[:, 1], e * X[:, 2]], axis=1)
    assert np.abs(u - exact).max() < 1e-12


def test_j2_elastic_regime_equals_linear_elastic_hex8():
    # test_j2_plasticity.py:167-201 on HEX8: below yield J2 == LE at rtol 1e-10
    X, conn = meshgen.structured_hex8(2, 2, 2)
    m = O.Mesh(X, conn)
    u = 1e-5 * np.random.default_rng(2).standard_normal(X.shape)
    le = O.internal_state(m, O.Material("linear_elastic", E=1e3, nu=0.3), u)[3]
    j2 = O.internal_state(m, O.Material("j2", E=1e3, nu=0.3, sigma_y=1e6, H=10.0), u,
                          O.J2State.zeros(m.n_points))[3]
    assert np.allclose(j2, le, rtol=1e-10, atol=1e-14)


def test_compression_direction_reference_case():
    # test_hex8.py:194-256: 2 x 2 x 2 grid, bottom fixed, -100 N on every top
    # node, linear elastic E = 1e6: every top node moves in -z
    X, conn = meshgen.structured_hex8(2, 2, 2, (2.0, 2.0, 2.0))
    fixed = np.zeros_like(X, dtype=bool)
    fixed[X[:, 2] < 0.1] = True
    f = np.zeros_like(X)
    top = X[:, 2] > 2.0 - 0.1
    f[top, 2] = -100.0
    u, info = O.consistent_newton(O.Mesh(X, conn), O.Material("linear_elastic", E=1e6, nu=0.3), f, fixed,
                                  np.zeros_like(X), tol=1e-10)
    assert info["converged"] and np.all(u[top, 2] < 0)


def test_hex8_vertebral_body_generator():
    vb = meshgen.vertebral_body(16, element="hex8")
    assert vb.conn.shape == (vb.info["n_voxels"], 8)
    m = O.Mesh(vb.X, vb.conn)
    h = vb.info["h"]
    assert np.allclose(m.elem_vol, h ** 3)
    assert vb.E.shape == (vb.conn.shape[0],)
    with pytest.raises(ValueError):
        meshgen.vertebral_body(8, element="tet10")


def _two_label_volume():
    lv = np.zeros((6, 5, 7), dtype=np.int16)
    lv[1:5, 1:4, 0:3] = 1          # lower body
    lv[1:5, 1:4, 3:5] = 2          # upper body, bonded on the z = 3 face
    lv[0, 0, 6] = 3                # a one-voxel label, below min_voxels
    return lv


def test_labelmap_bodies_follow_the_assembly_pipeline():
    # preprocessing/assembly.py:73-99, 207-249: per label the voxel centres
    # ijk * spacing + origin + spacing / 2, then voxels_to_hex_mesh
    lv = _two_label_volume()
    spacing, origin = np.array([0.5, 0.6, 0.7]), np.array([1.0, -2.0, 3.0])
    bodies = meshgen.labelmap_bodies(lv, spacing, origin, min_voxels=10)
    assert sorted(bodies) == [1, 2]
    X1, e1 = bodies[1]
    assert e1.shape == (36, 8) and X1.shape == (5 * 4 * 4, 3)
    c = meshgen.labelmap_voxel_centers(lv, spacing, origin, 1)
    assert np.allclose(c[0], origin + spacing / 2 + np.array([1, 1, 0]) * spacing)
    m = O.Mesh(X1, e1)
    assert np.allclose(m.elem_vol, np.prod(spacing))


def test_labelmap_hex8_bonds_labels_into_one_mesh():
    lv = _two_label_volume()
    X, conn, lab = meshgen.labelmap_hex8(lv, [1.0, 1.0, 1.0], labels=[1, 2])
    assert conn.shape == (36 + 24, 8) and np.array_equal(np.unique(lab), [1, 2])
    shared = set(conn[lab == 1].ravel()) & set(conn[lab == 2].ravel())
    assert len(shared) == 5 * 4        # the z = 3 interface nodes
    # two moduli by label, nu = 0, rollers: each layer strains uniformly, so
    # the interface moves by delta (L1 / E1) / (L1 / E1 + L2 / E2) only when
    # the labels share their interface nodes
    E = np.where(lab == 1, 1000.0, 250.0)
    fixed = np.zeros_like(X, dtype=bool)
    vals = np.zeros_like(X)
    for d in range(3):
        fixed[np.isclose(X[:, d], X[:, d].min()), d] = True
    top = np.isclose(X[:, 2], X[:, 2].max())
    fixed[top, 2] = True
    vals[top, 2] = -0.05
    u, info = O.consistent_newton(O.Mesh(X, conn), O.Material("linear_elastic", E=E, nu=0.0), np.zeros_like(X),
                                  fixed, vals, tol=1e-12)
    assert info["converged"]
    iface = np.isclose(X[:, 2], 3.0)
    c1, c2 = 3.0 / 1000.0, 2.0 / 250.0
    assert np.allclose(u[iface, 2], -0.05 * c1 / (c1 + c2), rtol=1e-10)
