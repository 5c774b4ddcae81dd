"""Input generators: sizes, conformity, orientation, load totals (CPU)."""
import numpy as np
import pytest

from oracle import fem_oracle as O
from simul_b200 import meshgen


def _max_face_share(conn):
    faces = np.sort(np.concatenate([conn[:, [0, 1, 2]], conn[:, [0, 1, 3]],
                                    conn[:, [0, 2, 3]], conn[:, [1, 2, 3]]]), axis=1)
    _, cnt = np.unique(faces, axis=0, return_counts=True)
    return cnt.max()


def test_cantilever_bar_sizes_and_load():
    bar = meshgen.cantilever_bar()
    assert bar.n_elements == 1920 and bar.n_nodes == 525
    np.testing.assert_allclose(bar.f_ext.sum(axis=0), [0.0, 0.0, -50.0], atol=1e-12)
    _, vol = O.reference_quantities(bar.X, bar.conn)
    assert vol.sum() == pytest.approx(10.0, rel=1e-12)
    assert _max_face_share(bar.conn) == 2
    assert bar.fixed_mask[np.isclose(bar.X[:, 0], 0)].all()


def test_vertebral_body_conforming_positive():
    v = meshgen.vertebral_body(n=16, seed=1)
    e = v.X[v.conn]
    det = np.einsum("ei,ei->e", np.cross(e[:, 1] - e[:, 0], e[:, 2] - e[:, 0]), e[:, 3] - e[:, 0])
    assert np.all(det > 0)
    assert _max_face_share(v.conn) == 2
    assert v.n_elements == 5 * v.info["n_voxels"]
    h = v.info["h"]
    assert np.sum(np.abs(det)) / 6 == pytest.approx(v.info["n_voxels"] * h ** 3, rel=1e-12)
    assert (v.E == 12e3).sum() == v.info["shell_elements"] > 0
    core = v.E[v.E != 12e3]
    assert 150 < np.median(core) < 600


def test_vertebral_body_full_size_counts():
    v = meshgen.vertebral_body(n=64)
    assert v.n_elements == 566000 and v.n_nodes == 121023
    top = np.isclose(v.X[:, 2], 25.0)
    assert np.allclose(v.fixed_vals[top, 2], -0.5)
    assert v.fixed_mask[np.isclose(v.X[:, 2], 0.0)].all()


def test_vertebral_body_seeded():
    a = meshgen.vertebral_body(n=12, seed=5)
    b = meshgen.vertebral_body(n=12, seed=5)
    c = meshgen.vertebral_body(n=12, seed=6)
    assert np.array_equal(a.E, b.E) and not np.array_equal(a.E, c.E)
