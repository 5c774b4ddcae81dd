"""The contact restatement (oracle/contact_oracle.py) against outputs of the
reference's own contact.py (tests/golden/ref_contact.npz), and the staggered
loop on oracle bodies (CPU)."""
import numpy as np
import pytest

from oracle import contact_oracle as CO
from oracle import fem_oracle as O
from simul_b200 import scene
from tests import contact_case as K
from tests.golden import gen_reference_fixtures as R

REF = np.load(R.HERE / "ref_contact.npz")


@pytest.mark.parametrize("name", sorted(R.contact_cases()))
def test_contact_restatement_matches_reference(name):
    pa, pb, sa, sb, gap, pen = R.contact_cases()[name]
    pairs, gaps = CO.detect(pa, pb, sa, sb, gap)
    np.testing.assert_array_equal(pairs, REF[f"{name}__pairs"])
    np.testing.assert_allclose(gaps, REF[f"{name}__gaps"], rtol=1e-15, atol=0)
    fa, fb = CO.compute_forces(pa, pb, pairs, gaps, pen, gap)
    np.testing.assert_allclose(fa, REF[f"{name}__fa"], rtol=1e-14, atol=1e-14 * np.abs(REF[f"{name}__fa"]).max())
    np.testing.assert_allclose(fb, REF[f"{name}__fb"], rtol=1e-14, atol=1e-14 * np.abs(REF[f"{name}__fb"]).max())
    tp, off = CO.detect_tied_pairs(pa, pb, sa, sb, gap)
    np.testing.assert_array_equal(tp, REF[f"{name}__tied_pairs"])
    np.testing.assert_array_equal(off, REF[f"{name}__tied_offsets"])
    ta, tb = CO.compute_tied_forces(REF[f"{name}__qa"], REF[f"{name}__qb"], tp, off, pen)
    np.testing.assert_array_equal(ta, REF[f"{name}__tied_fa"])
    np.testing.assert_array_equal(tb, REF[f"{name}__tied_fb"])
    assert len(pairs) > 5


def test_boundary_detection_matches_oracle():
    rng = np.random.default_rng(3)
    from simul_b200 import meshgen
    X, _ = meshgen.structured_tets(3, 5, 2, L=(1.5, 2.0, 0.7), origin=(-0.2, 0.3, 1.0))
    X = X[rng.permutation(X.shape[0])]
    np.testing.assert_array_equal(scene.boundary_nodes(X), CO.boundary_nodes(X))
    inner = np.setdiff1d(np.arange(X.shape[0]), CO.boundary_nodes(X))
    assert len(inner) == (3 - 1) * (5 - 1) * (2 - 1)


def _oracle_body(X, conn, fixed, vals):
    mesh = O.Mesh(X, conn)
    mat = O.Material("linear_elastic", E=K.E, nu=K.NU)
    state = {"u": np.zeros_like(X)}

    def solve(f):
        u, _ = O.consistent_newton(mesh, mat, f, fixed, vals, u0=state["u"], tol=1e-8, line_search=False)
        state["u"] = u
        return u
    return CO.Body(X, solve, has_fixed=bool(fixed.any()))


def oracle_staggered(tied=False):
    c = K.blocks()
    bodies = [_oracle_body(*c["a"]), _oracle_body(*c["b"])]
    con = CO.Contact(0, 1, c["surf_a"], c["surf_b"], K.PENALTY, K.GAP, tied=tied)
    res, hist = CO.solve_static(bodies, [con], max_contact_iters=50, contact_tol=1e-3)
    return res, hist, bodies


def test_staggered_contact_loop_converges_on_oracle_bodies():
    res, hist, bodies = oracle_staggered()
    assert res["converged"] and 5 < res["contact_iterations"] < 40, res
    # action = reaction, and A is pushed up by B
    assert np.allclose(bodies[0].f_contact.sum(axis=0), -bodies[1].f_contact.sum(axis=0), atol=1e-12)
    assert bodies[0].f_contact[:, 2].sum() > 0
    # the contact forces equal the penalty law at the final positions of the last injection
    assert res["total_contact_force"] == pytest.approx(hist[-1])
