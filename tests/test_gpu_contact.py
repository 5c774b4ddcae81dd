"""GPU contact: the node-to-node kernels against the reference's own
contact.py outputs (tests/golden/ref_contact.npz), and the staggered static
Scene solve against the same loop over FP64 oracle bodies."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import contact_oracle as CO
from simul_b200 import _lib
from simul_b200 import fem as B
from simul_b200 import scene as S
from tests import contact_case as K
from tests.golden import gen_reference_fixtures as R
from tests.test_contact_oracle import oracle_staggered

pytestmark = pytest.mark.gpu
REF = np.load(R.HERE / "ref_contact.npz")


def _d(a, cuda, dt=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=cuda)


def _p(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("name", sorted(R.contact_cases()))
def test_penalty_kernel_matches_reference(cuda, name):
    pa, pb, sa, sb, gap, pen = R.contact_cases()[name]
    dpa, dpb = _d(pa, cuda), _d(pb, cuda)
    dsa, dsb = _d(sa, cuda, torch.int32), _d(sb, cuda, torch.int32)
    fa = torch.zeros_like(dpa)
    fb = torch.zeros_like(dpb)
    npairs, tot = C.c_int32(), C.c_double()
    rc = _lib.load().fem_contact_penalty(_p(dpa), _p(dsa), len(sa), _p(dpb), _p(dsb), len(sb), gap, pen, _p(fa), _p(fb),
                                         C.byref(npairs), C.byref(tot), None)
    assert rc == 0, _lib.last_error()
    ref_fa, ref_fb = REF[f"{name}__fa"], REF[f"{name}__fb"]
    scale = np.abs(ref_fa).max()
    assert np.abs(fa.cpu().numpy() - ref_fa).max() <= 1e-12 * scale
    assert np.abs(fb.cpu().numpy() - ref_fb).max() <= 1e-12 * scale
    assert npairs.value == len(REF[f"{name}__pairs"])
    assert tot.value == pytest.approx(np.abs(ref_fa).sum(), rel=1e-13)
    # nearest-neighbour query alone: the reference's pair partners
    near = torch.empty(len(sa), dtype=torch.int32, device=cuda)
    dist = torch.empty(len(sa), dtype=torch.float64, device=cuda)
    assert _lib.load().fem_contact_nearest(_p(dpa), _p(dsa), len(sa), _p(dpb), _p(dsb), len(sb), _p(near),
                                           _p(dist), None) == 0
    torch.cuda.synchronize()
    m = dist.cpu().numpy() < gap
    got = np.column_stack([sa[m], sb[near.cpu().numpy()[m]]])
    np.testing.assert_array_equal(got, REF[f"{name}__pairs"])
    np.testing.assert_allclose(dist.cpu().numpy()[m], REF[f"{name}__gaps"], rtol=1e-14)


@pytest.mark.parametrize("name", sorted(R.contact_cases()))
def test_tied_kernel_matches_reference(cuda, name):
    pen = R.contact_cases()[name][5]
    qa, qb = _d(REF[f"{name}__qa"], cuda), _d(REF[f"{name}__qb"], cuda)
    pairs = _d(REF[f"{name}__tied_pairs"], cuda, torch.int32)
    off = _d(REF[f"{name}__tied_offsets"], cuda)
    fa, fb = torch.zeros_like(qa), torch.zeros_like(qb)
    tot = C.c_double()
    rc = _lib.load().fem_contact_tied(_p(qa), _p(qb), _p(pairs), _p(off), pairs.shape[0], qb.shape[0], pen, _p(fa),
                                      _p(fb), C.byref(tot), None)
    assert rc == 0, _lib.last_error()
    np.testing.assert_array_equal(fa.cpu().numpy(), REF[f"{name}__tied_fa"])
    np.testing.assert_array_equal(fb.cpu().numpy(), REF[f"{name}__tied_fb"])


def _gpu_scene(cuda, tied=False):
    c = K.blocks()
    bodies = []
    for key in ("a", "b"):
        X, conn, fixed, vals = c[key]
        mesh = B.FEMesh(X.shape[0], conn.shape[0], device=cuda)
        mesh.initialize_from_numpy(X, conn)
        idx = np.where(fixed.reshape(-1))[0]
        mesh.set_fixed_dofs(idx, vals.reshape(-1)[idx])
        bodies.append(S.FEMBody(mesh, B.LinearElastic(K.E, K.NU), tol=1e-8))
    sc = S.Scene()
    for b in bodies:
        sc.add(b)
    sc.add_contact(bodies[0], bodies[1], method=S.ContactType.TIED if tied else S.ContactType.PENALTY,
                   penalty=K.PENALTY, gap_tolerance=K.GAP, surface_a=c["surf_a"], surface_b=c["surf_b"])
    return sc, bodies


@pytest.mark.parametrize("tied", [False, True])
def test_staggered_scene_matches_oracle(cuda, tied):
    ref, ref_hist, ref_bodies = oracle_staggered(tied=tied)
    sc, bodies = _gpu_scene(cuda, tied=tied)
    res = sc.solve(mode="static", max_contact_iters=50, contact_tol=1e-3)
    assert res["converged"] == ref["converged"]
    assert res["contact_iterations"] == ref["contact_iterations"], (res["contact_force_history"], ref_hist)
    assert res["total_contact_force"] == pytest.approx(ref["total_contact_force"], rel=1e-6)
    np.testing.assert_allclose(res["contact_force_history"], ref_hist, rtol=1e-6)
    for gb, ob in zip(bodies, ref_bodies):
        u = gb.mesh.get_displacements()
        assert np.linalg.norm(u - ob.u) <= 1e-6 * np.linalg.norm(ob.u)
        assert np.abs(gb.contact_forces - ob.f_contact).max() <= 1e-6 * np.abs(ob.f_contact).max()
    # every body solve after the first contact iteration started from the last state
    assert all(r["converged"] for r in res["body_results"])


def test_scene_automatic_parameters_and_modes(cuda):
    c = K.blocks()
    bodies = []
    for key in ("a", "b"):
        X, conn, fixed, vals = c[key]
        mesh = B.FEMesh(X.shape[0], conn.shape[0], device=cuda)
        mesh.initialize_from_numpy(X, conn)
        bodies.append(S.FEMBody(mesh, B.LinearElastic(K.E, K.NU), spacing=0.25))
    sc = S.Scene()
    for b in bodies:
        sc.add(b)
    sc.add_contact(bodies[0], bodies[1])
    sc._build()
    cd = sc._contacts[0]
    # scene.py:154-172: the whole boundary, 1.5 x spacing, E_avg / spacing
    np.testing.assert_array_equal(cd.surface_a, CO.boundary_nodes(c["a"][0]))
    assert cd.gap_tolerance == pytest.approx(0.375) and cd.penalty == pytest.approx(K.E / 0.25)
    with pytest.raises(B.FEAValidationError):
        sc.solve(mode="explicit")
