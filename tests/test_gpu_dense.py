"""The dense SPD inverse kernels of the coarse operator (fem_dense.cu)
against numpy's inverse, on seeded SPD matrices of ragged and whole-tile
sizes (tiles are 64 in FP64, 128 in FP32), plus a matrix that is not
positive definite."""
import ctypes as C

import numpy as np
import pytest
import torch

from simul_b200 import _lib

pytestmark = pytest.mark.gpu


def _spd(n, seed, cond=1e3):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.geomspace(1.0, cond, n)
    return (Q * ev) @ Q.T


def _run(A, precision, cuda):
    n = A.shape[0]
    dA = torch.as_tensor(np.asfortranarray(A).ravel(order="F"), dtype=torch.float64, device=cuda)
    out = torch.full((n * n,), float("nan"), dtype=torch.float64, device=cuda)
    rc = _lib.load().fem_dense_spd_inverse(C.c_void_p(dA.data_ptr()), n, precision, C.c_void_p(out.data_ptr()), None)
    return rc, out.cpu().numpy().reshape(n, n, order="F")


@pytest.mark.parametrize("n", [1, 37, 64, 127, 128, 200, 513])
@pytest.mark.parametrize("precision,tol", [(64, 1e-11), (32, 2e-4), (19, 5e-2)])
def test_dense_spd_inverse_matches_numpy(cuda, n, precision, tol):
    A = _spd(n, seed=n)
    rc, X = _run(A, precision, cuda)
    assert rc == 0, _lib.last_error()
    ref = np.linalg.inv(A)
    lo = np.tril(np.ones((n, n), dtype=bool))
    err = np.abs(X[lo] - ref[lo]).max() / np.abs(ref).max()
    assert err < tol, err
    # above the diagonal only the diagonal tiles are written (with the
    # symmetric values); everything else is left as it was
    up = ~lo & ~np.isnan(X)
    if up.any():
        assert np.abs(X[up] - ref[up]).max() / np.abs(ref).max() < tol


@pytest.mark.parametrize("n", [128, 300, 1000])
def test_tf32_tensor_core_inverse_on_well_conditioned_matrices(cuda, n):
    """Precision 19 forms W = L^-1 and W^T W on TF32 tcgen05 tiles: on a
    matrix of condition 10 the result is within TF32 rounding of the FP64
    inverse (a wrong operand layout would give O(1) errors), and as a
    preconditioner its eigenvalues stay within 1 +- 1e-2."""
    A = _spd(n, seed=100 + n, cond=10.0)
    rc, X = _run(A, 19, cuda)
    assert rc == 0, _lib.last_error()
    ref = np.linalg.inv(A)
    lo = np.tril(np.ones((n, n), dtype=bool))
    assert np.abs(X[lo] - ref[lo]).max() / np.abs(ref).max() < 5e-3
    Xs = np.tril(X) + np.tril(X, -1).T
    ev = np.linalg.eigvals(Xs @ A).real
    assert ev.min() > 0.99 and ev.max() < 1.01, (ev.min(), ev.max())


def test_dense_spd_inverse_rejects_indefinite(cuda):
    A = _spd(150, seed=5)
    A[70, 70] = -5.0
    rc, _ = _run(A, 64, cuda)
    assert rc == _lib.FEM_ERR_NAN
    assert "not positive definite" in _lib.last_error()
    rc, _ = _run(A, 32, cuda)
    assert rc == _lib.FEM_ERR_NAN


def test_dense_spd_inverse_validates_arguments(cuda):
    assert _lib.load().fem_dense_spd_inverse(None, 4, 64, None, None) == _lib.FEM_ERR_INVALID
    A = torch.eye(4, dtype=torch.float64, device=cuda)
    out = torch.empty_like(A)
    assert _lib.load().fem_dense_spd_inverse(C.c_void_p(A.data_ptr()), 4, 16, C.c_void_p(out.data_ptr()),
                                             None) == _lib.FEM_ERR_INVALID
    assert "precision" in _lib.last_error()


def _enveloped_spd(n, width, seed):
    """Symmetric, diagonally dominant (so SPD) matrix whose lower-triangle
    row r is nonzero only from column first[r] (a ragged, non-monotone
    envelope, as the coarse operator of a lattice has)."""
    rng = np.random.default_rng(seed)
    first = np.maximum(0, np.arange(n) - rng.integers(0, width + 1, n))
    A = np.zeros((n, n))
    for r in range(n):
        A[r, first[r]:r] = rng.standard_normal(r - first[r])
    A = A + A.T
    A[np.arange(n), np.arange(n)] = np.abs(A).sum(1) + 1.0
    return A, first.astype(np.int32)


def _run_banded(A, first, precision, cuda):
    n = A.shape[0]
    dA = torch.as_tensor(np.asfortranarray(A).ravel(order="F"), dtype=torch.float64, device=cuda)
    out = torch.full((n * n,), float("nan"), dtype=torch.float64, device=cuda)
    rf = np.ascontiguousarray(first, dtype=np.int32)
    rc = _lib.load().fem_dense_spd_inverse_banded(C.c_void_p(dA.data_ptr()), n, precision,
                                                  rf.ctypes.data_as(C.POINTER(C.c_int32)),
                                                  C.c_void_p(out.data_ptr()), None)
    return rc, out.cpu().numpy().reshape(n, n, order="F")


@pytest.mark.parametrize("n,width", [(700, 150), (1000, 300), (513, 40)])
@pytest.mark.parametrize("precision", [64, 32, 19])
def test_banded_inverse_skips_only_zero_tiles(cuda, n, width, precision):
    """The envelope form skips the tiles of L (and of W's update) outside
    the rows' envelope: the products it leaves out would add exact zeros,
    so its result equals the dense entry point's, entry for entry."""
    A, first = _enveloped_spd(n, width, seed=n + width)
    rc, Xb = _run_banded(A, first, precision, cuda)
    assert rc == 0, _lib.last_error()
    rc, Xd = _run(A, precision, cuda)
    assert rc == 0, _lib.last_error()
    lo = np.tril(np.ones((n, n), dtype=bool))
    assert np.array_equal(Xb[lo], Xd[lo])
    ref = np.linalg.inv(A)
    tol = {64: 1e-11, 32: 2e-4, 19: 5e-2}[precision]
    assert np.abs(Xb[lo] - ref[lo]).max() / np.abs(ref).max() < tol


def test_banded_inverse_validates_envelope(cuda):
    A = torch.eye(4, dtype=torch.float64, device=cuda)
    out = torch.empty_like(A)
    lib = _lib.load()
    bad = np.array([0, 0, 3, 1], dtype=np.int32)  # row 2 cannot start right of its diagonal
    assert lib.fem_dense_spd_inverse_banded(C.c_void_p(A.data_ptr()), 4, 64, bad.ctypes.data_as(C.POINTER(C.c_int32)),
                                            C.c_void_p(out.data_ptr()), None) == _lib.FEM_ERR_INVALID
    assert "row_first" in _lib.last_error()
    assert lib.fem_dense_spd_inverse_banded(C.c_void_p(A.data_ptr()), 4, 64, None, C.c_void_p(out.data_ptr()),
                                            None) == _lib.FEM_ERR_INVALID
