"""How much a learned *linear* change to the two-level preconditioner can gain.

A preconditioner inside CG must stay one fixed SPD operator; the network
used as a nonlinear map z = N(r) inside flexible PCG breaks conjugacy (the
GPU tests of the learned path measure that).  The linear places a network
could act in the two-level method z = S r + P Ac^-1 P^T r are the smoother
S (e.g. a per-node scaling of the 3 x 3 block inverse) and the coarse
interpolation weights P.  This study bounds both on the synthetic vertebral
body (n = 16, J2 elastic tangent, 4-voxel lattice cells) with FP64 numpy
PCG on the assembled tangent:

- the best global scaling of the block smoother saves <= 5 % of the CG
  iterations (a per-node learned scaling can only pick a better one per
  node; the material-wise split tried in development did no better);
- energy-minimising corner weights on the same 8-corner pattern (projected
  Jacobi sweeps with rows kept summing to 1, the target a learned
  interpolation would have to approach) save 10-20 %.

So the learned linear forms are bounded well below the 6x the coarse
space already gives over Jacobi-PCG.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import fem_oracle as O
from simul_b200 import meshgen


def _setup(n=16, cell=4):
    v = meshgen.vertebral_body(n=n, seed=0)
    X, conn = v.X, v.conn.astype(np.int64)
    m = O.Mesh(X, conn)
    nu = 0.3
    lam1, mu1 = nu / ((1 + nu) * (1 - 2 * nu)), 1 / (2 * (1 + nu))
    I = np.eye(3)
    A1 = lam1 * np.einsum("ij,kl->ijkl", I, I) + mu1 * (np.einsum("ik,jl->ijkl", I, I) + np.einsum("il,jk->ijkl", I, I))
    A = np.broadcast_to(A1, (conn.shape[0], 3, 3, 3, 3)) * v.E[:, None, None, None, None]
    K = O.assemble(O.element_stiffness(A, m.dNdX, m.vol), conn, X.shape[0]).tocsr()
    nn = X.shape[0]
    fm = v.fixed_mask.reshape(nn, 3).astype(bool)
    free = ~fm.reshape(-1)
    Kf = K[free][:, free].tocsr()
    # nodal 3 x 3 block smoother on the free DOFs
    B = np.stack([np.stack([np.asarray(K[np.arange(nn) * 3 + d, np.arange(nn) * 3 + e]).ravel()
                            for e in range(3)], -1) for d in range(3)], 1)
    B[fm] = 0.0
    B = B * (~fm)[:, None, :]
    B[np.arange(nn)[:, None], np.arange(3)[None, :], np.arange(3)[None, :]] += fm
    Binv = np.linalg.inv(B) * (~fm)[:, :, None] * (~fm)[:, None, :]
    Bf = sp.block_diag([sp.csr_matrix(b) for b in Binv], format="csr")[free][:, free]
    # trilinear lattice of `cell` voxels
    H = cell * 32.0 / n
    lo = X.min(0) - 1e-9
    idx = np.floor((X - lo) / H).astype(int)
    loc = (X - lo) / H - idx
    dims = idx.max(0) + 2
    rows, cols, vals = [], [], []
    for c in range(8):
        o = np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1])
        rows.append(np.arange(nn))
        cols.append(np.ravel_multi_index((idx + o).T, dims))
        vals.append(np.prod(np.where(o[None, :] == 1, loc, 1 - loc), axis=1))
    Pn = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                       shape=(nn, int(np.prod(dims)))).tocsc()
    Pn = Pn[:, np.unique(Pn.nonzero()[1])].tocsr()
    Ks = ((K[0::3, 0::3] + K[1::3, 1::3] + K[2::3, 2::3]) / 3.0).tocsr()
    us = np.sin(X[:, :1] / 7.0) * np.cos(X[:, 1:2] / 5.0) * np.array([[1.0, 0.5, -0.7]])
    rng = np.random.default_rng(1)
    rhs = [rng.standard_normal(int(free.sum())), Kf @ us.reshape(-1)[free]]
    return Kf, Bf, Pn, Ks, free, rhs


def _pcg_iters(Kf, M, b, tol=1e-8, maxit=2000):
    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    p = z.copy()
    rz = r @ z
    r0 = np.linalg.norm(b)
    for it in range(1, maxit + 1):
        q = Kf @ p
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        if np.linalg.norm(r) <= tol * r0:
            return it
        z = M(r)
        rzn = r @ z
        p = z + (rzn / rz) * p
        rz = rzn
    return maxit


def _coarse(Kf, Pn, free):
    P = sp.kron(Pn, sp.eye(3)).tocsr()[free]
    Ac = (P.T @ Kf @ P).toarray()
    ev, V = np.linalg.eigh(0.5 * (Ac + Ac.T))
    good = ev > 1e-10 * ev.max()
    Ainv = (V[:, good] / ev[good]) @ V[:, good].T
    return lambda r: P @ (Ainv @ (P.T @ r))


@pytest.mark.timeout(600)
def test_linear_learned_forms_have_small_headroom():
    Kf, Bf, Pn, Ks, free, rhs = _setup()
    cf = _coarse(Kf, Pn, free)
    base = sum(_pcg_iters(Kf, lambda r: Bf @ r + cf(r), b) for b in rhs)
    scaled = min(sum(_pcg_iters(Kf, lambda r, w=w: w * (Bf @ r) + cf(r), b) for b in rhs)
                 for w in (0.6, 1.3, 1.7))
    # energy-minimising weights on the 8-corner pattern, rows summing to 1
    pat = (Pn != 0).astype(np.float64).tocsr()
    cnt = np.asarray(pat.sum(1)).ravel()
    Pc = Pn.copy()
    for _ in range(6):
        G = (sp.diags(1.0 / Ks.diagonal()) @ (Ks @ Pc)).multiply(pat).tocsr()
        G = G - sp.diags(np.asarray(G.sum(1)).ravel() / cnt) @ pat
        Pc = (Pc - 0.6 * G).multiply(pat).tocsr()
    cf_em = _coarse(Kf, Pc, free)
    emin = sum(_pcg_iters(Kf, lambda r: Bf @ r + cf_em(r), b) for b in rhs)
    gain_scale = 1.0 - scaled / base
    gain_emin = 1.0 - emin / base
    print(f"two-level CG iterations {base}; best smoother scaling {scaled} ({gain_scale:.1%}); "
          f"energy-minimising interpolation {emin} ({gain_emin:.1%})")
    assert -0.02 <= gain_scale <= 0.05
    assert 0.05 <= gain_emin <= 0.25
