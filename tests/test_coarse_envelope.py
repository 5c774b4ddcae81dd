"""The coarse operator's envelope and the tile skipping of its inverse,
checked on the CPU with the FP64 oracle's elastic tangent (n = 16).

The coarse space (fem_coarse.cu) assembles each element into the lattice
cell of its centroid, with its nodes' trilinear weights clamped to that
cell, so two coarse nodes couple only through a shared cell.  Coarse nodes
are numbered in lattice order (fem_ctx.cu, build_coarse), which makes
Ac = sum_e P_e^T K_e P_e banded: row 3 a + d is zero left of column
3 min{b : b shares a cell with a}.  The dense inverse (fem_dense.cu) takes
that envelope and, at Cholesky step k, launches only the tile rows
k + 1 .. last(k), last from the suffix minimum of the tile rows' first
columns.  This file restates the element-to-cell Galerkin assembly, the
envelope and the blocked right-looking schedule in numpy and checks that:
entries outside the envelope are exactly zero, the Cholesky factor's fill
stays inside it, and the skipping schedule gives exactly the dense
schedule's inverse.
"""
import numpy as np

from oracle import fem_oracle as O
from simul_b200 import meshgen


def _galerkin(n=16, cell=4):
    """Ac of the elastic tangent on the lattice of `cell`-voxel cells, the
    per-element construction of the coarse space, and the lattice envelope."""
    v = meshgen.vertebral_body(n=n, seed=0)
    X, conn = v.X, v.conn.astype(np.int64)
    m = O.Mesh(X, conn)
    nu = 0.3
    lam1, mu1 = nu / ((1 + nu) * (1 - 2 * nu)), 1 / (2 * (1 + nu))
    I3 = np.eye(3)
    A1 = lam1 * np.einsum("ij,kl->ijkl", I3, I3) + mu1 * (np.einsum("ik,jl->ijkl", I3, I3)
                                                          + np.einsum("il,jk->ijkl", I3, I3))
    A = np.broadcast_to(A1, (conn.shape[0], 3, 3, 3, 3)) * v.E[:, None, None, None, None]
    Ke = O.element_stiffness(A, m.dNdX, m.vol)
    free = ~v.fixed_mask.reshape(-1).astype(bool)
    # lattice of the element centroids (cell edge `cell` voxels)
    hmesh = 32.0 / n
    H = cell * hmesh
    lo, hi = X.min(0), X.max(0)
    g = np.maximum(1, np.ceil((hi - lo) / H - 1e-9).astype(int))
    org = lo - np.floor(0.5 * (g * H - (hi - lo)) / hmesh + 1e-6) * hmesh
    ijk = np.clip(np.floor((X[conn].mean(1) - org) / H).astype(int), 0, g - 1)
    G = g + 1
    off = np.array([[q >> 2 & 1, q >> 1 & 1, q & 1] for q in range(8)])
    lat = (((ijk[:, None, 0] + off[None, :, 0]) * G[1] + ijk[:, None, 1] + off[None, :, 1]) * G[2]
           + ijk[:, None, 2] + off[None, :, 2])                          # (Ne, 8) lattice corners
    used = np.unique(lat)                                                # lattice order
    corner = np.searchsorted(used, lat)                                  # (Ne, 8) coarse nodes
    ncn = used.size
    # element nodes' weights on their element's cell corners (clamped)
    loc = np.clip((X[conn] - org) / H - ijk[:, None, :], 0.0, 1.0)     # (Ne, npe, 3)
    w = np.prod(np.where(off[None, None] == 1, loc[:, :, None, :], 1 - loc[:, :, None, :]), axis=-1)
    npe = conn.shape[1]
    Pe = np.zeros((conn.shape[0], 3 * npe, 24))
    for d in range(3):
        Pe[:, d::3, d::3] = w
    fd = free[(conn[:, :, None] * 3 + np.arange(3)).reshape(len(conn), -1)]
    Kf = Ke * fd[:, :, None] * fd[:, None, :]                           # free DOFs only
    Ace = np.einsum("eia,eij,ejb->eab", Pe, Kf, Pe)                      # (Ne, 24, 24)
    cd = (corner[:, :, None] * 3 + np.arange(3)).reshape(len(conn), 24)
    Ac = np.zeros((3 * ncn, 3 * ncn))
    np.add.at(Ac, (cd[:, :, None], cd[:, None, :]), Ace)
    dg = np.arange(3 * ncn)
    Ac[dg, dg] = np.where(Ac[dg, dg] > 0, Ac[dg, dg], 1.0)              # unreached DOFs: unit diagonal
    # envelope: lowest coarse node sharing a cell, per node
    first_node = np.arange(ncn)
    np.minimum.at(first_node, corner, np.repeat(corner.min(1)[:, None], 8, axis=1))
    row_first = 3 * first_node[np.arange(3 * ncn) // 3]
    return Ac, row_first


def _last_tiles(row_first, n, B):
    """The schedule's last(k): tile row i may be nonzero in tile column k iff
    the suffix minimum of the tile rows' first tile columns is <= k."""
    nt = (n + B - 1) // B
    fm = [min([i] + [int(row_first[r]) // B for r in range(i * B, min(n, (i + 1) * B))]) for i in range(nt)]
    for i in range(nt - 2, -1, -1):
        fm[i] = min(fm[i], fm[i + 1])
    last, i = [], 0
    for k in range(nt):
        while i + 1 < nt and fm[i + 1] <= k:
            i += 1
        last.append(max(i, k))
    return last


def _blocked_inverse(A, B, last):
    """Right-looking blocked Cholesky, W = L^-1 and W^T W, with the
    schedule's tile ranges: panel and updates over tile rows k+1..last[k]."""
    n = A.shape[0]
    nt = (n + B - 1) // B
    N = nt * B
    M = np.eye(N)
    M[:n, :n] = np.tril(A)
    W = np.zeros((N, N))

    def T(a, b):
        return slice(a * B, (a + 1) * B), slice(b * B, (b + 1) * B)

    for k in range(nt):
        Akk = np.tril(M[T(k, k)])
        Lkk = np.linalg.cholesky(Akk + np.tril(Akk, -1).T)
        M[T(k, k)] = Lkk
        Wkk = np.linalg.inv(Lkk)
        W[T(k, k)] = Wkk
        for i in range(k + 1, last[k] + 1):
            M[T(i, k)] = M[T(i, k)] @ Wkk.T
        for j in range(k):
            W[T(k, j)] = Wkk @ W[T(k, j)]
        for i in range(k + 1, last[k] + 1):
            for j in range(k + 1):
                W[T(i, j)] -= M[T(i, k)] @ W[T(k, j)]
        for j in range(k + 1, last[k] + 1):
            for i in range(j, last[k] + 1):
                M[T(i, j)] -= M[T(i, k)] @ M[T(j, k)].T
    return (W.T @ W)[:n, :n]


def test_coarse_operator_is_zero_outside_the_lattice_envelope_and_so_is_its_factor():
    Ac, row_first = _galerkin()
    n = Ac.shape[0]
    cols = np.arange(n)
    outside = cols[None, :] < row_first[:, None]                         # left of each row's envelope
    assert outside.sum() > n * n // 4                                   # the band is narrow
    assert np.all(Ac[outside] == 0.0)
    assert np.allclose(Ac, Ac.T, rtol=0, atol=1e-12 * np.abs(Ac).max())
    L = np.linalg.cholesky(Ac)                                           # reads the lower triangle
    assert np.all(L[outside] == 0.0)                                     # no fill outside


def test_envelope_schedule_reproduces_the_dense_inverse_exactly():
    Ac, row_first = _galerkin()
    n = Ac.shape[0]
    B = 16                                                              # 15 tiles at n = 16
    nt = (n + B - 1) // B
    last = _last_tiles(row_first, n, B)
    assert all(k <= last[k] <= nt - 1 for k in range(nt))
    assert sum(last[k] < nt - 1 for k in range(nt)) >= nt // 2         # the schedule does skip
    Xb = _blocked_inverse(Ac, B, last)
    Xd = _blocked_inverse(Ac, B, [nt - 1] * nt)
    assert np.array_equal(Xb, Xd)
    ref = np.linalg.inv(Ac)
    assert np.abs(Xb - ref).max() <= 1e-8 * np.abs(ref).max()
