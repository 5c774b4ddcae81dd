"""Deterministic TET4 and HEX8 input generators for the static-solve workloads.

* ``cantilever_bar``  — structured hex grid, every hex split into 6 Kuhn tets
  along its (0,0,0)->(1,1,1) diagonal; tip traction turned into consistent
  nodal forces (area/3 of every loaded boundary triangle to each vertex).
* ``vertebral_body``  — voxelised elliptic cylinder (semi-axes 15 x 12 mm,
  height 25 mm) on an n^3 grid of spacing 32/n mm, every voxel split into
  5 tets with parity-alternating orientation so neighbouring voxels share
  face diagonals; 2-voxel cortical shell (E = 12 GPa) around a smoothed
  lognormal cancellous core (median 300 MPa).

The reference builds HEX8 grids (``framework/_adapters/fem_adapter.py:41-70``)
and voxel HEX8 meshes (``preprocessing/voxel_to_hex.py:11-68``):
``structured_hex8`` and ``voxels_to_hex_mesh`` restate those two (same node and
element numbering), ``vertebral_body(..., element="hex8")`` builds the
vertebral body from one HEX8 per voxel; the other generators produce the
tetrahedral equivalents.  All arrays are NumPy; units are mm, N, MPa.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

# Kuhn (6-tet) split: every permutation of the axes walks 000 -> 111.
_KUHN_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))

# 5-tet split: corner bits (x, y, z) of the hex.  Even voxels keep the
# "central" tet on the even corners, odd voxels on the odd ones.
_FIVE_EVEN = ((0b000, 0b110, 0b101, 0b011),
              (0b100, 0b000, 0b110, 0b101),
              (0b010, 0b000, 0b011, 0b110),
              (0b001, 0b000, 0b101, 0b011),
              (0b111, 0b110, 0b011, 0b101))
_FIVE_ODD = ((0b100, 0b010, 0b001, 0b111),
             (0b000, 0b100, 0b001, 0b010),
             (0b110, 0b100, 0b010, 0b111),
             (0b101, 0b100, 0b111, 0b001),
             (0b011, 0b010, 0b001, 0b111))


# HEX8 vertex offsets in the reference's order (preprocessing/voxel_to_hex.py:38-50,
# core/element.py:297-315): bottom face counter-clockwise, then the top face.
HEX8_CORNERS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                         [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)


def structured_hex8(nx, ny, nz, L=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    """Structured HEX8 grid numbered as the reference's FEMAdapter builds it
    (framework/_adapters/fem_adapter.py:41-70): node i + j (nx+1) + k (nx+1)(ny+1)
    at origin + (i dx, j dy, k dz); elements x fastest, then y, then z."""
    dx, dy, dz = L[0] / nx, L[1] / ny, L[2] / nz
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    X = np.stack([origin[0] + i.ravel() * dx, origin[1] + j.ravel() * dy, origin[2] + k.ravel() * dz],
                 axis=1).astype(np.float64)
    ez, ey, ex = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (ex + ey * (nx + 1) + ez * (nx + 1) * (ny + 1)).ravel()
    n3 = n0 + (nx + 1)
    n4 = n0 + (nx + 1) * (ny + 1)
    n7 = n4 + (nx + 1)
    conn = np.stack([n0, n0 + 1, n3 + 1, n3, n4, n4 + 1, n7 + 1, n7], axis=1)
    return X, conn.astype(np.int32)


def voxels_to_hex_mesh(voxel_centers: np.ndarray, spacing) -> tuple:
    """Voxel centres -> HEX8 mesh (preprocessing/voxel_to_hex.py:11-68): the
    8 corners of every voxel, merged where their coordinates agree on a grid
    of min(spacing) * 1e-4; nodes in ascending order of that rounded key
    (lexicographic x, y, z), elements (n_voxels, 8) int64."""
    centers = np.asarray(voxel_centers, dtype=np.float64).reshape(-1, 3)
    spacing = np.asarray(spacing, dtype=np.float64).reshape(3)
    if centers.shape[0] == 0:
        return np.empty((0, 3)), np.empty((0, 8), dtype=np.int64)
    verts = (centers[:, None, :] + HEX8_CORNERS[None, :, :] * (0.5 * spacing)[None, None, :]).reshape(-1, 3)
    key = np.round(verts / (np.min(spacing) * 1e-4)).astype(np.int64)
    _, first, inverse = np.unique(key, axis=0, return_index=True, return_inverse=True)
    return verts[first], inverse.reshape(-1, 8).astype(np.int64)


def voxel_hex8(mask: np.ndarray, h: float, origin=(0.0, 0.0, 0.0)):
    """One HEX8 per True voxel of ``mask`` (indexed [i,j,k] = x,y,z), through
    ``voxels_to_hex_mesh``.  Returns nodes, connectivity (int32) and the voxel
    indices in element order."""
    vi, vj, vk = np.nonzero(mask)
    centers = np.stack([origin[0] + (vi + 0.5) * h, origin[1] + (vj + 0.5) * h, origin[2] + (vk + 0.5) * h],
                       axis=1)
    X, conn = voxels_to_hex_mesh(centers, (h, h, h))
    return X, conn.astype(np.int32), (vi, vj, vk)


def labelmap_voxel_centers(label_volume: np.ndarray, spacing, origin=(0.0, 0.0, 0.0), label: int = 1):
    """Physical centres of the voxels carrying ``label`` (preprocessing/assembly.py:82-90):
    ijk * spacing + origin + spacing / 2, voxels in C order of (i, j, k)."""
    spacing = np.asarray(spacing, dtype=np.float64).reshape(3)
    origin = np.asarray(origin, dtype=np.float64).reshape(3)
    ijk = np.argwhere(np.asarray(label_volume) == label)
    return ijk.astype(np.float64) * spacing + origin + spacing / 2.0


def labelmap_bodies(label_volume: np.ndarray, spacing, origin=(0.0, 0.0, 0.0), min_voxels: int = 10) -> dict:
    """One HEX8 body per non-zero label with at least ``min_voxels`` voxels,
    as the labelmap assembly builds its FEM bodies (preprocessing/assembly.py:73-99,
    207-249): label -> (nodes, elements) from ``voxels_to_hex_mesh``.  The
    scene, contacts and particle bodies around them are not built here."""
    out = {}
    labels = np.unique(label_volume)
    for label in labels[labels != 0]:
        centers = labelmap_voxel_centers(label_volume, spacing, origin, int(label))
        if centers.shape[0] < min_voxels:
            continue
        out[int(label)] = voxels_to_hex_mesh(centers, spacing)
    return out


def labelmap_hex8(label_volume: np.ndarray, spacing, origin=(0.0, 0.0, 0.0), labels=None):
    """All voxels of ``labels`` (default: every non-zero label) as one
    conforming HEX8 mesh: neighbouring voxels of different labels share their
    face nodes (bonded bodies).  Returns nodes, connectivity (int32) and the
    label of every element, for a per-label material table."""
    lv = np.asarray(label_volume)
    if labels is None:
        labels = [int(v) for v in np.unique(lv) if v != 0]
    centers, elabel = [], []
    for label in labels:
        c = labelmap_voxel_centers(lv, spacing, origin, label)
        centers.append(c)
        elabel.append(np.full(c.shape[0], label, dtype=np.int32))
    X, conn = voxels_to_hex_mesh(np.concatenate(centers) if centers else np.empty((0, 3)), spacing)
    return X, conn.astype(np.int32), (np.concatenate(elabel) if elabel else np.empty(0, dtype=np.int32))


@dataclass
class TetMesh:
    """A TET4 (or HEX8) mesh with boundary data, in the caller's (generator) order."""
    X: np.ndarray                    # (Nn,3) float64
    conn: np.ndarray                 # (Ne,4) int32, positively oriented (HEX8: (Ne,8))
    E: Optional[np.ndarray] = None   # (Ne,) per-element Young's modulus
    fixed_mask: Optional[np.ndarray] = None   # (Nn,3) bool
    fixed_vals: Optional[np.ndarray] = None   # (Nn,3) float64 (full-load value)
    f_ext: Optional[np.ndarray] = None        # (Nn,3) float64 (full-load value)
    info: dict = field(default_factory=dict)

    @property
    def n_nodes(self):
        return self.X.shape[0]

    @property
    def n_elements(self):
        return self.conn.shape[0]


def _orient(X, conn):
    """Swap nodes 2,3 of negatively oriented tets so det J > 0."""
    e = X[conn]
    d = np.einsum("ei,ei->e", np.cross(e[:, 1] - e[:, 0], e[:, 2] - e[:, 0]), e[:, 3] - e[:, 0])
    neg = d < 0
    conn = conn.copy()
    conn[neg, 2], conn[neg, 3] = conn[neg, 3].copy(), conn[neg, 2].copy()
    return conn


def boundary_triangles(conn: np.ndarray) -> np.ndarray:
    """Faces (k,3) used by exactly one tet."""
    faces = np.concatenate([conn[:, [0, 1, 2]], conn[:, [0, 1, 3]],
                            conn[:, [0, 2, 3]], conn[:, [1, 2, 3]]])
    key = np.sort(faces, axis=1)
    _, idx, cnt = np.unique(key, axis=0, return_index=True, return_counts=True)
    return faces[idx[cnt == 1]]


def traction_nodal_forces(X, conn, face_select, traction) -> np.ndarray:
    """Consistent nodal forces of a uniform traction on boundary triangles.

    ``face_select(centroids) -> bool mask``; each selected triangle gives
    area/3 * traction to each of its vertices.
    """
    tri = boundary_triangles(conn)
    c = X[tri].mean(axis=1)
    tri = tri[face_select(c)]
    p = X[tri]
    area = 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1)
    f = np.zeros_like(X)
    contrib = (area / 3.0)[:, None] * np.asarray(traction, dtype=np.float64)[None, :]
    for k in range(3):
        np.add.at(f, tri[:, k], contrib)
    return f


def structured_tets(nx, ny, nz, L=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    """Structured (nx,ny,nz) hex grid split into 6 Kuhn tets per hex."""
    xs = origin[0] + np.linspace(0.0, L[0], nx + 1)
    ys = origin[1] + np.linspace(0.0, L[1], ny + 1)
    zs = origin[2] + np.linspace(0.0, L[2], nz + 1)
    Z, Y, Xg = np.meshgrid(zs, ys, xs, indexing="ij")
    X = np.stack([Xg.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def nid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    order = np.lexsort((ii, jj, kk))
    ii, jj, kk = ii[order], jj[order], kk[order]
    tets = []
    for perm in _KUHN_PERMS:
        cur = np.zeros((ii.size, 3), dtype=np.int64)
        verts = [nid(ii, jj, kk)]
        for ax in perm:
            cur[:, ax] += 1
            verts.append(nid(ii + cur[:, 0], jj + cur[:, 1], kk + cur[:, 2]))
        tets.append(np.stack(verts, axis=1))
    conn = np.stack(tets, axis=1).reshape(-1, 4)
    return X, _orient(X, conn).astype(np.int32)


def cantilever_bar(nx=20, ny=4, nz=4, length=10.0, width=1.0, height=1.0,
                   E=17e3, nu=0.3, traction=50.0) -> TetMesh:
    """Neo-Hookean cantilever bar (1,920 tets, 525 nodes at the default grid).

    x = 0 face fully fixed; uniform traction ``traction`` (MPa) in -z on the
    x = length face as consistent nodal forces (total -traction*width*height N).
    """
    X, conn = structured_tets(nx, ny, nz, (length, width, height))
    fixed = np.zeros((X.shape[0], 3), dtype=bool)
    fixed[np.isclose(X[:, 0], 0.0)] = True
    tol = 1e-9 * length
    f = traction_nodal_forces(X, conn, lambda c: np.abs(c[:, 0] - length) < tol,
                              (0.0, 0.0, -traction))
    return TetMesh(X=X, conn=conn, E=np.full(conn.shape[0], float(E)), fixed_mask=fixed,
                   fixed_vals=np.zeros_like(X), f_ext=f,
                   info={"kind": "cantilever_bar", "grid": (nx, ny, nz), "nu": nu})


def voxel_tets(mask: np.ndarray, h: float, origin=(0.0, 0.0, 0.0)):
    """Split every True voxel of ``mask`` (indexed [i,j,k] = x,y,z) into 5 tets.

    Returns node coordinates, connectivity and the voxel index of each tet.
    """
    nx, ny, nz = mask.shape
    vi, vj, vk = np.nonzero(mask)
    nvox = vi.size
    # global corner id on the (n+1)^3 lattice, compacted afterwards
    def lat(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k
    corners = np.empty((nvox, 8), dtype=np.int64)
    for b in range(8):
        corners[:, b] = lat(vi + (b >> 2 & 1), vj + (b >> 1 & 1), vk + (b & 1))
    # bit layout used by the split tables is (x<<2 | y<<1 | z) — matches b above
    parity = (vi + vj + vk) & 1
    conn = np.empty((nvox, 5, 4), dtype=np.int64)
    for t in range(5):
        for a in range(4):
            conn[:, t, a] = np.where(parity == 0,
                                     corners[np.arange(nvox), _FIVE_EVEN[t][a]],
                                     corners[np.arange(nvox), _FIVE_ODD[t][a]])
    conn = conn.reshape(-1, 4)
    used, inv = np.unique(conn, return_inverse=True)
    conn = inv.reshape(-1, 4)
    i = used // ((ny + 1) * (nz + 1))
    j = (used // (nz + 1)) % (ny + 1)
    k = used % (nz + 1)
    X = np.stack([origin[0] + i * h, origin[1] + j * h, origin[2] + k * h], axis=1).astype(np.float64)
    voxel_of_tet = np.repeat(np.arange(nvox), 5)
    return X, _orient(X, conn).astype(np.int32), voxel_of_tet, (vi, vj, vk)


def vertebral_body(n=64, seed=0, a=15.0, b=12.0, height=25.0, extent=32.0,
                   E_cortical=12e3, E_core_median=300.0, core_sigma=0.3,
                   smooth_voxels=3.0, shell_voxels=2, nu=0.3,
                   axial_strain=0.02, element="tet4") -> TetMesh:
    """Synthetic vertebral body of the plain-method workload.

    Voxel (i,j,k) of spacing h = extent/n is inside when its centre satisfies
    (x/a)^2 + (y/b)^2 <= 1 and 0 <= z < height.  Bottom face fixed; the top
    face gets u_z = -axial_strain*height (full load; callers step it).
    ``element="hex8"`` makes every voxel one HEX8 (``voxel_hex8``) instead of
    five tets.
    """
    if element not in ("tet4", "hex8"):
        raise ValueError(f"element must be 'tet4' or 'hex8', got {element!r}")
    from scipy import ndimage

    h = extent / n
    c = (np.arange(n) + 0.5) * h
    xc = c - extent / 2.0
    zc = c
    Xv, Yv, Zv = np.meshgrid(xc, xc, zc, indexing="ij")
    mask = ((Xv / a) ** 2 + (Yv / b) ** 2 <= 1.0) & (Zv >= 0.0) & (Zv < height)
    core = ndimage.binary_erosion(mask, iterations=shell_voxels)
    rng = np.random.default_rng(seed)
    z = ndimage.gaussian_filter(rng.standard_normal(mask.shape), sigma=smooth_voxels)
    zc_ = z[core]
    z = (z - zc_.mean()) / zc_.std()
    Evox = np.where(core, E_core_median * np.exp(core_sigma * z), E_cortical)
    if element == "hex8":
        X, conn, (vi, vj, vk) = voxel_hex8(mask, h, origin=(-extent / 2.0, -extent / 2.0, 0.0))
        E = Evox[vi, vj, vk]
    else:
        X, conn, vox, (vi, vj, vk) = voxel_tets(mask, h, origin=(-extent / 2.0, -extent / 2.0, 0.0))
        E = Evox[vi, vj, vk][vox]
    top_z = X[:, 2].max()
    fixed = np.zeros((X.shape[0], 3), dtype=bool)
    fixed_vals = np.zeros_like(X)
    bottom = np.isclose(X[:, 2], 0.0)
    top = np.isclose(X[:, 2], top_z)
    fixed[bottom] = True
    fixed[top, 2] = True
    fixed_vals[top, 2] = -axial_strain * top_z
    return TetMesh(X=X, conn=conn, E=E.astype(np.float64), fixed_mask=fixed,
                   fixed_vals=fixed_vals, f_ext=np.zeros_like(X),
                   info={"kind": "vertebral_body", "element": element, "n": n, "h": h, "seed": seed, "nu": nu,
                         "n_voxels": int(mask.sum()), "height": float(top_z),
                         "shell_elements": int(np.sum(E == E_cortical))})


def top_moment_forces(X: np.ndarray, top: np.ndarray, case: str, moment: float) -> np.ndarray:
    """Nodal forces on the ``top`` nodes equivalent to a moment (N mm) about
    the top face's centroid: a linear force couple (flexion / extension about
    x, lateral bending about y) or a tangential couple (torsion about z).
    No rigid plate is modelled."""
    f = np.zeros_like(X)
    xc = X[top, 0] - X[top, 0].mean()
    yc = X[top, 1] - X[top, 1].mean()
    ft = np.zeros((int(np.count_nonzero(top)), 3))
    if case in ("flexion", "extension"):
        sgn = 1.0 if case == "flexion" else -1.0
        ft[:, 2] = -sgn * moment * yc / np.sum(yc * yc)
    elif case == "lateral_bending":
        ft[:, 2] = -moment * xc / np.sum(xc * xc)
    elif case == "torsion":
        r2 = np.sum(xc * xc + yc * yc)
        ft[:, 0] = -moment * yc / r2
        ft[:, 1] = moment * xc / r2
    else:
        raise ValueError(f"unknown moment case {case!r}")
    f[top] = ft
    return f


def motion_segment(n=80, seed=0, a=15.0, b=12.0, body_height=25.0, disc_height=10.0, extent=32.0,
                   E_cortical=12e3, E_core_median=300.0, core_sigma=0.3, smooth_voxels=3.0,
                   shell_voxels=2, screw_radius=3.0, screw_length=45.0) -> TetMesh:
    """Synthetic motion segment: two vertebral bodies (as ``vertebral_body``,
    n voxels across ``extent``) joined by an intervertebral disc, with a
    titanium pedicle-screw cylinder in the lower body.

    Voxel spacing h = extent / n; the stack is body (z in [0, H)), disc
    ([H, H + D)), body ([H + D, 2H + D)), all with the elliptic cross-section.
    The screw (radius 3 mm, length 45 mm) runs along y through the lower
    body's mid-height, its tip at the anterior surface; the part behind the
    body (up to the grid's edge) stays screw material.  Material ids per element: 0 bone (per-element
    modulus in ``E``), 1 disc, 2 screw.  Bottom face fixed; loads are left to
    the caller (``top_moment_forces``).
    """
    from scipy import ndimage

    h = extent / n
    H, D = body_height, disc_height
    nz = int(round((2 * H + D) / h))
    c = (np.arange(n) + 0.5) * h - extent / 2.0
    zc = (np.arange(nz) + 0.5) * h
    Xv, Yv, Zv = np.meshgrid(c, c, zc, indexing="ij")
    ell = (Xv / a) ** 2 + (Yv / b) ** 2 <= 1.0
    lower = ell & (Zv < H)
    disc = ell & (Zv >= H) & (Zv < H + D)
    upper = ell & (Zv >= H + D) & (Zv < 2 * H + D)
    # the screw's tip reaches the anterior surface (y = +b); the rest runs
    # posteriorly, clipped to the voxel grid
    y_tip = b
    screw = ((Xv ** 2 + (Zv - H / 2.0) ** 2) <= screw_radius ** 2) & (Yv < y_tip) & (Yv >= y_tip - screw_length)
    bone = (lower | upper) & ~screw
    mask = bone | disc | screw
    rng = np.random.default_rng(seed)
    core = ndimage.binary_erosion(lower, iterations=shell_voxels) | ndimage.binary_erosion(upper, iterations=shell_voxels)
    z = ndimage.gaussian_filter(rng.standard_normal(mask.shape), sigma=smooth_voxels)
    zsel = z[core & bone]
    z = (z - zsel.mean()) / zsel.std()
    Evox = np.where(core, E_core_median * np.exp(core_sigma * z), E_cortical)
    mid = np.zeros(mask.shape, dtype=np.int32)
    mid[disc] = 1
    mid[screw] = 2
    X, conn, vox, (vi, vj, vk) = voxel_tets(mask, h, origin=(-extent / 2.0, -extent / 2.0, 0.0))
    E = Evox[vi, vj, vk][vox]
    ids = mid[vi, vj, vk][vox]
    E = np.where(ids == 0, E, 1.0)
    fixed = np.zeros((X.shape[0], 3), dtype=bool)
    fixed[np.isclose(X[:, 2], 0.0)] = True
    return TetMesh(X=X, conn=conn, E=E.astype(np.float64), fixed_mask=fixed, fixed_vals=np.zeros_like(X),
                   f_ext=np.zeros_like(X),
                   info={"kind": "motion_segment", "n": n, "h": h, "seed": seed, "material_ids": ids,
                         "n_voxels": int(mask.sum()), "height": float(X[:, 2].max()),
                         "disc_elements": int(np.sum(ids == 1)), "screw_elements": int(np.sum(ids == 2))})
