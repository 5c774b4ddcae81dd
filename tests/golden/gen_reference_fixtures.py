"""Golden vectors made by running the reference's own code.

Two reference modules on this path import only numpy and scipy, so they run
in this container even though the Taichi kernels around them do not:

- ``backend/fea/fem/solver/assembly.py`` — ``assemble_stiffness_matrix``
  (initial-C material stiffness, single- and multi-material, chunked) and
  ``assemble_geometric_stiffness`` (``assembly.py:20-287``), the tangent the
  reference's Newton solves with;
- ``backend/preprocessing/voxel_to_hex.py`` — ``voxels_to_hex_mesh``
  (``voxel_to_hex.py:11-68``), the labelmap-to-HEX8 mesher;
- ``backend/fea/framework/contact.py`` — ``NodeNodeContact`` (``:43-273``):
  nearest-pair detection, penalty forces, tied pairs and tied forces.

Each module is loaded by file path (``importlib.util.spec_from_file_location``),
which skips the package ``__init__`` files that import Taichi.  The inputs
(meshes, shape-function gradients, Cauchy stresses) come from the project's
generators and the FP64 oracle; the outputs stored here are the reference's.
Sparse matrices are stored as probes (K V for four seeded vectors, the
diagonal, the number of stored entries after duplicates are summed, the
number of entries above 1e-10 of the largest, and the Frobenius norm) to keep the fixture small; voxel meshes are stored whole.

Run ``python tests/golden/gen_reference_fixtures.py [reference_root]``
(default ``/root/reference``).  It writes ``ref_assembly.npz``,
``ref_voxel_to_hex.npz`` and ``ref_contact.npz`` next to this file.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle import fem_oracle as O  # noqa: E402
from simul_b200 import meshgen  # noqa: E402

DEFAULT_REFERENCE = "/root/reference"
ASSEMBLY = "backend/fea/fem/solver/assembly.py"
VOXEL_TO_HEX = "backend/preprocessing/voxel_to_hex.py"
CONTACT = "backend/fea/framework/contact.py"
N_PROBES = 4


def load_module(reference_root: str, rel: str, name: str):
    """Imports one reference file by path, without its package."""
    path = Path(reference_root) / rel
    if not path.is_file():
        raise FileNotFoundError(path)
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# ───────────────────────── assembly cases (inputs from generators + oracle) ─────────────────────────

def _probe_vectors(n_dof: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).standard_normal((n_dof, N_PROBES))


def probes(K) -> dict:
    """Summary of a sparse matrix that pins every entry up to rounding."""
    K = K.tocsr()
    K.sum_duplicates()
    V = _probe_vectors(K.shape[0], 11)
    big = np.abs(K.data) > 1e-10 * np.abs(K.data).max()
    return {"KV": K @ V, "diag": K.diagonal(), "nnz": np.array(K.nnz), "nnz_significant": np.array(big.sum()),
            "fro": np.array(np.sqrt(np.sum(K.data ** 2)))}


def assembly_cases():
    """name -> dict(mesh, C or C_map + material_ids, sigma, chunk_size)."""
    cases = {}
    bar = meshgen.cantilever_bar()
    m = O.Mesh(bar.X, bar.conn)
    rng = np.random.default_rng(200)
    u = rng.standard_normal(bar.X.shape) * 0.05
    nh = O.Material("neo_hookean", E=17e3, nu=0.3)
    F, sigma, _, _, _ = O.internal_state(m, nh, u)
    cases["bar_nh"] = dict(mesh=m, C=O.isotropic_voigt_C(17e3, 0.3), sigma=sigma, chunk_size=10000)
    ti_C = O.ti_global_C(17e3, 11.5e3, 0.3, 0.35, 3.3e3, (1.0, 1.0, 0.0))
    cases["bar_ti"] = dict(mesh=m, C=ti_C, sigma=sigma, chunk_size=700)
    v = meshgen.vertebral_body(n=12, seed=3)
    mv = O.Mesh(v.X, v.conn)
    ids = (v.E > 1e4).astype(np.int64)          # 1 = cortical shell, 0 = core
    C_map = {0: O.isotropic_voigt_C(300.0, 0.3), 1: O.isotropic_voigt_C(12e3, 0.3)}
    uv = np.zeros_like(v.X)
    uv[:, 2] = -0.01 * v.X[:, 2]
    uv += np.random.default_rng(201).standard_normal(v.X.shape) * 0.005
    j2 = O.Material("j2", E=v.E, nu=0.3, sigma_y=100.0, H=0.02 * v.E)
    _, sv, _, _, _ = O.internal_state(mv, j2, uv, O.J2State.zeros(mv.n_elements))
    cases["vox12_multi"] = dict(mesh=mv, C_map=C_map, material_ids=ids, sigma=sv, chunk_size=3000)
    Xh, ch = meshgen.structured_hex8(6, 3, 3, L=(3.0, 1.0, 1.2))
    mh = O.Mesh(Xh, ch)
    uh = np.random.default_rng(202).standard_normal(Xh.shape) * 0.02
    _, sh, _, _, _ = O.internal_state(mh, O.Material("neo_hookean", E=5e3, nu=0.35), uh)
    cases["hex_nh"] = dict(mesh=mh, C=O.isotropic_voigt_C(5e3, 0.35), sigma=sh, chunk_size=20)
    return cases


def reference_assembly(asm, case) -> dict:
    """The reference's K_material and K_geometric for one case."""
    mesh = case["mesh"]
    ngp = mesh.ngp
    conn = mesh.conn.astype(np.int32)
    if "C_map" in case:
        Km = asm.assemble_stiffness_matrix(conn, mesh.dNdX, mesh.vol, mesh.n_nodes, ngp, 3,
                                           material_ids=case["material_ids"], C_map=case["C_map"],
                                           chunk_size=case["chunk_size"])
    else:
        Km = asm.assemble_stiffness_matrix(conn, mesh.dNdX, mesh.vol, mesh.n_nodes, ngp, 3,
                                           C_single=case["C"], chunk_size=case["chunk_size"])
    Kg = asm.assemble_geometric_stiffness(conn, mesh.dNdX, mesh.vol, case["sigma"], mesh.n_nodes, ngp, 3,
                                          chunk_size=case["chunk_size"])
    out = {}
    for tag, K in (("mat", Km), ("geo", Kg)):
        for k, val in probes(K).items():
            out[f"{tag}_{k}"] = val
    return out


# ───────────────────────── voxel-to-hex cases ─────────────────────────

def voxel_cases():
    """name -> (voxel_centres, spacing)."""
    rng = np.random.default_rng(300)
    cases = {}
    lab = rng.random((9, 8, 7)) < 0.55
    cases["random_iso"] = (meshgen.labelmap_voxel_centers(lab.astype(np.int32), (0.5, 0.5, 0.5)), (0.5, 0.5, 0.5))
    lab2 = (rng.random((7, 10, 6)) < 0.4).astype(np.int32) * 3
    cases["random_aniso"] = (meshgen.labelmap_voxel_centers(lab2, (0.4, 0.55, 0.7), origin=(-3.1, 2.2, 10.0),
                                                            label=3), (0.4, 0.55, 0.7))
    n = 16
    h = 32.0 / n
    c = (np.arange(n) + 0.5) * h
    Xv, Yv, Zv = np.meshgrid(c - 16.0, c - 16.0, c, indexing="ij")
    mask = ((Xv / 15.0) ** 2 + (Yv / 12.0) ** 2 <= 1.0) & (Zv < 25.0)
    vi, vj, vk = np.nonzero(mask)
    centres = np.stack([-16.0 + (vi + 0.5) * h, -16.0 + (vj + 0.5) * h, (vk + 0.5) * h], axis=1)
    cases["vertebra16"] = (centres, (h, h, h))
    cases["one_voxel"] = (np.array([[0.25, -0.5, 1.75]]), (0.5, 1.0, 0.25))
    # voxels listed out of lattice order (the mesher must not depend on the order)
    cen = cases["random_iso"][0]
    cases["shuffled"] = (cen[rng.permutation(cen.shape[0])], (0.5, 0.5, 0.5))
    return cases


# ───────────────────────── contact cases ─────────────────────────

def contact_cases():
    """name -> (pos_a, pos_b, surface_a, surface_b, gap, penalty): seeded
    point sets (current coordinates) with a band of near pairs, and the
    two-block interface of the staggered-solve test."""
    rng = np.random.default_rng(400)
    cases = {}
    pa = rng.uniform(0.0, 1.0, (300, 3))
    pb = pa[rng.permutation(300)[:200]] + rng.normal(0.0, 0.05, (200, 3))
    cases["cloud"] = (pa, pb, np.arange(0, 300, 2), np.arange(1, 200), 0.08, 37.5)
    Xa, _ = meshgen.structured_tets(4, 4, 4, L=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 1.05))
    Xb, _ = meshgen.structured_tets(4, 4, 4, L=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0))
    Xa = Xa + rng.normal(0.0, 0.003, Xa.shape)
    sa = np.where(np.isclose(Xa[:, 2], Xa[:, 2].min(), atol=0.02))[0]
    sb = np.where(np.isclose(Xb[:, 2], Xb[:, 2].max()))[0]
    cases["blocks"] = (Xa, Xb, sa, sb, 0.1, 2.0)
    return cases


def reference_contact(con, case) -> dict:
    pa, pb, sa, sb, gap, pen = case
    algo = con.NodeNodeContact()
    pairs, gaps = algo.detect(pa, pb, sa, sb, gap)
    fa, fb = algo.compute_forces(pa, pb, pairs, gaps, pen, gap)
    tp, off = algo.detect_tied_pairs(pa, pb, sa, sb, gap)
    # the tied springs after a seeded motion of both sets
    rng = np.random.default_rng(401)
    qa = pa + rng.normal(0.0, 0.01, pa.shape)
    qb = pb + rng.normal(0.0, 0.01, pb.shape)
    ta, tb = algo.compute_tied_forces(qa, qb, tp, off, pen)
    return {"pairs": pairs, "gaps": gaps, "fa": fa, "fb": fb, "tied_pairs": tp, "tied_offsets": off,
            "tied_fa": ta, "tied_fb": tb, "qa": qa, "qb": qb}


def main(reference_root: str = DEFAULT_REFERENCE):
    asm = load_module(reference_root, ASSEMBLY, "ref_assembly")
    v2h = load_module(reference_root, VOXEL_TO_HEX, "ref_voxel_to_hex")
    out = {}
    for name, case in assembly_cases().items():
        for k, val in reference_assembly(asm, case).items():
            out[f"{name}__{k}"] = val
    np.savez_compressed(HERE / "ref_assembly.npz", **out)
    vox = {}
    for name, (centres, spacing) in voxel_cases().items():
        nodes, elems = v2h.voxels_to_hex_mesh(centres, np.asarray(spacing))
        vox[f"{name}__nodes"] = nodes
        vox[f"{name}__elements"] = elems
    np.savez_compressed(HERE / "ref_voxel_to_hex.npz", **vox)
    con = load_module(reference_root, CONTACT, "ref_contact")
    cont = {}
    for name, case in contact_cases().items():
        for k, val in reference_contact(con, case).items():
            cont[f"{name}__{k}"] = val
    np.savez_compressed(HERE / "ref_contact.npz", **cont)
    print("ref_assembly.npz:", len(out), "arrays; ref_voxel_to_hex.npz:", len(vox), "arrays; ref_contact.npz:",
          len(cont), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_REFERENCE)
