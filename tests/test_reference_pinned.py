"""The oracle against outputs of the reference's own code (CPU).

``tests/golden/gen_reference_fixtures.py`` ran the reference's
``fem/solver/assembly.py`` and ``preprocessing/voxel_to_hex.py`` (both pure
numpy/scipy) and stored their outputs.  Here the oracle's restatements of
the reference tangent (``reference_K_material``, ``reference_K_geometric``,
the multi-material grouping) and the project's mesher
(``meshgen.voxels_to_hex_mesh``) must reproduce them: the tangent to 1e-12
relative, the voxel mesh bit for bit.  When the reference tree is present
the same checks also run live against the imported modules.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import fem_oracle as O
from simul_b200 import meshgen
from tests.golden import gen_reference_fixtures as R

ASM = np.load(R.HERE / "ref_assembly.npz")
VOX = np.load(R.HERE / "ref_voxel_to_hex.npz")
CASES = R.assembly_cases()


def _oracle_K(case):
    mesh = case["mesh"]
    if "C_map" in case:
        Km = O._multi_material_K(mesh, case["C_map"], case["material_ids"])
    else:
        Km = O.reference_K_material(mesh, case["C"])
    Kg = O.reference_K_geometric(mesh, case["sigma"])
    return Km, Kg


def _close(a, b, tol=1e-12):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_tangent_matches_reference_assembler(name):
    Km, Kg = _oracle_K(CASES[name])
    for tag, K in (("mat", Km), ("geo", Kg)):
        got = R.probes(K)
        for key in ("KV", "diag", "fro"):
            ref = ASM[f"{name}__{tag}_{key}"]
            assert _close(got[key], ref), (name, tag, key, np.abs(got[key] - ref).max())


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_tangent_sparsity_matches_reference(name):
    # the same pattern of significant entries once duplicates are summed.
    # Entries whose element contributions cancel can end as an exact zero in
    # one summation order and as a rounding residue in another (per Gauss
    # point here, per element in assembly.py:150; per material here, one COO
    # in assembly.py:121-139), so exact stored counts are compared only where
    # both sum in the same order (one TET4 material).
    Km, Kg = _oracle_K(CASES[name])
    pm, pg = R.probes(Km), R.probes(Kg)
    assert pm["nnz_significant"] == ASM[f"{name}__mat_nnz_significant"]
    assert pg["nnz_significant"] == ASM[f"{name}__geo_nnz_significant"]
    if "C_map" not in CASES[name] and CASES[name]["mesh"].ngp == 1:
        assert pm["nnz"] == ASM[f"{name}__mat_nnz"]
        assert pg["nnz"] == ASM[f"{name}__geo_nnz"]


@pytest.mark.parametrize("name", sorted(R.voxel_cases()))
def test_voxels_to_hex_mesh_bit_identical_to_reference(name):
    centres, spacing = R.voxel_cases()[name]
    nodes, elems = meshgen.voxels_to_hex_mesh(centres, spacing)
    ref_nodes, ref_elems = VOX[f"{name}__nodes"], VOX[f"{name}__elements"]
    assert nodes.dtype == ref_nodes.dtype and elems.dtype == ref_elems.dtype
    assert nodes.shape == ref_nodes.shape and elems.shape == ref_elems.shape
    assert nodes.tobytes() == ref_nodes.tobytes()
    assert elems.tobytes() == ref_elems.tobytes()


def test_reference_tangent_drives_the_reference_newton():
    # the oracle's reference-quirk Newton assembles exactly the pinned
    # matrices: one iteration's tangent equals K_mat + K_geo at its state
    case = CASES["bar_nh"]
    Km, Kg = _oracle_K(case)
    K = (Km + Kg).tocsr()
    ref = ASM["bar_nh__mat_KV"] + ASM["bar_nh__geo_KV"]
    assert _close(K @ R._probe_vectors(K.shape[0], 11), ref)


_REF_ROOT = os.environ.get("SIMUL_REFERENCE_ROOT", R.DEFAULT_REFERENCE)
_HAS_REF = os.path.isfile(os.path.join(_REF_ROOT, R.ASSEMBLY))


@pytest.mark.skipif(not _HAS_REF, reason="reference tree not present")
def test_live_reference_assembler_and_mesher():
    asm = R.load_module(_REF_ROOT, R.ASSEMBLY, "ref_assembly_live")
    v2h = R.load_module(_REF_ROOT, R.VOXEL_TO_HEX, "ref_voxel_to_hex_live")
    for name, case in CASES.items():
        ref = R.reference_assembly(asm, case)
        Km, Kg = _oracle_K(case)
        for tag, K in (("mat", Km), ("geo", Kg)):
            got = R.probes(K)
            assert _close(got["KV"], ref[f"{tag}_KV"]), (name, tag)
    for name, (centres, spacing) in R.voxel_cases().items():
        a = v2h.voxels_to_hex_mesh(centres, np.asarray(spacing))
        b = meshgen.voxels_to_hex_mesh(centres, spacing)
        assert a[0].tobytes() == b[0].tobytes() and a[1].tobytes() == b[1].tobytes(), name
