"""Nodal von Mises stress (fem_nodal_mises, core/mesh.py:459-492) against the
FP64 oracle: the reference's summed form and the averaged form, for a
hyperelastic bar at a random displacement and the J2 body at its golden
plastic state; the gather is deterministic (bitwise equal on repeat)."""
import numpy as np
import pytest
import torch

from oracle import fem_oracle as O
from simul_b200 import fem as B
from simul_b200 import meshgen
from tests.golden import gen_golden as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("average", [False, True])
def test_nodal_mises_neo_hookean_matches_oracle(cuda, average):
    bar = meshgen.cantilever_bar()
    mesh = B.FEMesh(bar.n_nodes, bar.n_elements, device=cuda)
    mesh.initialize_from_numpy(bar.X, bar.conn)
    mat = B.NeoHookean(17e3, 0.3)
    u = np.random.default_rng(7).standard_normal(bar.X.shape) * 0.02
    mesh.u.copy_(torch.from_numpy(u))
    mat.compute_stress(mesh)
    mesh.compute_mises_stress(average=average)
    got = mesh.mises.cpu().numpy()
    ref = O.nodal_mises(O.Mesh(bar.X, bar.conn), O.Material("neo_hookean", E=17e3, nu=0.3), u, average=average)
    assert np.max(np.abs(got - ref)) <= 1e-9 * np.max(np.abs(ref))
    mesh.compute_mises_stress(average=average)
    assert np.array_equal(mesh.mises.cpu().numpy(), got)


def test_nodal_mises_j2_through_static_solver(cuda):
    vox = G.vox_mesh()
    ref = np.load(G.path_of("vox12_j2_forces"))
    mesh = B.FEMesh(vox.X.shape[0], vox.conn.shape[0], device=cuda)
    mesh.initialize_from_numpy(vox.X, vox.conn)
    mat = B.J2Plasticity(vox.E, 0.3, 100.0, hardening_modulus=0.02 * vox.E)
    solver = B.StaticSolver(mesh, mat)
    mesh.u.copy_(torch.from_numpy(ref["u"]))
    got = solver.get_mises_stress()
    om = O.Material("j2", E=vox.E, nu=0.3, sigma_y=100.0, H=0.02 * vox.E)
    want = O.nodal_mises(O.Mesh(vox.X, vox.conn), om, ref["u"])
    # the return map rounds a little differently on each side near the yield surface
    assert np.max(np.abs(got - want)) <= 1e-8 * np.max(np.abs(want))


def test_export_mesh_result_writes_gpu_fields(cuda, tmp_path):
    import xml.etree.ElementTree as ET
    from simul_b200.vtk_export import export_mesh_result
    bar = meshgen.cantilever_bar(nx=4, ny=2, nz=2)
    mesh = B.FEMesh(bar.n_nodes, bar.n_elements, device=cuda)
    mesh.initialize_from_numpy(bar.X, bar.conn)
    mat = B.NeoHookean(17e3, 0.3)
    u = np.random.default_rng(8).standard_normal(bar.X.shape) * 0.01
    mesh.u.copy_(torch.from_numpy(u))
    path = export_mesh_result(str(tmp_path / "bar"), mesh, mat, binary=False)
    arrays = {el.get("Name"): el for el in ET.parse(path).getroot().iter("DataArray")}
    vm = np.array(arrays["von_mises"].text.split(), dtype=np.float64)
    ref = O.nodal_mises(O.Mesh(bar.X, bar.conn), O.Material("neo_hookean", E=17e3, nu=0.3), u)
    assert np.max(np.abs(vm - ref)) <= 1e-9 * np.max(np.abs(ref))
