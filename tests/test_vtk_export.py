"""VTU export (simul_b200.vtk_export, vtk_export.py:60-389): the written XML
parses, holds the cells, points and fields, and the base64 blocks decode to
the arrays written; a series writes a .pvd collection."""
import base64
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from simul_b200 import meshgen
from simul_b200.vtk_export import export_vtk, export_vtk_series


def _decode(el, dtype):
    raw = base64.b64decode(el.text)
    n = struct.unpack("<I", raw[:4])[0]
    return np.frombuffer(raw[4:4 + n], dtype=dtype)


@pytest.mark.parametrize("binary", [False, True])
def test_export_vtk_roundtrip(tmp_path, binary):
    bar = meshgen.cantilever_bar(nx=3, ny=1, nz=1)
    rng = np.random.default_rng(0)
    u = rng.standard_normal(bar.X.shape)
    mises = rng.random(bar.n_nodes)
    sig = rng.standard_normal((bar.n_elements, 3, 3))
    path = export_vtk(str(tmp_path / "out"), bar.X, bar.conn, 3, 4,
                      {"displacement": u, "von_mises": mises}, {"stress": sig}, binary=binary)
    assert path.endswith(".vtu")
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    assert int(piece.get("NumberOfPoints")) == bar.n_nodes
    assert int(piece.get("NumberOfCells")) == bar.n_elements
    arrays = {el.get("Name"): el for el in piece.iter("DataArray")}
    if binary:
        conn = _decode(arrays["connectivity"], np.int64).reshape(-1, 4)
        disp = _decode(arrays["displacement"], np.float64).reshape(-1, 3)
        vm = _decode(arrays["von_mises"], np.float64)
        st = _decode(arrays["stress"], np.float64).reshape(-1, 6)
        types = _decode(arrays["types"], np.uint8)
    else:
        conn = np.array(arrays["connectivity"].text.split(), dtype=np.int64).reshape(-1, 4)
        disp = np.array(arrays["displacement"].text.split(), dtype=np.float64).reshape(-1, 3)
        vm = np.array(arrays["von_mises"].text.split(), dtype=np.float64)
        st = np.array(arrays["stress"].text.split(), dtype=np.float64).reshape(-1, 6)
        types = np.array(arrays["types"].text.split(), dtype=np.int64)
    assert np.array_equal(conn, bar.conn) and np.all(types == 10)
    assert np.allclose(disp, u, rtol=0, atol=0 if binary else 1e-15)
    assert np.allclose(vm, mises, rtol=0, atol=0 if binary else 1e-15)
    voigt = np.stack([sig[:, 0, 0], sig[:, 1, 1], sig[:, 2, 2], sig[:, 0, 1], sig[:, 1, 2], sig[:, 0, 2]], 1)
    assert np.allclose(st, voigt, rtol=0, atol=0 if binary else 1e-15)


def test_export_series_writes_collection(tmp_path):
    bar = meshgen.cantilever_bar(nx=2, ny=1, nz=1)
    series = [{"displacement": np.full(bar.X.shape, float(k))} for k in range(3)]
    pvd = export_vtk_series(str(tmp_path / "run"), bar.X, bar.conn, series, times=[0.0, 0.5, 1.0], nodes_per_elem=4)
    ds = ET.parse(pvd).getroot().findall("Collection/DataSet")
    assert [d.get("timestep") for d in ds] == ["0.0", "0.5", "1.0"]
    assert all((tmp_path / d.get("file")).exists() for d in ds)


def test_bad_field_shape_raises(tmp_path):
    bar = meshgen.cantilever_bar(nx=2, ny=1, nz=1)
    with pytest.raises(ValueError):
        export_vtk(str(tmp_path / "bad.vtu"), bar.X, bar.conn, 3, 4, {"x": np.zeros(bar.n_nodes + 1)})
