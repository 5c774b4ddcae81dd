"""VTK XML unstructured-grid (.vtu) export of FEM results.

Same entry points and field conventions as the reference's exporter
(backend/fea/fem/io/vtk_export.py:60-389): ``export_vtk`` writes one .vtu
(point data: scalars (n,), vectors (n, 2|3) padded to 3 components, tensors
(n, d, d) as 6 Voigt components; cell data: scalars or vectors per element;
ASCII, or base64 "binary" blocks with a UInt32 byte-count header),
``export_vtk_series`` writes numbered files plus a .pvd collection, and
``export_mesh_result`` writes a GPU mesh's nodes, displacement, nodal von
Mises stress (``fem_nodal_mises``) and element stress.  Host-side IO: no
kernel runs here except the Mises / stress evaluation of
``export_mesh_result``.
"""
from __future__ import annotations

import base64
import struct
import xml.etree.ElementTree as ET
from pathlib import Path
from typing import Dict, List, Optional, Sequence

import numpy as np

_CELL_TYPES = {(2, 3): 5, (2, 4): 9, (3, 4): 10, (3, 8): 12}  # triangle, quad, tetra, hexahedron
_VOIGT = ((0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2))


def _cell_type(dim: int, nodes_per_elem: int) -> int:
    try:
        return _CELL_TYPES[(dim, nodes_per_elem)]
    except KeyError:
        raise ValueError(f"no VTK cell type for dim={dim}, {nodes_per_elem} nodes per element") from None


def _b64(a: np.ndarray) -> str:
    raw = np.ascontiguousarray(a).tobytes()
    return base64.b64encode(struct.pack("<I", len(raw)) + raw).decode("ascii")


def _vtk_type(a: np.ndarray) -> str:
    if a.dtype.kind == "f":
        return "Float64" if a.dtype.itemsize == 8 else "Float32"
    if a.dtype.kind in "iu":
        return {(True, 8): "Int64", (True, 4): "Int32", (True, 1): "Int8",
                (False, 8): "UInt64", (False, 4): "UInt32", (False, 1): "UInt8"}[(a.dtype.kind == "i",
                                                                                  a.dtype.itemsize)]
    raise ValueError(f"unsupported dtype {a.dtype}")


def _data_array(parent, name: Optional[str], a: np.ndarray, ncomp: int, binary: bool):
    attrs = {"type": _vtk_type(a), "format": "binary" if binary else "ascii"}
    if name is not None:
        attrs["Name"] = name
    if ncomp > 1:
        attrs["NumberOfComponents"] = str(ncomp)
    el = ET.SubElement(parent, "DataArray", attrs)
    if binary:
        el.text = _b64(a.reshape(-1))
    else:
        flat = a.reshape(-1)
        el.text = " ".join(repr(float(v)) if a.dtype.kind == "f" else str(int(v)) for v in flat)
    return el


def _as_field(v: np.ndarray, n: int, dim: int, what: str):
    """(array with VTK component layout, number of components)."""
    v = np.asarray(v)
    if v.shape == (n,):
        return v.astype(np.float64), 1
    if v.ndim == 2 and v.shape[0] == n and v.shape[1] in (2, 3):
        out = np.zeros((n, 3))
        out[:, :v.shape[1]] = v
        return out, 3
    if v.ndim == 3 and v.shape[0] == n and v.shape[1] == v.shape[2] == dim:
        comps = [(i, j) for i, j in _VOIGT if i < dim and j < dim]
        return np.stack([v[:, i, j] for i, j in comps], 1).astype(np.float64), len(comps)
    if v.ndim == 2 and v.shape[0] == n:
        return v.astype(np.float64), v.shape[1]
    raise ValueError(f"{what} field of shape {v.shape} does not match {n} entries")


def export_vtk(filename: str, nodes: np.ndarray, elements: np.ndarray, dim: int = 3, nodes_per_elem: int = 8,
               fields: Optional[Dict[str, np.ndarray]] = None, cell_fields: Optional[Dict[str, np.ndarray]] = None,
               binary: bool = False) -> str:
    """Write one .vtu file; returns its path (vtk_export.py:60-180)."""
    fields = fields or {}
    cell_fields = cell_fields or {}
    path = Path(filename)
    if path.suffix != ".vtu":
        path = path.with_suffix(".vtu")
    nodes = np.asarray(nodes, dtype=np.float64)
    elements = np.asarray(elements, dtype=np.int64)
    n, ne = nodes.shape[0], elements.shape[0]
    ctype = _cell_type(dim, nodes_per_elem)
    pts = np.zeros((n, 3))
    pts[:, :nodes.shape[1]] = nodes
    root = ET.Element("VTKFile", {"type": "UnstructuredGrid", "version": "0.1", "byte_order": "LittleEndian",
                                  **({"header_type": "UInt32"} if binary else {})})
    piece = ET.SubElement(ET.SubElement(root, "UnstructuredGrid"), "Piece",
                          {"NumberOfPoints": str(n), "NumberOfCells": str(ne)})
    _data_array(ET.SubElement(piece, "Points"), None, pts, 3, binary)
    cells = ET.SubElement(piece, "Cells")
    _data_array(cells, "connectivity", elements.reshape(-1), 1, binary)
    _data_array(cells, "offsets", np.arange(1, ne + 1, dtype=np.int64) * nodes_per_elem, 1, binary)
    _data_array(cells, "types", np.full(ne, ctype, dtype=np.uint8), 1, binary)
    if fields:
        pd = ET.SubElement(piece, "PointData")
        for name, v in fields.items():
            arr, nc = _as_field(v, n, dim, f"point field {name!r}")
            _data_array(pd, name, arr, nc, binary)
    if cell_fields:
        cd = ET.SubElement(piece, "CellData")
        for name, v in cell_fields.items():
            arr, nc = _as_field(v, ne, dim, f"cell field {name!r}")
            _data_array(cd, name, arr, nc, binary)
    path.parent.mkdir(parents=True, exist_ok=True)
    ET.ElementTree(root).write(path, encoding="utf-8", xml_declaration=True)
    return str(path)


def export_vtk_series(basename: str, nodes: np.ndarray, elements: np.ndarray,
                      field_series: Sequence[Dict[str, np.ndarray]], times: Optional[Sequence[float]] = None,
                      dim: int = 3, nodes_per_elem: int = 8, binary: bool = False) -> str:
    """One .vtu per entry of ``field_series`` and a .pvd collection that
    lists them with their times (vtk_export.py:243-306); returns the .pvd path."""
    base = Path(basename)
    times = list(times) if times is not None else list(range(len(field_series)))
    files: List[str] = []
    for k, fs in enumerate(field_series):
        files.append(export_vtk(str(base.parent / f"{base.stem}_{k:04d}.vtu"), nodes, elements, dim,
                                nodes_per_elem, fs, None, binary))
    root = ET.Element("VTKFile", {"type": "Collection", "version": "0.1", "byte_order": "LittleEndian"})
    col = ET.SubElement(root, "Collection")
    for t, f in zip(times, files):
        ET.SubElement(col, "DataSet", {"timestep": repr(float(t)), "group": "", "part": "0",
                                       "file": Path(f).name})
    pvd = base.with_suffix(".pvd")
    ET.ElementTree(root).write(pvd, encoding="utf-8", xml_declaration=True)
    return str(pvd)


def export_mesh_result(filename: str, mesh, material=None, binary: bool = True, average_mises: bool = False) -> str:
    """Nodes, displacement, nodal von Mises and element stress of a GPU mesh
    (vtk_export.py:309-386).  ``material`` (optional) is bound first; the
    Mises field follows ``fem_nodal_mises`` (the reference's sum unless
    ``average_mises``)."""
    if material is not None:
        material.compute_stress(mesh)
    mesh.compute_mises_stress(average=average_mises)
    fields = {"displacement": mesh.get_displacements(), "von_mises": mesh.mises.cpu().numpy()}
    st = mesh.get_stress()
    # HEX8: the element's Gauss-point mean stress as its cell value
    cell = {"stress": st.reshape(mesh.n_elements, mesh.n_gauss, 3, 3).mean(axis=1)}
    return export_vtk(filename, mesh.X, mesh.elements, 3, mesh.nodes_per_elem, fields, cell, binary)
