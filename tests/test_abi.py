"""The C-ABI library loads and exports what include/femb200.h declares (CPU only)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from simul_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "femb200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fem_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_struct_layouts_match_c(tmp_path):
    probe = tmp_path / "probe.c"
    probe.write_text(f'''
#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu\\n", sizeof(FemMeshDesc), sizeof(FemMaterial), sizeof(FemSolveParams), sizeof(FemSolveResult));
  printf("%zu %zu %zu %zu\\n", offsetof(FemMaterial, C_voigt), offsetof(FemMaterial, fiber_E),
         offsetof(FemSolveParams, progress), offsetof(FemSolveResult, first_residual));
  return 0;
}}''')
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-O0", "-o", str(exe), str(probe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(v) for v in out]
    assert sizes[:4] == [C.sizeof(_lib.FemMeshDesc), C.sizeof(_lib.FemMaterial),
                         C.sizeof(_lib.FemSolveParams), C.sizeof(_lib.FemSolveResult)]
    assert sizes[4:] == [_lib.FemMaterial.C_voigt.offset, _lib.FemMaterial.fiber_E.offset,
                         _lib.FemSolveParams.progress.offset, _lib.FemSolveResult.first_residual.offset]


def test_default_solve_params_without_gpu():
    p = _lib.FemSolveParams()
    _lib.load().fem_default_solve_params(C.byref(p))
    assert p.max_iterations == 50 and p.tol == pytest.approx(1e-8)
    assert p.precond == _lib.FEM_PRECOND_JACOBI and p.auto_commit == 1


def test_create_rejects_bad_mesh_before_touching_the_gpu():
    import numpy as np
    lib = _lib.load()
    X = np.zeros((4, 3))
    conn = np.array([[0, 1, 2, 9]], dtype=np.int32)
    desc = _lib.FemMeshDesc(4, 1, X.ctypes.data_as(C.POINTER(C.c_double)),
                            conn.ctypes.data_as(C.POINTER(C.c_int32)), 0, 0, None)
    ctx = C.c_void_p()
    assert lib.fem_ctx_create(C.byref(desc), C.byref(ctx)) == _lib.FEM_ERR_INVALID
    assert "out of range" in _lib.last_error(None)
    assert not ctx.value
