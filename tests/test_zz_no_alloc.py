"""Allocation-free entry point fem_dot_f64_noalloc, through the C ABI.

For callers that cannot call cudaMalloc (an application whose allocator owns
all device memory, a loop that forbids allocation after start-up), the
library offers one reduction whose scratch is a static device array.  Its
result must match what the existing entry point reports: the FP64 residual
norm that fem_element_forces computes with context scratch.  Two calls in a
row check that the shared array carries nothing over between calls.  This file
is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from simul_b200 import _lib, meshgen
from simul_b200 import fem as B

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_dot_matches_residual_norm_on_two_calls(cuda):
    bar = meshgen.cantilever_bar()
    mesh = B.FEMesh(bar.n_nodes, bar.n_elements, device=cuda)
    mesh.initialize_from_numpy(bar.X, bar.conn)
    mesh.set_fixed_nodes(np.where(bar.fixed_mask[:, 0])[0])
    mesh.set_nodal_forces(np.arange(bar.n_nodes), bar.f_ext)
    mat = B.NeoHookean(17e3, 0.3)
    mat.compute_nodal_forces(mesh)  # binds the material and pushes the boundary conditions
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    rng = np.random.default_rng(11)
    results = []
    for scale in (0.01, 0.03):       # two calls in a row on different residuals
        u = torch.from_numpy(rng.standard_normal(bar.X.shape) * scale).to(cuda)
        R = torch.empty_like(u)
        rnorm = C.c_double()
        assert lib.fem_element_forces(mesh.ctx, _ptr(u), None, _ptr(R), C.byref(rnorm)) == 0, \
            _lib.last_error(mesh.ctx)
        out = torch.full((1,), -1.0, dtype=torch.float64, device=cuda)
        rc = lib.fem_dot_f64_noalloc(_ptr(R), _ptr(R), R.numel(), _ptr(out), stream)
        assert rc == 0, _lib.last_error(None)
        torch.cuda.synchronize()
        got = float(np.sqrt(out.item()))
        assert got == pytest.approx(rnorm.value, rel=1e-12)
        assert got == pytest.approx(float(R.norm().item()), rel=1e-12)
        results.append(got)
    assert results[0] != results[1]


def test_noalloc_dot_allocates_nothing_and_rejects_oversize(cuda):
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    n = 1_000_003
    a = torch.randn(n, dtype=torch.float64, device=cuda)
    b = torch.randn(n, dtype=torch.float64, device=cuda)
    out = torch.empty(1, dtype=torch.float64, device=cuda)
    assert lib.fem_dot_f64_noalloc(_ptr(a), _ptr(b), n, _ptr(out), stream) == 0  # set-up call
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(cuda)[0]
    vals = []
    for _ in range(3):
        assert lib.fem_dot_f64_noalloc(_ptr(a), _ptr(b), n, _ptr(out), stream) == 0
        torch.cuda.synchronize()
        vals.append(out.item())
    assert torch.cuda.mem_get_info(cuda)[0] == free0
    assert vals[0] == vals[1] == vals[2]                      # deterministic
    assert vals[0] == pytest.approx(float(torch.dot(a, b).item()), rel=1e-10)
    assert lib.fem_dot_f64_noalloc(_ptr(a), _ptr(b), 8_388_609, _ptr(out), stream) == _lib.FEM_ERR_INVALID
    assert "allocation-free maximum" in _lib.last_error(None)
    assert lib.fem_dot_f64_noalloc(_ptr(a), _ptr(b), 0, _ptr(out), stream) == 0
    torch.cuda.synchronize()
    assert out.item() == 0.0
