"""Known-answer check of the tcgen05 tile the learned preconditioner is built on.

BF16 products are exact in FP32, so the tensor-core result differs from an
FP64 product of the same BF16 operands only by FP32 accumulation order:
relative error below 1e-5 of the row magnitude.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from simul_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(64, 128), (128, 64), (64, 16), (16, 32), (256, 256)])
def test_umma_tile_matches_host_product(cuda, N, K):
    g = torch.Generator().manual_seed(N * 1000 + K)
    A = torch.randn(128, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    dA, dB = A.to(cuda), B.to(cuda)
    D = torch.full((128, N), float("nan"), dtype=torch.float32, device=cuda)
    stream = torch.cuda.current_stream(cuda).cuda_stream
    rc = _lib.load().fem_selftest_umma(C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()),
                                       C.c_void_p(D.data_ptr()), N, K, C.c_void_p(stream))
    assert rc == 0, _lib.last_error(None)
    ref = A.double().numpy() @ B.double().numpy().T
    got = D.cpu().numpy().astype(np.float64)
    scale = np.abs(A.double().numpy()) @ np.abs(B.double().numpy()).T
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - ref) / np.maximum(scale, 1e-30)) < 1e-5


def test_umma_rejects_bad_shapes(cuda):
    x = torch.zeros(128 * 256, dtype=torch.bfloat16, device=cuda)
    d = torch.zeros(128 * 256, dtype=torch.float32, device=cuda)
    lib = _lib.load()
    for N, K in [(8, 16), (48, 24), (512, 16), (16, 0)]:
        assert lib.fem_selftest_umma(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()),
                                     C.c_void_p(d.data_ptr()), N, K, None) == _lib.FEM_ERR_INVALID
