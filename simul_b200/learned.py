"""Learned preconditioner: weights, training data from the plain solver, training.

The network (a 4-layer message-passing network over mesh nodes, width 64,
BF16 weights on the tensor cores) is applied inside flexible PCG by
``StaticSolver(..., precond="learned")``.  Everything here drives the C ABI
(``fem_mpnn_*``): pairs are produced by the library's own Jacobi-PCG, the
forward and backward passes and the Adam updates run on the GPU.

Typical use::

    pairs = solver_pairs(mesh, random_rhs(mesh_X, fixed_mask, 64, rng))
    set_weights(mesh, init_weights(seed=0))
    train(mesh, *pairs, steps=400, batch=8, lr=2e-3)
    w = get_weights(mesh)            # reuse on other meshes: set_weights(other, w)
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .fem import _ptr
from .validation import FEAValidationError

HIDDEN = 64
IN_FEATURES = 16
N_LAYERS = 4
N_PARAMS = _lib.MPNN_PARAMS


def init_weights(seed: int = 0, out_scale: float = 0.0) -> np.ndarray:
    """He-style initial weights in the ABI's flat order; a zero decoder
    (``out_scale=0``) makes the preconditioner exactly Jacobi at start."""
    rng = np.random.default_rng(seed)
    parts = [rng.standard_normal((HIDDEN, IN_FEATURES)) * np.sqrt(2.0 / 7.0), np.zeros(HIDDEN)]
    for _ in range(N_LAYERS):
        parts += [rng.standard_normal((HIDDEN, 2 * HIDDEN)) * np.sqrt(2.0 / (2 * HIDDEN)) * 0.5, np.zeros(HIDDEN)]
    parts += [rng.standard_normal((3, HIDDEN)) * out_scale, np.zeros(3)]
    w = np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)
    assert w.size == N_PARAMS
    return w


def set_weights(mesh, w) -> None:
    w = np.ascontiguousarray(np.asarray(w, dtype=np.float32).reshape(-1))
    rc = _lib.load().fem_mpnn_set_weights(mesh.ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size)
    _check(rc, mesh, "fem_mpnn_set_weights")


def get_weights(mesh) -> np.ndarray:
    w = np.zeros(N_PARAMS, dtype=np.float32)
    rc = _lib.load().fem_mpnn_get_weights(mesh.ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size)
    _check(rc, mesh, "fem_mpnn_get_weights")
    return w


def save(path, w) -> None:
    np.savez_compressed(path, w=np.asarray(w, dtype=np.float32), n_params=N_PARAMS)


def load(path) -> np.ndarray:
    d = np.load(Path(path))
    w = d["w"].astype(np.float32)
    if w.size != N_PARAMS:
        raise FEAValidationError(f"weights file has {w.size} parameters, expected {N_PARAMS}")
    return w


def random_rhs(X: np.ndarray, fixed_mask: np.ndarray, n: int, rng, n_modes: int = 6,
               rough: float = 0.3) -> np.ndarray:
    """Right-hand sides for training pairs: random smooth fields (sums of
    sinusoids with random wave vectors over the mesh's extent) plus a rough
    white-noise part, zero on fixed DOFs.  Returns (n, N, 3) float64."""
    X = np.asarray(X, dtype=np.float64)
    lo, hi = X.min(0), X.max(0)
    ext = np.maximum(hi - lo, 1e-12)
    out = np.zeros((n, X.shape[0], 3))
    for k in range(n):
        f = np.zeros((X.shape[0], 3))
        for _ in range(n_modes):
            kv = rng.integers(0, 4, size=3) * np.pi / ext
            ph = rng.uniform(0, 2 * np.pi)
            amp = rng.standard_normal(3)
            f += np.sin((X - lo) @ kv + ph)[:, None] * amp[None, :]
        f /= max(np.sqrt(np.mean(f * f)), 1e-30)
        f += rough * rng.standard_normal(f.shape)
        f[np.asarray(fixed_mask, dtype=bool)] = 0.0
        out[k] = f
    return out


def solver_pairs(mesh, rhs: np.ndarray, rtol: float = 1e-6, max_iterations: int = 20000):
    """(R, E) device tensors [n, N, 3] FP32: each E_k solves K_ff E_k = R_k with
    the library's Jacobi-PCG at the mesh's current tangent."""
    lib = _lib.load()
    dev = mesh.device
    n = rhs.shape[0]
    R = torch.as_tensor(np.asarray(rhs, dtype=np.float32), device=dev).contiguous()
    E = torch.empty_like(R)
    r64 = torch.empty(rhs.shape[1:], dtype=torch.float64, device=dev)
    du = torch.empty_like(r64)
    it = C.c_int32()
    rel = C.c_double()
    for k in range(n):
        r64.copy_(R[k])
        rc = lib.fem_pcg(mesh.ctx, _lib.FEM_PRECOND_JACOBI, _ptr(r64), _ptr(du),
                         rtol, max_iterations, C.byref(it), C.byref(rel))
        _check(rc, mesh, "fem_pcg")
        E[k].copy_(du)
    torch.cuda.synchronize(dev)
    return R, E


def train(mesh, R, E, steps: int = 300, batch: int = 8, lr: float = 2e-3, seed: int = 0,
          reset_optimizer: bool = True) -> dict:
    """Adam on the GPU; returns the mean loss at the start and at the end."""
    prm = _lib.FemTrainParams()
    prm.steps = int(steps)
    prm.batch = int(batch)
    prm.lr = float(lr)
    prm.seed = int(seed)
    prm.reset_optimizer = 1 if reset_optimizer else 0
    prm.progress = _lib.PROGRESS_FN(0)
    prm.progress_user = None
    res = _lib.FemTrainResult()
    rc = _lib.load().fem_mpnn_train(mesh.ctx, _ptr(R), _ptr(E), int(R.shape[0]),
                                    C.byref(prm), C.byref(res))
    _check(rc, mesh, "fem_mpnn_train")
    return {"steps": res.steps_done, "loss_first": res.loss_first, "loss_last": res.loss_last}


def evaluate(mesh, R, E) -> dict:
    """Mean A-norm loss of the network and of the same preconditioner without it."""
    a = C.c_double()
    b = C.c_double()
    rc = _lib.load().fem_mpnn_eval(mesh.ctx, _ptr(R), _ptr(E), int(R.shape[0]),
                                   C.byref(a), C.byref(b))
    _check(rc, mesh, "fem_mpnn_eval")
    return {"loss_net": a.value, "loss_base": b.value}


def set_coarse(mesh, enabled: bool) -> None:
    """Whether the learned preconditioner adds the two-level coarse correction."""
    rc = _lib.load().fem_set_option(mesh.ctx, _lib.FEM_OPT_LEARNED_COARSE, 1 if enabled else 0)
    _check(rc, mesh, "fem_set_option")


def _check(rc, mesh, what):
    from .fem import _check as check
    check(rc, mesh.ctx, what)
