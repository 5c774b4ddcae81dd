"""Generates the golden fixtures under tests/golden/ from the FP64 oracle.

The reference ships no golden vectors and cannot run here (Taichi is not
installed), so the fixtures are the oracle's outputs on seeded inputs; the
oracle itself is pinned by tests/test_oracle.py against the reference's
known-answer tests and by tests/test_reference_pinned.py against outputs of
the reference's own assembler and mesher.  Run
``python tests/golden/gen_golden.py [case ...]`` to regenerate all (or the
named) fixtures.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle import fem_oracle as O  # noqa: E402
from simul_b200 import meshgen  # noqa: E402

FIBRES = np.array([[np.cos(np.pi / 6), np.sin(np.pi / 6), 0.0],
                   [np.cos(np.pi / 6), -np.sin(np.pi / 6), 0.0]])
TI_C = O.ti_global_C(17e3, 11.5e3, 0.3, 0.35, 3.3e3, (1.0, 1.0, 0.0))

MATERIALS = {
    "nh": O.Material("neo_hookean", E=17e3, nu=0.3),
    "mr": O.Material("mooney_rivlin", C10=0.18, C01=0.045, D1=0.5),
    "fmr": O.Material("ti_hyper", C10=0.18, C01=0.045, D1=0.5, fiber_a=FIBRES, fiber_E=500.0),
    "le": O.Material("linear_elastic", E=1e3, nu=0.3),
    "ti": O.Material("transverse_isotropic", C_voigt=TI_C),
}
DISP_SCALE = {"nh": 0.05, "mr": 0.3, "fmr": 0.3, "le": 0.05, "ti": 0.05}


def mesh_checksum(X, conn) -> np.ndarray:
    """Order-sensitive fingerprint of a generated mesh (detects generator drift)."""
    w = np.arange(1, X.shape[0] + 1, dtype=np.float64)
    return np.array([np.sum(X * w[:, None]), float(np.sum(conn.astype(np.int64) * np.arange(1, 5))),
                     X.shape[0], conn.shape[0]])


def vox_mesh():
    return _vox_mesh()


def bar_mesh():
    return _bar()


def path_of(name: str) -> Path:
    return HERE / f"{name}.npz"


def _bar():
    return meshgen.cantilever_bar()


def _forces_case(key):
    def make():
        bar = _bar()
        m = O.Mesh(bar.X, bar.conn)
        rng = np.random.default_rng(100 + list(MATERIALS).index(key))
        u = rng.standard_normal(bar.X.shape) * DISP_SCALE[key]
        p = rng.standard_normal(bar.X.shape)
        mat = MATERIALS[key]
        F, sigma, P, f, aux = O.internal_state(m, mat, u)
        y = O.tangent_matvec(mat, F, None, m.dNdX, m.vol, m.conn, p)
        out = {"mesh_sum": mesh_checksum(bar.X, bar.conn), "u": u, "p": p, "f": f,
               "sigma": sigma, "y": y}
        if key == "nh":
            out.update(F=F, dNdX=m.dNdX, vol=m.vol)
        return out
    return make


def _vox_mesh(n=12):
    v = meshgen.vertebral_body(n=n, seed=3)
    return v


def _j2_forces():
    v = _vox_mesh()
    m = O.Mesh(v.X, v.conn)
    rng = np.random.default_rng(7)
    # smooth compression plus noise, large enough to yield the shell
    u = np.zeros_like(v.X)
    u[:, 2] = -0.01 * v.X[:, 2]
    u += rng.standard_normal(v.X.shape) * 0.01
    p = rng.standard_normal(v.X.shape)
    mat = O.Material("j2", E=v.E, nu=0.3, sigma_y=100.0, H=0.02 * v.E)
    st = O.J2State.zeros(m.n_elements)
    F, sigma, P, f, aux = O.internal_state(m, mat, u, st)
    y = O.tangent_matvec(mat, F, aux[1], m.dNdX, m.vol, m.conn, p)
    return {"mesh_sum": mesh_checksum(v.X, v.conn), "u": u, "p": p, "f": f,
            "sigma": sigma, "y": y, "epe": aux[0].epe, "ep": aux[0].ep}


def _j2_steps(n_steps=4, total=20):
    v = _vox_mesh()
    m = O.Mesh(v.X, v.conn)
    mat = O.Material("j2", E=v.E, nu=0.3, sigma_y=100.0, H=0.02 * v.E)
    st = O.J2State.zeros(m.n_elements)
    u = np.zeros_like(v.X)
    us, epes, iters = [], [], []
    # a stronger compression than the full-size workload so the shell yields within 4 steps
    for k in range(1, n_steps + 1):
        fv = v.fixed_vals * (k / total) * 5.0
        u, info = O.consistent_newton(m, mat, v.f_ext, v.fixed_mask, fv, u0=u, j2_state=st, tol=1e-11,
                                      line_search=False)
        assert info["converged"], info
        us.append(u.copy())
        epes.append(st.epe.copy())
        iters.append(info["iterations"])
    return {"mesh_sum": mesh_checksum(v.X, v.conn), "load_factor": np.array(5.0),
            "u_steps": np.array(us), "epe_steps": np.array(epes),
            "n_total": np.array(total), "iters": np.array(iters)}


def _bar_steps(n_steps=10):
    """The plain-method cantilever workload: all ten traction load steps,
    each a solve to 1e-10 relative residual from the previous step's state."""
    bar = _bar()
    m = O.Mesh(bar.X, bar.conn)
    mat = MATERIALS["nh"]
    u = np.zeros_like(bar.X)
    us, iters, rels = [], [], []
    for k in range(1, n_steps + 1):
        u, info = O.consistent_newton(m, mat, bar.f_ext * k / 10.0, bar.fixed_mask, bar.fixed_vals,
                                      u0=u, tol=1e-10, line_search=False)
        assert info["converged"]
        us.append(u.copy())
        iters.append(info["iterations"])
        rels.append(info["relative_residual"])
    return {"mesh_sum": mesh_checksum(bar.X, bar.conn), "u_steps": np.array(us),
            "iters": np.array(iters), "relative_residual": np.array(rels)}


CASES = {f"bar_{k}_forces": _forces_case(k) for k in MATERIALS}
CASES["vox12_j2_forces"] = _j2_forces
CASES["vox12_j2_steps"] = _j2_steps
CASES["bar_nh_steps"] = _bar_steps


def main(names=None):
    for name, make in CASES.items():
        if names and name not in names:
            continue
        out = make()
        np.savez_compressed(path_of(name), **out)
        print(name, {k: v.shape for k, v in out.items()}, os.path.getsize(path_of(name)))


if __name__ == "__main__":
    main(sys.argv[1:])
