"""Python driver of the C++/OpenMP CPU restatement (oracle/cpu_fem.cpp).

Test and benchmark infrastructure: the CPU baseline, never the product.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import build_cpu

MODELS = {"linear_elastic": 0, "neo_hookean": 1, "j2": 3}


class CpuSolver:
    def __init__(self, X, conn, model, E, nu=0.3, sigma_y=0.0, H_ratio=0.0, threads=0):
        self.lib = build_cpu.load()
        self.X = np.ascontiguousarray(X, dtype=np.float64)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32)
        self.E = np.ascontiguousarray(np.broadcast_to(np.asarray(E, dtype=np.float64), (self.conn.shape[0],)))
        self.model = MODELS[model]
        self.nu, self.sy, self.Hr = float(nu), float(sigma_y), float(H_ratio)
        self.threads = int(threads)
        self.u = np.zeros_like(self.X)
        self.ep = np.zeros((self.conn.shape[0], 6))
        self.epe = np.zeros(self.conn.shape[0])

    @property
    def n_threads(self):
        if self.threads > 0:
            return self.threads
        return int(self.lib.cpu_fem_threads())

    def solve(self, fixed_mask, fixed_vals, f_ext, tol=1e-8, max_newton=50, max_cg=20000,
              cg_rtol_min=1e-5, max_cg_total=0):
        P = C.POINTER
        fm = np.ascontiguousarray(fixed_mask, dtype=np.uint8)
        fv = np.ascontiguousarray(fixed_vals, dtype=np.float64)
        fe = np.ascontiguousarray(f_ext, dtype=np.float64)
        stats = np.zeros(5)
        d = lambda a: a.ctypes.data_as(P(C.c_double))
        self.lib.cpu_fem_solve(self.X.shape[0], self.conn.shape[0], d(self.X),
                               self.conn.ctypes.data_as(P(C.c_int)), self.model, d(self.E),
                               self.nu, self.sy, self.Hr, fm.ctypes.data_as(P(C.c_uint8)), d(fv), d(fe),
                               d(self.u), d(self.ep), d(self.epe), tol, max_newton, max_cg, cg_rtol_min,
                               max_cg_total, self.threads, d(stats))
        return {"iterations": int(stats[0]), "cg_iterations": int(stats[1]),
                "relative_residual": float(stats[2]), "residual_evals": int(stats[3]),
                "converged": bool(stats[4])}
