"""The C++/OpenMP CPU restatement agrees with the NumPy oracle (CPU only)."""
import numpy as np

from oracle.cpu_solver import CpuSolver
from simul_b200 import meshgen
from tests.golden import gen_golden as G


def test_cpu_restatement_bar_matches_oracle():
    ref = np.load(G.path_of("bar_nh_steps"))
    bar = meshgen.cantilever_bar()
    s = CpuSolver(bar.X, bar.conn, "neo_hookean", 17e3, 0.3)
    for k in range(ref["u_steps"].shape[0]):
        info = s.solve(bar.fixed_mask, bar.fixed_vals, bar.f_ext * (k + 1) / 10.0, tol=1e-10)
        assert info["converged"], info
        assert np.linalg.norm(s.u - ref["u_steps"][k]) / np.linalg.norm(ref["u_steps"][k]) < 1e-6


def test_cpu_restatement_j2_matches_oracle():
    ref = np.load(G.path_of("vox12_j2_steps"))
    v = G.vox_mesh()
    s = CpuSolver(v.X, v.conn, "j2", v.E, 0.3, sigma_y=100.0, H_ratio=0.02)
    lf, total = float(ref["load_factor"]), int(ref["n_total"])
    for k in range(ref["u_steps"].shape[0]):
        info = s.solve(v.fixed_mask, v.fixed_vals * (k + 1) / total * lf, v.f_ext, tol=1e-10)
        assert info["converged"], info
        assert np.linalg.norm(s.u - ref["u_steps"][k]) / np.linalg.norm(ref["u_steps"][k]) < 1e-6
        assert np.abs(s.epe - ref["epe_steps"][k]).max() <= 1e-6 * max(ref["epe_steps"][k].max(), 1e-12) + 1e-12
