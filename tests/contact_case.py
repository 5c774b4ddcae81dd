"""The two-block contact workload shared by the CPU and GPU contact tests.

Block A (upper, [0,1]^2 x [1.05, 2.05]) and block B (lower, [0,1]^3), each
4 x 4 x 4 hexahedra split into 6 tets, linear elastic E = 1000, nu = 0.3.
B's bottom face is fixed; A's top face is fixed with u_z = -0.03, which
brings A's bottom face within 0.02 of B's top face.  The contact pairs A's
bottom-face nodes with B's top-face nodes (gap tolerance 0.1, penalty 2):
the staggered solve converges to 1e-3 in about 14 contact iterations.
"""
import numpy as np

from simul_b200 import meshgen

E, NU = 1000.0, 0.3
GAP, PENALTY, TOP_DZ = 0.1, 2.0, -0.03


def blocks():
    Xa, ca = meshgen.structured_tets(4, 4, 4, L=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 1.05))
    Xb, cb = meshgen.structured_tets(4, 4, 4, L=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0))
    top_a = np.isclose(Xa[:, 2], Xa[:, 2].max())
    fixed_a = np.zeros(Xa.shape, dtype=bool)
    fixed_a[top_a] = True
    vals_a = np.zeros_like(Xa)
    vals_a[top_a, 2] = TOP_DZ
    fixed_b = np.zeros(Xb.shape, dtype=bool)
    fixed_b[np.isclose(Xb[:, 2], 0.0)] = True
    surf_a = np.where(np.isclose(Xa[:, 2], Xa[:, 2].min()))[0]
    surf_b = np.where(np.isclose(Xb[:, 2], Xb[:, 2].max()))[0]
    return {"a": (Xa, ca, fixed_a, vals_a), "b": (Xb, cb, fixed_b, np.zeros_like(Xb)),
            "surf_a": surf_a, "surf_b": surf_b}
