"""The dynamic oracle's textbook Newmark (average acceleration) conserves the
energy of an undamped linear system exactly, and its lumped mass adds up to
the body's mass; the reference-as-written form does not conserve it
(dynamic_solver.py:167-208 scales the acceleration by beta dt^2 twice)."""
import numpy as np

from oracle import fem_oracle as O
from oracle.dynamic_oracle import DynamicOracle
from simul_b200 import meshgen


def _setup(formulation):
    bar = meshgen.cantilever_bar(nx=6, ny=2, nz=2)
    m = O.Mesh(bar.X, bar.conn)
    mat = O.Material("linear_elastic", E=1000.0, nu=0.3)
    d = DynamicOracle(m, mat, 1000.0, 0.3, bar.fixed_mask, density=1e-3, formulation=formulation)
    rng = np.random.default_rng(3)
    d.v = rng.standard_normal(d.v.shape) * 0.1
    d.v[~d.free] = 0.0
    return bar, m, d


def test_lumped_mass_is_the_body_mass():
    bar, m, d = _setup("consistent")
    assert abs(d.M.sum() / 3.0 - 1e-3 * m.vol.sum()) <= 1e-12 * d.M.sum()


def test_consistent_newmark_conserves_energy():
    bar, m, d = _setup("consistent")
    e0 = d.energy()
    for _ in range(50):
        d.step(np.zeros(d.u.size))
    assert abs(d.energy() - e0) <= 1e-9 * e0


def test_reference_newmark_as_written_does_not():
    bar, m, d = _setup("reference")
    e0 = d.energy()
    for _ in range(50):
        d.step(np.zeros(d.u.size))
    assert abs(d.energy() - e0) > 1e-3 * e0
