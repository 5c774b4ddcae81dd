"""simul_b200 — B200-native TET4 FEM static-solve path (drop-in for backend/fea/fem).

The solver, kernels and C ABI live in ``libfemb200.so`` (``simul_b200/csrc``,
declared in ``include/femb200.h``); this package is the Python host side that
mirrors the reference's ``FEMesh`` / material / ``StaticSolver`` API.
"""
from .fem import (B200StaticSolver, ElementType, FEMesh, FibreReinforcedMooneyRivlin, J2Plasticity,
                  LinearElastic, MaterialBase, MooneyRivlin, NeoHookean, StaticSolver,
                  TransverseIsotropic)
from .validation import FEAConvergenceError, FEAValidationError

__all__ = ["B200StaticSolver", "ElementType", "FEMesh", "FibreReinforcedMooneyRivlin", "J2Plasticity",
           "LinearElastic", "MaterialBase", "MooneyRivlin", "NeoHookean", "StaticSolver",
           "TransverseIsotropic", "FEAConvergenceError", "FEAValidationError"]
