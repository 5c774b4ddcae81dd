"""Error types and input checks mirroring ``backend/fea/fem/validation.py``.

``FEAValidationError`` (validation.py:18-41) and ``FEAConvergenceError``
(validation.py:43-66) keep the reference's constructor arguments and message
prefixes so callers that catch them keep working.
"""
from __future__ import annotations

import logging

logger = logging.getLogger("fea.fem")


class FEAValidationError(ValueError):
    """Invalid FEA input (validation.py:18-41)."""

    def __init__(self, message: str, parameter: str = "", value=None, suggestion: str = ""):
        self.parameter = parameter
        self.value = value
        self.suggestion = suggestion
        full = f"[FEA 검증 오류] {message}"
        if suggestion:
            full += f" → 제안: {suggestion}"
        super().__init__(full)


class FEAConvergenceError(RuntimeError):
    """Solver failure (validation.py:43-66); ``reason="nan_divergence"`` for NaN/Inf."""

    def __init__(self, message: str, iterations: int = 0, residual: float = 0.0, reason: str = ""):
        self.iterations = iterations
        self.residual = residual
        self.reason = reason
        super().__init__(f"[FEA 수렴 실패] {message}")


def validate_elastic_constants(E, nu, name="재료"):
    """E > 0 and -1 < nu < 0.5 (validation.py:71-98)."""
    import numpy as np
    Ea = np.asarray(E, dtype=np.float64)
    if Ea.size == 0 or np.any(~np.isfinite(Ea)) or np.any(Ea <= 0):
        raise FEAValidationError(f"{name}의 영 계수(E)가 {E}입니다. 양수여야 합니다.",
                                 parameter="E", value=E)
    if nu < -1.0 or nu >= 0.5:
        raise FEAValidationError(f"{name}의 푸아송 비(ν)가 {nu}입니다. -1.0 < ν < 0.5 범위여야 합니다.",
                                 parameter="nu", value=nu)


def validate_positive(value, parameter, name="재료", allow_zero=False):
    import numpy as np
    v = np.asarray(value, dtype=np.float64)
    bad = np.any(v < 0) if allow_zero else np.any(v <= 0)
    if v.size == 0 or np.any(~np.isfinite(v)) or bad:
        cmp = "0 이상" if allow_zero else "양수"
        raise FEAValidationError(f"{name}의 {parameter}가 {value}입니다. {cmp}여야 합니다.",
                                 parameter=parameter, value=value)


def validate_bc_indices(node_ids, n_nodes, label="경계조건"):
    """Node indices inside [0, n_nodes) (validation.py:188-216)."""
    import numpy as np
    ids = np.asarray(node_ids)
    if ids.size == 0:
        return
    if ids.min() < 0 or ids.max() >= n_nodes:
        raise FEAValidationError(
            f"{label} 노드 인덱스가 범위를 벗어났습니다 (0 ~ {n_nodes - 1}).",
            parameter="node_ids", value=(int(ids.min()), int(ids.max())))
