"""Output structures of ``cv_fastlpr`` and ``cv_fastkde``.

Same fields as the reference dataclasses (structures.py:23-71), so code
written against the reference reads the results unchanged.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np


@dataclass
class RegressionOutput:
    """Result of :func:`cv_fastlpr`: fitted values, grid, selected bandwidth,
    GCV curve (``gcv_yhat``), interpolant ``fpp_yhat`` and metadata."""

    yhat: np.ndarray
    grid: tuple
    h: np.ndarray
    gcv_yhat: Optional[Dict[str, object]] = None
    fpp_yhat: Optional[object] = None
    metadata: Optional[Dict[str, object]] = None
    dof: Optional[float] = None
    dof_stderr: Optional[float] = None
    d: Optional[float] = None
    s0: Optional[np.ndarray] = None


@dataclass
class KDEOutput:
    """Result of :func:`cv_fastkde`: density on the grid, selected bandwidth,
    LCV curve (``lcv``), interpolant ``fpp`` and metadata."""

    fhat: np.ndarray
    grid: tuple
    h: np.ndarray
    lcv: Optional[Dict[str, object]] = None
    fpp: Optional[object] = None
    metadata: Optional[Dict[str, object]] = None
