"""fastlpr_b200: fastLPR's NUFFT path (local polynomial regression with GCV,
kernel density estimation with LCV) on NVIDIA B200 GPUs.

Public API mirrors the reference package ``fastlpr``:

    from fastlpr_b200 import cv_fastlpr, cv_fastkde, get_hlist
    regs = cv_fastlpr(x, y, get_hlist(20, [0.01, 1.0]), {"order": 1})

The hot path runs in the in-tree CUDA library ``libfastlpr_b200.so``
(C ABI: include/fastlpr_b200.h); there is no CPU fallback.
"""
from .bandwidth import get_hlist
from .structures import KDEOutput, RegressionOutput
from .api import cv_fastkde, cv_fastlpr, cv_fastlpr_device, clear_fastlpr_caches
from .confidence import fastlpr_interval
from .batch import (SharedData, batch_evaluate_at_points, compute_gcv_scores_batch,
                    cv_fastlpr_batch, precompute_shared)
from .plan import LprPlan, cv_fastlpr_many

import numpy as np

__version__ = "0.1.0"


def fastlpr_predict(regression: RegressionOutput, x_new):
    """Evaluate a fitted regression at new points (reference predict.py:15-131):
    the fitted grid's interpolant, evaluated on the GPU."""
    if regression.fpp_yhat is None:
        raise ValueError("Regression output does not contain an interpolant (fpp).")
    points = np.asarray(x_new, dtype=float)
    if points.ndim == 1:
        points = points[:, None]
    return np.asarray(regression.fpp_yhat(points))


__all__ = [
    "__version__",
    "cv_fastlpr",
    "cv_fastkde",
    "cv_fastlpr_device",
    "get_hlist",
    "fastlpr_predict",
    "fastlpr_interval",
    "SharedData",
    "precompute_shared",
    "cv_fastlpr_batch",
    "batch_evaluate_at_points",
    "compute_gcv_scores_batch",
    "LprPlan",
    "cv_fastlpr_many",
    "RegressionOutput",
    "KDEOutput",
    "clear_fastlpr_caches",
]
