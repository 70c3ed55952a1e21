import ast
import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_files(kind=None):
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        z = np.load(f)
        if kind is None or str(z["kind"]) == kind:
            out.append(f)
    return out


def load_golden(path):
    z = dict(np.load(path))
    z["kind"] = str(z["kind"])
    if "opts" in z:
        z["opts"] = ast.literal_eval(str(z["opts"]))
    return z


def _both_nan(a, b):
    return np.isnan(a) & np.isnan(b)


def rel_err(a, b):
    """max |a - b| / max |b| (0 when both are empty); entries that are NaN
    in both (scores of a fit without DoF) count as equal."""
    a = np.asarray(a)
    b = np.asarray(b)
    if b.size == 0:
        return 0.0
    same = _both_nan(a, b) if np.issubdtype(b.dtype, np.inexact) else np.zeros(b.shape, bool)
    if np.all(same):
        return 0.0
    den = np.max(np.abs(b[~same]))
    return float(np.max(np.abs(a - b)[~same]) / (den if den > 0 else 1.0))


def elem_rel_err(a, b):
    a = np.asarray(a, dtype=complex)
    b = np.asarray(b, dtype=complex)
    same = _both_nan(a, b)
    if np.all(same):
        return 0.0
    return float(np.max((np.abs(a - b) / np.maximum(np.abs(b), 1e-300))[~same]))


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
