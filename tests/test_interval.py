"""Confidence / prediction intervals (reference confidence.py:60-216): the
asymptotic variance constant from the kernel moment matrices, the interval
formula on the reference's own grid arrays, and (GPU) the whole chain."""
import numpy as np
import pytest

import os

from conftest import GOLDEN, load_golden, rel_err
from fastlpr_b200 import fastlpr_interval
from fastlpr_b200.confidence import asymptotic_nu
from fastlpr_b200.structures import RegressionOutput


class _Grid:
    def __init__(self, values):
        self.values = values


def test_nu_closed_forms():
    assert np.isclose(asymptotic_nu(1, 0), 1 / (2 * np.sqrt(np.pi)), rtol=1e-14)
    assert np.isclose(asymptotic_nu(1, 1), 1 / (2 * np.sqrt(np.pi)), rtol=1e-14)
    assert np.isclose(asymptotic_nu(1, 2), 27 / (32 * np.sqrt(np.pi)), rtol=1e-14)
    assert np.isclose(asymptotic_nu(2, 1), 1 / (4 * np.pi), rtol=1e-14)
    assert np.isclose(asymptotic_nu(3, 0), 1 / (8 * np.pi ** 1.5), rtol=1e-14)
    # order 2 in d dims: (1 + d/2)^2 ... closed form through the moment matrices
    assert asymptotic_nu(2, 2) > asymptotic_nu(2, 1)


def test_interval_formula_matches_reference_on_its_grids():
    g = load_golden(os.path.join(GOLDEN, "interval1d.npz"))
    mu = RegressionOutput(yhat=g["mu_values"], grid=(np.zeros(1),), h=g["mu_h"],
                          fpp_yhat=_Grid(g["mu_values"]), metadata={"order": 1}, s0=g["s0"])
    var = RegressionOutput(yhat=g["var_values"], grid=(np.zeros(1),), h=g["var_h"],
                           fpp_yhat=_Grid(g["var_values"]), metadata={"order": 1})
    ci = fastlpr_interval(mu, var, 0.05, type="confidence")
    pi = fastlpr_interval(mu, var, 0.1, type="prediction")
    assert ci.shape == g["ci"].shape
    # the reference tabulates nu to 12 digits (4e-13 relative from the exact value)
    assert rel_err(ci, g["ci"]) < 1e-11
    assert rel_err(pi, g["pi"]) < 1e-11


def test_interval_argument_errors():
    mu = RegressionOutput(yhat=np.zeros(4), grid=(np.zeros(4),), h=np.array([0.1]),
                          fpp_yhat=_Grid(np.zeros(4)), metadata={"order": 1}, s0=np.ones(4))
    with pytest.raises(ValueError, match="alpha"):
        fastlpr_interval(mu, 1.0, alpha=1.5)
    with pytest.raises(ValueError, match="type"):
        fastlpr_interval(mu, 1.0, type="band")
    with pytest.raises(ValueError, match="Shape mismatch"):
        fastlpr_interval(mu, np.ones(3))


@pytest.mark.gpu
def test_interval_chain_matches_reference(cuda_ok):
    import fastlpr_b200
    g = load_golden(os.path.join(GOLDEN, "interval1d.npz"))
    x, y, h = g["x"], g["y"], g["h"]
    mu = fastlpr_b200.cv_fastlpr(x, y, h, {"order": 1, "N": 256, "precision": "fp64"})
    res = (y - mu.yhat) ** 2
    var = fastlpr_b200.cv_fastlpr(x, res, h, {"order": 1, "N": 256, "y_type_out": "variance",
                                              "dstd": 10, "precision": "fp64"})
    assert np.allclose(mu.h, g["mu_h"]) and np.allclose(var.h, g["var_h"])
    ci = fastlpr_interval(mu, var, 0.05, type="confidence")
    pi = fastlpr_interval(mu, var, 0.1, type="prediction")
    assert rel_err(ci, g["ci"]) < 1e-9
    assert rel_err(pi, g["pi"]) < 1e-9
    # prediction at new points goes through the GPU interpolant
    xq = np.linspace(0.05, 0.95, 7)[:, None]
    yq = fastlpr_b200.fastlpr_predict(mu, xq)
    assert yq.shape == (7,)
    assert np.max(np.abs(yq - np.sin(2 * np.pi * xq[:, 0]))) < 0.1
