"""Pointwise confidence and prediction intervals (reference confidence.py:60-216).

    ci = fastlpr_interval(regs_mu, regs_var, alpha=0.05, type="confidence")

On the native grid of the mean fit: se^2 = sigma^2 nu / (prod(h) s_0) with
s_0 the zero-order kernel moment plane of the selected bandwidth
(``RegressionOutput.s0``), and

    confidence:  m_hat +/- z se
    prediction:  m_hat +/- z sqrt(sigma^2 + se^2),

z = Phi^{-1}(1 - alpha/2).  nu(d, l) = e1' M_K^{-1} M_{K^2} M_K^{-1} e1 is the
asymptotic variance constant of the local polynomial estimator of order l
with the product Gaussian kernel, where M_K and M_{K^2} are the moment
matrices int K(u) X(u) X(u)' du and int K(u)^2 X(u) X(u)' du over the
monomials X(u) of total degree <= l.  It is computed here from the Gaussian
moments (E u^{2k} = (2k-1)!! under N(0, 1); K^2 = c N(0, 1/2) per axis with
c = 1 / (2 sqrt(pi))).
"""
from __future__ import annotations

import itertools
from functools import lru_cache
from typing import Union

import numpy as np
from scipy.stats import norm

from .structures import RegressionOutput


def _monomials(d: int, order: int):
    return [e for tot in range(order + 1)
            for e in itertools.product(range(tot + 1), repeat=d) if sum(e) == tot]


def _gauss_moment(k: int, var: float) -> float:
    """E[u^k] for u ~ N(0, var)."""
    if k % 2:
        return 0.0
    return float(np.prod(np.arange(k - 1, 0, -2))) * var ** (k // 2) if k else 1.0


@lru_cache(maxsize=None)
def asymptotic_nu(d: int, order: int) -> float:
    """nu(d, l) of the product Gaussian kernel (see the module docstring)."""
    if d < 1 or order < 0:
        raise ValueError(f"nu needs d >= 1 and order >= 0, got d={d}, order={order}")
    mon = _monomials(d, order)
    c = 1.0 / (2.0 * np.sqrt(np.pi))
    MK = np.empty((len(mon), len(mon)))
    MK2 = np.empty_like(MK)
    for i, a in enumerate(mon):
        for j, b in enumerate(mon):
            p = [ai + bi for ai, bi in zip(a, b)]
            MK[i, j] = np.prod([_gauss_moment(k, 1.0) for k in p])
            MK2[i, j] = c ** d * np.prod([_gauss_moment(k, 0.5) for k in p])
    v = np.linalg.solve(MK, np.eye(len(mon))[:, 0])
    return float(v @ MK2 @ v)


def _grid_values(r: RegressionOutput) -> np.ndarray:
    f = r.fpp_yhat
    if f is not None and hasattr(f, "values"):
        return np.asarray(f.values)
    return np.asarray(r.yhat)


def fastlpr_interval(mu: RegressionOutput, sigma: Union[RegressionOutput, float, np.ndarray],
                     alpha: float = 0.05, type: str = "confidence") -> np.ndarray:
    """Interval bounds on the mean fit's grid, shape grid + (2,): [..., 0] the
    upper and [..., 1] the lower bound (reference confidence.py:60-216)."""
    if not isinstance(mu, RegressionOutput):
        raise TypeError("mu must be a RegressionOutput object from cv_fastlpr")
    if mu.yhat is None:
        raise ValueError("mu must have .yhat field (fitted values)")
    if not isinstance(sigma, (RegressionOutput, float, int, np.ndarray)):
        raise TypeError("sigma must be RegressionOutput, float, or ndarray")
    if isinstance(sigma, RegressionOutput) and sigma.yhat is None:
        raise ValueError("sigma must have .yhat field (fitted values)")
    if not (0 < alpha < 1):
        raise ValueError(f"alpha must be in (0, 1), got {alpha}")
    kind = type.lower()
    if kind not in ("confidence", "prediction"):
        raise ValueError(f"type must be 'confidence' or 'prediction', got '{type}'")
    if mu.s0 is None:
        raise ValueError("mu.s0 is None: the RegressionOutput must carry s_0 "
                         "(zero-th kernel moment)")
    z = norm.ppf(1 - alpha / 2)
    mu_values = _grid_values(mu)
    sig = _grid_values(sigma) if isinstance(sigma, RegressionOutput) else np.asarray(sigma)
    sig = np.maximum(sig, 0)
    s0 = np.maximum(np.asarray(mu.s0), 1e-10)
    if sig.shape != s0.shape:
        raise ValueError(f"Shape mismatch: sigma has shape {sig.shape} but s0 has shape "
                         f"{s0.shape}. Ensure mu and sigma use the same grid.")
    if mu_values.shape != s0.shape:
        raise ValueError(f"Shape mismatch: mu has shape {mu_values.shape} but s0 has shape "
                         f"{s0.shape}. Ensure mu grid values and s0 are aligned.")
    d = len(mu.grid)
    order = int(mu.metadata["order"]) if mu.metadata else 0
    prod_h = float(np.prod(np.atleast_1d(mu.h).astype(float)))
    se_sq = sig * asymptotic_nu(d, order) / (prod_h * s0)
    half = z * np.sqrt(se_sq) if kind == "confidence" else z * np.sqrt(sig + se_sq)
    return np.stack([mu_values + half, mu_values - half], axis=-1)
