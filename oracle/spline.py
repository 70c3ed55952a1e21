"""Not-a-knot tensor-product cubic spline interpolation -- TEST INFRASTRUCTURE ONLY.

The reference's 'cubic' GCV/DoF interpolation (api.py:594-600,
api.py:651-657, regression.py:1015-1020) is scipy's
``RegularGridInterpolator(method='cubic', fill_value=None)``; with scipy
1.18.1 (the version the golden fixtures were made with) that builds
``make_ndbspl``: per axis the not-a-knot knot vector
``t = [x0]*4 + x[2:-2] + [x_end]*4``, the tensor-product collocation system
``A coef = values`` and ``NdBSpline`` evaluation (the end polynomial pieces
extend beyond the grid).  scipy solves that system iteratively
(``gcrotmk``, atol 1e-6, default rtol 1e-5), so the reference's values carry
that solver's residual; this restatement solves it exactly, axis by axis
(the tensor collocation matrix is the Kronecker product of the per-axis
ones).  Basis values follow the Cox-de Boor recursion in the triangular form
of Piegl and Tiller, The NURBS Book, algorithm A2.2.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

K = 3


def not_a_knot_knots(axis: np.ndarray) -> np.ndarray:
    axis = np.asarray(axis, dtype=float)
    if axis.size < K + 1:
        raise ValueError(f"cubic interpolation needs at least {K + 1} grid points per axis, "
                         f"got {axis.size}")
    return np.concatenate([[axis[0]] * (K + 1), axis[2:-2], [axis[-1]] * (K + 1)])


def span(t: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Knot span l with t[l] <= x < t[l+1], clamped to the first / last
    polynomial piece (l in [K, nc-1], nc = len(t) - K - 1)."""
    nc = len(t) - K - 1
    l = np.searchsorted(t, x, side="right") - 1
    return np.clip(l, K, nc - 1)


def basis(t: np.ndarray, l: np.ndarray, x: np.ndarray) -> np.ndarray:
    """(len(x), K+1) values of the B-splines l-K..l at x."""
    x = np.asarray(x, dtype=float)
    N = np.zeros((x.size, K + 1))
    N[:, 0] = 1.0
    left = np.zeros((x.size, K + 1))
    right = np.zeros((x.size, K + 1))
    for j in range(1, K + 1):
        left[:, j] = x - t[l + 1 - j]
        right[:, j] = t[l + j] - x
        saved = np.zeros(x.size)
        for r in range(j):
            temp = N[:, r] / (right[:, r + 1] + left[:, j - r])
            N[:, r] = saved + right[:, r + 1] * temp
            saved = left[:, j - r] * temp
        N[:, j] = saved
    return N


def collocation(axis: np.ndarray) -> np.ndarray:
    """Dense (G, G) matrix A[i, k] = B_k(axis[i])."""
    t = not_a_knot_knots(axis)
    G = len(axis)
    l = span(t, axis)
    b = basis(t, l, axis)
    A = np.zeros((G, G))
    for j in range(K + 1):
        A[np.arange(G), l - K + j] = b[:, j]
    return A


def coefficients(axes: Sequence[np.ndarray], values: np.ndarray) -> np.ndarray:
    """Spline coefficients of values (grid axes first, batch axes after)."""
    c = np.asarray(values)
    c = c.astype(np.complex128 if np.iscomplexobj(c) else np.float64)
    for a, ax in enumerate(axes):
        A = collocation(np.asarray(ax, dtype=float))
        c = np.moveaxis(np.tensordot(np.linalg.inv(A), np.moveaxis(c, a, 0), axes=(1, 0)), 0, a)
    return c


def evaluate(axes: Sequence[np.ndarray], coef: np.ndarray, pts: np.ndarray) -> np.ndarray:
    """Spline with coefficients coef at pts (n, d) -> (n, batch...)."""
    pts = np.atleast_2d(np.asarray(pts, dtype=float))
    d = len(axes)
    idx, w = [], []
    for a in range(d):
        t = not_a_knot_knots(axes[a])
        l = span(t, pts[:, a])
        idx.append(l - K)
        w.append(basis(t, l, pts[:, a]))
    out = np.zeros((pts.shape[0],) + coef.shape[d:], dtype=coef.dtype)
    for taps in np.ndindex(*([K + 1] * d)):
        wt = np.ones(pts.shape[0])
        sel = []
        for a in range(d):
            wt = wt * w[a][:, taps[a]]
            sel.append(idx[a] + taps[a])
        vals = coef[tuple(sel)]
        out += wt.reshape((-1,) + (1,) * (vals.ndim - 1)) * vals
    return out


def cubic_interp(axes: Sequence[np.ndarray], values: np.ndarray, pts: np.ndarray) -> np.ndarray:
    """Exact not-a-knot cubic interpolation of grid values at pts."""
    axes = [np.asarray(a, dtype=float) for a in axes]
    return evaluate(axes, coefficients(axes, values), pts)
