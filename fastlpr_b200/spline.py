"""Host side of the not-a-knot cubic spline interpolation (the reference's
'cubic' GCV / DoF / output interpolation: scipy
``RegularGridInterpolator(method='cubic')``, api.py:594-600, api.py:651-657,
regression.py:1015-1020).

Per axis the knots are ``[x0]*4 + x[2:-2] + [x_end]*4``; the collocation
matrix A[i, k] = B_k(x_i) is banded (three diagonals either side at most).
It is factored here, A = L U without pivoting (B-spline collocation matrices
are totally positive, so elimination without pivoting is stable), into the
7-column row table that ``flpr_spline_prefilter`` consumes; the device solves
every grid line with it.  Basis values: Cox-de Boor recursion in the
triangular form of Piegl and Tiller, The NURBS Book, algorithm A2.2.
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

METHODS = ("linear", "cubic")


def _knots(axis: np.ndarray) -> np.ndarray:
    return np.concatenate([np.repeat(axis[0], 4), axis[2:-2], np.repeat(axis[-1], 4)])


def _basis_at_nodes(axis: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Span index l (t[l] <= x < t[l+1], clamped to [3, G-1]) and the values
    of B_{l-3..l} at every grid node."""
    t = _knots(axis)
    G = axis.size
    l = np.clip(np.searchsorted(t, axis, side="right") - 1, 3, G - 1)
    N = np.zeros((G, 4))
    N[:, 0] = 1.0
    left = np.zeros((G, 4))
    right = np.zeros((G, 4))
    for j in range(1, 4):
        left[:, j] = axis - t[l + 1 - j]
        right[:, j] = t[l + j] - axis
        saved = np.zeros(G)
        for r in range(j):
            tmp = N[:, r] / (right[:, r + 1] + left[:, j - r])
            N[:, r] = saved + right[:, r + 1] * tmp
            saved = left[:, j - r] * tmp
        N[:, j] = saved
    return l, N


def band_lu(axis: np.ndarray) -> np.ndarray:
    """(G, 7) rows [l3, l2, l1, 1/u0, u1, u2, u3] of the LU factors of the
    axis' collocation matrix (L unit lower, U upper, both within the band)."""
    axis = np.asarray(axis, dtype=np.float64)
    G = axis.size
    if G < 4:
        raise ValueError(f"There are {G} points in a dimension, but cubic interpolation "
                         "requires at least 4 points per dimension.")
    if not np.all(np.diff(axis) > 0):
        raise ValueError("cubic interpolation needs strictly ascending grid axes")
    l, N = _basis_at_nodes(axis)
    B = np.zeros((G, 7))                       # B[i, 3 + k - i] = A[i, k]
    rows = np.arange(G)
    for j in range(4):
        off = l - 3 + j - rows
        B[rows, 3 + off] = N[:, j]
    for k in range(G):
        piv = B[k, 3]
        for i in range(k + 1, min(k + 4, G)):
            lik = B[i, 3 + k - i] / piv
            B[i, 3 + k - i] = lik
            if lik != 0.0:
                for j in range(k + 1, min(k + 4, G)):
                    B[i, 3 + j - i] -= lik * B[k, 3 + j - k]
    out = B.copy()
    out[:, 3] = 1.0 / B[:, 3]
    # entries outside the matrix stay zero
    for i in range(G):
        for c in range(7):
            if not 0 <= i + c - 3 < G:
                out[i, c] = 0.0
    return out


class SplineTables:
    """Device copies of the concatenated raw axes and LU tables of one grid."""

    def __init__(self, axes: Sequence[np.ndarray], device: torch.device):
        axes = [np.asarray(a, dtype=np.float64).ravel() for a in axes]
        self.G = [a.size for a in axes]
        lu = np.concatenate([band_lu(a).ravel() for a in axes])
        self.axes = torch.from_numpy(np.concatenate(axes)).to(device)
        self.lu = torch.from_numpy(lu).to(device)


_CACHE: Dict[Tuple, SplineTables] = {}


def tables(axes: Sequence[np.ndarray], device: torch.device) -> SplineTables:
    key = (str(device),) + tuple(np.asarray(a, dtype=np.float64).tobytes() for a in axes)
    t = _CACHE.get(key)
    if t is None:
        if len(_CACHE) > 64:
            _CACHE.clear()
        t = _CACHE[key] = SplineTables(axes, device)
    return t


def check_method(key: str, method) -> str:
    m = str(method)
    if m not in METHODS:
        raise NotImplementedError(f"{key}={method!r}: only 'linear' and 'cubic' interpolation "
                                  "are implemented")
    return m


def axes_list(axes) -> List[np.ndarray]:
    return [np.asarray(a, dtype=np.float64).ravel() for a in axes]
