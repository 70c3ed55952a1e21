"""Bandwidth candidate grids (reference bandwidth.py:22-137)."""
from __future__ import annotations

from typing import Callable, Sequence, Union

import numpy as np


def get_hlist(
    n: Union[Sequence[int], int],
    range: np.ndarray,  # noqa: A002 -- reference argument name
    spacing: Callable[[float, float, int], np.ndarray] | None = None,
) -> np.ndarray:
    """Bandwidth candidates, shape (prod(n), dims).

    Per axis ``spacing(lo, hi, n)`` (default logarithmic), then the Cartesian
    product with the first axis varying fastest (MATLAB ``ndgrid`` order,
    bandwidth.py:126-136).  Raises ValueError when ``n`` and ``range`` disagree
    on the number of dimensions.
    """
    r = np.asarray(range, dtype=float)
    if r.ndim == 1:
        r = r.reshape(1, 2)
    dims = r.shape[0]
    n_list = [int(n)] * dims if np.isscalar(n) else [int(v) for v in n]
    if len(n_list) != dims:
        raise ValueError("n must match the number of rows in range.")
    if spacing is None:
        def spacing(lo, hi, num):
            return np.logspace(np.log10(lo), np.log10(hi), num)
    axes = [spacing(lo, hi, num) if num > 1 else np.array([lo], dtype=float)
            for (lo, hi), num in zip(r, n_list)]
    mesh = np.meshgrid(*axes, indexing="ij")
    return np.column_stack([m.ravel("F") for m in mesh])
