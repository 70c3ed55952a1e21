"""Grid interpolant returned as ``fpp_yhat`` / ``fpp``.

Mirrors the reference OptimizedInterpolator (interp_optimized.py:271-436),
evaluated on the GPU: method 'cubic' is the not-a-knot cubic spline of
scipy's RegularGridInterpolator (``flpr_spline_prefilter`` once, then
``flpr_spline_eval``; end pieces extended beyond the grid), every other
method the clamped multilinear interpolation (``flpr_interp_eval``), as in
the reference, where only 'cubic' leaves the linear path.  Same call
convention: points are ``np.atleast_2d``'d, so 1-D data is passed as an
(n, 1) array.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from . import _lib, spline


class GridInterpolant:
    """extrapolate=True continues the edge cells' linear functions beyond the
    grid instead of clamping (scipy's RegularGridInterpolator with
    fill_value=None, used by the reference's batch helpers); the spline
    always extends its end pieces."""

    def __init__(self, axes: Sequence[np.ndarray], values: np.ndarray, device: torch.device,
                 method: str = "linear", extrapolate: bool = False):
        self.grid_axes = tuple(np.asarray(a, dtype=float).ravel() for a in axes)
        self.ndim = len(self.grid_axes)
        self.values = np.ascontiguousarray(values)
        self.method = method
        self.is_complex = np.iscomplexobj(self.values)
        self.device = device
        self._G = [len(a) for a in self.grid_axes]
        self._M = int(np.prod(self._G))
        extra = self.values.shape[self.ndim:]
        self._extra = extra
        self._dvals = None  # device copy (spline coefficients if cubic), made at first use
        self._cubic = str(method) == "cubic"
        self._extrap = bool(extrapolate)
        self._spl = None
        ax = []
        for a in self.grid_axes:
            ax += [float(a[0]), float(a[1] - a[0]) if len(a) > 1 else 1.0]
        self._ax = ax
        self.bounds = [(a.min(), a.max()) for a in self.grid_axes]

    def __call__(self, points) -> np.ndarray:
        pts = np.atleast_2d(np.asarray(points, dtype=float))
        if pts.shape[1] != self.ndim:
            raise ValueError(f"points must have {self.ndim} columns, got {pts.shape[1]}")
        n = pts.shape[0]
        lib = _lib.load()
        with torch.cuda.device(self.device):
            if self._dvals is None:
                flat = self.values.reshape(self._M, -1)  # (M, nval)
                parts = [flat.real, flat.imag] if self.is_complex else [flat]
                stacked = np.concatenate([p.T for p in parts], axis=0).astype(np.float64)
                self._dvals = torch.from_numpy(np.ascontiguousarray(stacked)).to(self.device)
                if self._cubic:
                    self._spl = spline.tables(self.grid_axes, self.device)
                    stream = torch.cuda.current_stream(self.device).cuda_stream
                    _lib.check(lib.flpr_spline_prefilter(self.ndim, _lib.ivec(self._G),
                                                         self._dvals.shape[0], 1,
                                                         self._spl.lu.data_ptr(),
                                                         self._dvals.data_ptr(), stream),
                               "flpr_spline_prefilter")
            dx = torch.from_numpy(np.ascontiguousarray(pts)).to(self.device)
            nval = self._dvals.shape[0]
            out = torch.empty((nval, n), dtype=torch.float64, device=self.device)
            stream = torch.cuda.current_stream(self.device).cuda_stream
            if self._cubic:
                _lib.check(lib.flpr_spline_eval(self.ndim, n, dx.data_ptr(),
                                                self._spl.axes.data_ptr(), _lib.ivec(self._G),
                                                nval, self._dvals.data_ptr(), out.data_ptr(),
                                                stream), "flpr_spline_eval")
            else:
                fn = lib.flpr_interp_eval_extrap if self._extrap else lib.flpr_interp_eval
                _lib.check(fn(self.ndim, n, dx.data_ptr(), _lib.dvec(self._ax),
                              _lib.ivec(self._G), nval, self._dvals.data_ptr(), out.data_ptr(),
                              stream), "flpr_interp_eval")
            res = out.cpu().numpy()
        k = nval // 2 if self.is_complex else nval
        vals = res[:k] + 1j * res[k:] if self.is_complex else res
        vals = vals.T  # (n, nval)
        if not self._extra:
            return vals[:, 0]
        return vals.reshape((n,) + self._extra)
