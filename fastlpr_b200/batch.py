"""Shared-data batch API (reference batch.py:49-760).

    shared = precompute_shared(x, y, h, {"order": 1})
    regs = cv_fastlpr_batch(shared)                      # all bandwidths, GCV selection
    vals = batch_evaluate_at_points(shared, x_new, [0, 3])

``precompute_shared`` does the bandwidth-independent work once and keeps it
on the GPU: upload, point statistics, Hutchinson probes, spread and forward
FFT of every channel, adjoint deposits.  ``cv_fastlpr_batch`` and
``batch_evaluate_at_points`` then run the per-bandwidth work (kernel
spectra, convolutions, solves, GCV) on those spectra.  The reference keeps
the full (L^d, H) kernel table (``kd_ft``) and the design planes (``S``)
between calls; here the per-axis kernel factors are rebuilt on the device
for each call instead (they cost far less than storing them), so those two
fields are None.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import _lib
from .api import (_Ctx, _PhaseEvents, _as_column_matrix, _check_interp_methods,
                  _check_supported, _default_hrange, _device, _evaluate_lpr, _filter_bandwidths,
                  _finalize_lpr, _precision, _prepare_bandwidths, _prepare_lpr, set_defaults)
from .interpolant import GridInterpolant
from .structures import RegressionOutput


@dataclass
class SharedData:
    """Precomputed, bandwidth-independent state of one data set (reference
    batch.py:49-107).  The device-resident part lives in private fields."""

    x_raw: np.ndarray
    y_raw: np.ndarray
    mean: np.ndarray
    std: np.ndarray
    grid_axes_raw: List[np.ndarray]
    grid_axes_scaled: List[np.ndarray]
    kdf_params: dict
    bandwidths_filtered: np.ndarray
    grid_shape: np.ndarray
    options: dict
    kd_ft: Optional[Union[np.ndarray, list]] = None
    S: Optional[Union[np.ndarray, list]] = None
    S_params: Optional[dict] = None
    y_raw_original: Optional[np.ndarray] = None
    _ctx: object = field(default=None, repr=False)
    _state: object = field(default=None, repr=False)
    _bandwidths: Optional[np.ndarray] = field(default=None, repr=False)

    @property
    def x_scaled(self) -> np.ndarray:
        """z-scored, mid-range-centred predictors (model.py:58-68)."""
        g = self._state.geom
        return (self.x_raw - g.mean) / g.std - g.center


def precompute_shared(x, y, h=None, options: Optional[dict] = None,
                      compute_design_matrix_for_dof: bool = True) -> SharedData:
    """Bandwidth-independent work of a fit, kept on the GPU (reference
    batch.py:139-284).  ``compute_design_matrix_for_dof`` is accepted for
    compatibility; the design planes are formed per call on the device."""
    x_arr = _as_column_matrix(x)
    y_arr = np.asarray(y)
    if y_arr.ndim == 1:
        y_arr = y_arr[:, None]
    elif y_arr.ndim == 2:
        if y_arr.shape[0] == 1 and y_arr.shape[1] > 1:
            y_arr = y_arr.T
    else:
        raise ValueError(f"Response y must be 1D or 2D array. Got {y_arr.ndim}D.")
    if y_arr.shape[0] != x_arr.shape[0]:
        raise ValueError(
            f"Response y must have same number of samples as x. x has {x_arr.shape[0]} samples, "
            f"y has {y_arr.shape[0]} samples.")
    opts = set_defaults(options, order=0, regularization=1e-8, num_dof_sample=10,
                        kernel_type="gaussian", y_type_out="mean", calc_dof=True,
                        gcv_selection="first")
    n, dims = x_arr.shape
    if n < 2:
        raise ValueError("Input x must have at least two samples.")
    if opts.get("accuracy") is None:
        opts["accuracy"] = max(6 - int(np.ceil(np.log10(n))), 4)
    order = int(opts["order"])
    if order not in (0, 1, 2):
        raise ValueError("Polynomial order must be 0, 1, or 2.")
    bandwidths = _prepare_bandwidths(h, dims, opts, lambda: _default_hrange(x_arr))
    _check_supported(dims, opts)
    variance = str(opts.get("y_type_out", "mean")) == "variance"
    y_is_complex = bool(np.iscomplexobj(y_arr))
    if variance and y_is_complex:
        raise NotImplementedError("variance mode needs a real response")
    _check_interp_methods(opts, dims, n)
    prec = _precision(opts)
    ctx = _Ctx(_device(opts))
    with torch.cuda.device(ctx.device):
        st = _prepare_lpr(ctx, x_arr, y_arr, y_arr.shape[1], opts, order, prec, variance,
                          y_is_complex, None, _PhaseEvents(None), bandwidths=bandwidths)
        _, bw, keep, _ = _filter_bandwidths(ctx, st.geom, bandwidths, 2 * order + 1, st.kid)
    g = st.geom
    axes_scaled = [np.linspace(g.lo[a], g.hi[a], int(g.G[a])) for a in range(dims)]
    return SharedData(
        x_raw=x_arr, y_raw=y_arr if not variance else np.log(y_arr + 1.0 / n),
        mean=g.mean, std=g.std, grid_axes_raw=list(st.axes_raw), grid_axes_scaled=axes_scaled,
        kdf_params={"L": g.L.copy(), "qin": g.qin.copy(), "qout": g.qout.copy(),
                    "dh": int(len(keep)), "msp": g.msp, "tau": g.tau.copy()},
        bandwidths_filtered=bw[keep], grid_shape=g.G.copy(), options=opts,
        y_raw_original=y_arr if variance else None,
        _ctx=ctx, _state=st, _bandwidths=bandwidths)


def _evaluate_all(shared: SharedData):
    ctx, st = shared._ctx, shared._state
    ev = _PhaseEvents(None)
    with torch.cuda.device(ctx.device):
        r = _evaluate_lpr(ctx, st, shared._bandwidths, ev)
    return r, ev


def _grids(shared: SharedData, r: dict) -> np.ndarray:
    """(H, G..., ny) host copy of the fitted grids of every bandwidth."""
    st = shared._state
    m = r["m"][:, :, :st.ny].cpu().numpy()
    gshape = tuple(int(g) for g in st.geom.G)
    if st.y_is_complex:
        m = m[..., 0::2] + 1j * m[..., 1::2]
    return m.reshape((m.shape[0],) + gshape + (m.shape[-1],))


def cv_fastlpr_batch(shared: SharedData, return_all_grid_values: bool = False) -> RegressionOutput:
    """GCV sweep over every bandwidth on the precomputed spectra (reference
    batch.py:287-592); same result as cv_fastlpr on the same inputs."""
    r, ev = _evaluate_all(shared)
    ctx, st = shared._ctx, shared._state
    with torch.cuda.device(ctx.device):
        out = _finalize_lpr(ctx, st, r, ev, None)
    if return_all_grid_values:
        grids = _grids(shared, r)
        out.metadata["all_grid_values"] = [g[..., 0] if g.shape[-1] == 1 else g for g in grids]
    return out


def _batch_method(shared: SharedData, key: str) -> str:
    """Interpolation of the batch helpers (batch.py:646-651, 718-720): the
    option `key`, else linear in 1-D and the cubic spline otherwise."""
    d = shared.x_raw.shape[1]
    return str(shared.options.get(key, "linear" if d == 1 else "cubic"))


def _rgi(shared: SharedData, values: np.ndarray, method: str) -> GridInterpolant:
    """scipy's RegularGridInterpolator(fill_value=None) on the GPU: the
    cubic spline with extended end pieces, or linear continuing the edge
    cells beyond the grid."""
    if method not in ("linear", "cubic"):
        raise NotImplementedError(f"interpolation method {method!r}: only 'linear' and 'cubic'")
    return GridInterpolant(shared.grid_axes_raw, values, shared._ctx.device, method=method,
                           extrapolate=True)


def batch_evaluate_at_points(shared: SharedData, eval_points,
                             bandwidth_indices: Optional[Sequence[int]] = None) -> np.ndarray:
    """Fitted surfaces of the chosen bandwidths at new points, (M, k) (or
    (M, k, dy)), interpolated on the GPU like the reference (batch.py:595-669:
    option 'interp_method', default linear in 1-D and cubic otherwise,
    continued beyond the grid)."""
    r, _ = _evaluate_all(shared)
    grids = _grids(shared, r)
    H = grids.shape[0]
    idx = list(range(H)) if bandwidth_indices is None else [int(i) for i in bandwidth_indices]
    if any(i < 0 or i >= H for i in idx):
        raise IndexError(f"bandwidth index out of range 0..{H - 1}")
    sel = np.moveaxis(grids[idx], 0, -2)               # G... x k x dy
    if sel.shape[-1] == 1:
        sel = sel[..., 0]
    interp = _rgi(shared, sel, _batch_method(shared, "interp_method"))
    return interp(np.atleast_2d(np.asarray(eval_points, dtype=float)))


def compute_gcv_scores_batch(shared: SharedData, m_all: np.ndarray, dof_all: np.ndarray,
                             dof_stderr_all: np.ndarray,
                             penalty_std_all: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """GCV score and standard error per bandwidth from given fitted grids and
    degrees of freedom (reference batch.py:672-760, regression.py:280-471):
    GCV = (RSS/N) / max(clip(1 - dof/N, 0, 1), 0.01)^2, stderr = (RSS/N) x
    penalty_std, columns aggregated by the ``gcv_selection`` option; fitted
    values interpolated with option 'gcv_interp_method' (default linear in
    1-D, cubic otherwise)."""
    m = np.asarray(m_all)
    gshape = tuple(int(g) for g in shared.grid_shape)
    H = len(np.atleast_1d(dof_all))
    if m.shape[:len(gshape)] != gshape:
        raise ValueError(f"m_all must start with the grid shape {gshape}, got {m.shape}")
    interp = _rgi(shared, m, _batch_method(shared, "gcv_interp_method"))
    yhat = interp(shared.x_raw)                        # (N, H) or (N, H, dy)
    y = np.asarray(shared.y_raw)
    N = y.shape[0]
    agg = str(shared.options.get("gcv_selection", "first"))
    scores, errs = np.empty(H), np.empty(H)
    for k in range(H):
        yh = yhat[:, k] if yhat.ndim == 2 else yhat[:, k, :]
        if yh.ndim == 1:
            yh = yh[:, None]
        mse = np.sum(np.abs(y - yh) ** 2, axis=0) / N
        pdof = float(np.clip(1.0 - float(np.atleast_1d(dof_all)[k]) / N, 0.0, 1.0))
        pen = 1.0 / max(pdof, 0.01) ** 2
        per_col = mse * pen
        if agg == "first":
            s, mse_a = per_col[0], mse[0]
        elif agg == "average":
            s, mse_a = np.mean(per_col), np.mean(mse)
        elif agg == "sum":
            s, mse_a = np.sum(per_col), np.sum(mse)
        else:
            raise ValueError(f"Unknown aggregation method: {agg}. Use 'first', 'average', or 'sum'.")
        ps = float(np.atleast_1d(penalty_std_all)[k])
        scores[k] = s
        errs[k] = mse_a * ps if ps > 0 else 0.0
    return scores, errs
