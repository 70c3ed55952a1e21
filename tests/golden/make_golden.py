"""Generate golden fixtures by running the reference fastLPR Python package.

This script is the only committed file that executes the reference.  It
imports ``fastlpr`` from a read-only checkout of the reference (the
``fastLPR_py/src`` directory, given in the environment variable
``FASTLPR_REF_SRC``), runs
it on small seeded inputs and stores inputs and outputs as ``.npz`` files
next to this script.  The fixtures pin the CPU oracle (``oracle/``) and the
GPU path without needing the reference at test time.

Two patches are applied to the reference, both to its FP64 configuration:

* ``fastlpr.nufftn_type1.get_complex_dtype`` returns ``complex128`` so the
  whole chain (spreading grid, FFT, kernel multiply, solve) runs in FP64
  without changing the spreading width or Gaussian width
  (``py/nufftn_type1.py:550-557``, ``py/type_utils.py:158-168``).
* The 2-D order-2 closed form reads a data file that the package does not
  ship (``py/lwp_formulas.py:436-444``).  It is replaced by a batched
  ``numpy.linalg.solve`` of ``e1' (S + lambda I)^-1 T`` -- the definition the
  closed form implements (``py/lwp_formulas.py:12-14``).

Run:  FASTLPR_REF_SRC=<checkout>/fastLPR_py/src python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = os.environ.get("FASTLPR_REF_SRC")


def _import_reference():
    if not REF_SRC:
        raise SystemExit("set FASTLPR_REF_SRC to the reference's fastLPR_py/src directory")
    os.environ.setdefault("FASTLPR_QUIET", "1")
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")
    sys.path.insert(0, REF_SRC)
    import fastlpr  # noqa: F401
    import fastlpr.nufftn_type1 as nt
    import fastlpr.lwp_formulas as lf

    nt.get_complex_dtype = lambda acc: np.complex128

    def _solve_2d_order2(s, t):
        s_b, t_s = lf._prepare_broadcasting(s, t)
        nt_ = 6
        shape = np.broadcast_shapes(*[a.shape for a in s_b], *[a.shape for a in t_s])
        dtype = np.result_type(*s_b, *t_s)
        S = np.empty(shape + (nt_, nt_), dtype=np.result_type(*s_b))
        k = 0
        for j in range(nt_):
            for i in range(j, nt_):
                S[..., i, j] = np.broadcast_to(s_b[k], shape)
                S[..., j, i] = np.broadcast_to(s_b[k], shape)
                k += 1
        T = np.stack([np.broadcast_to(a, shape) for a in t_s], axis=-1).astype(dtype)
        beta = np.linalg.solve(S.astype(dtype), T[..., None])[..., 0]
        return beta[..., 0]

    lf._lwp_2d_order2_real = _solve_2d_order2
    return fastlpr


def _lpr_case(fastlpr, name, x, y, h, opts, extra=None):
    from fastlpr import cv_fastlpr

    fastlpr.clear_fastlpr_caches()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        r = cv_fastlpr(x, y, h, dict(opts))
    g = r.gcv_yhat
    out = dict(
        kind="lpr",
        x=x,
        y=y,
        h=np.asarray(h, dtype=float),
        opts=repr(opts),
        yhat=np.asarray(r.yhat),
        h_sel=np.asarray(r.h),
        grid_values=np.asarray(r.fpp_yhat.values),
        gcv_m=np.asarray(g["gcv_m"]),
        gcv_sd=np.asarray(g["gcv_sd"]),
        dof=np.asarray(g["dof"]),
        dof_stderr=np.asarray(g["dof_stderr"]),
        idmin=int(g["idmin"]),
        id1se=int(g["id1se"]),
        bandwidths=np.asarray(g["bandwidths"]),
        s0=np.asarray(r.s0),
        d_norm=np.nan if r.d is None else float(r.d),
        mean=np.asarray(r.metadata["mean"]),
        std=np.asarray(r.metadata["std"]),
    )
    for k, ax in enumerate(r.grid):
        out[f"axis{k}"] = np.asarray(ax)
    if extra:
        out.update(extra)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: N={x.shape[0]} d={x.shape[1]} H={len(h)} id1se={out['id1se']}")


def _kde_case(fastlpr, name, x, h, opts):
    from fastlpr import cv_fastkde

    fastlpr.clear_fastlpr_caches()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        k = cv_fastkde(x, h, dict(opts))
    out = dict(
        kind="kde",
        x=x,
        h=np.asarray(h, dtype=float),
        opts=repr(opts),
        fhat=np.asarray(k.fhat),
        fhat_all=np.asarray(k.metadata["fhat_all"]),
        h_sel=np.asarray(k.h),
        lcv_m=np.asarray(k.lcv["lcv_m"]),
        lcv_sd=np.asarray(k.lcv["lcv_sd"]),
        idmax=int(k.lcv["idmax"]),
        id1se=int(k.lcv["id1se"]),
    )
    for j, ax in enumerate(k.grid):
        out[f"axis{j}"] = np.asarray(ax)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: N={x.shape[0]} d={x.shape[1]} H={len(h)} id1se={out['id1se']}")


def _intermediates_case(fastlpr, name):
    """Spread spectra and design-matrix planes for a 2-D order-1 problem."""
    from fastlpr.model import create_regression_model
    from fastlpr.convolution import nufft_transform, compute_kernel_fourier
    from fastlpr.regression import compute_design_matrix

    rng = np.random.default_rng(11)
    n = 3000
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.1 * rng.standard_normal(n)
    hv = np.array([0.05, 0.1, 0.3])
    h = np.column_stack([hv, hv])
    G = np.array([32, 32])
    opts = {"order": 1, "N": [32, 32]}
    fastlpr.clear_fastlpr_caches()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        model = create_regression_model(x, y[:, None], h, opts)
        kd, prm = compute_kernel_fourier(model.x_scaled, h, G, order=1)
        spec_ones = nufft_transform(model.x_scaled, np.ones(n), prm["L"], eval_grid_shape=G,
                                    qin=prm["qin"], accuracy=4)
        spec_y = nufft_transform(model.x_scaled, y, prm["L"], eval_grid_shape=G,
                                 qin=prm["qin"], accuracy=4)
        S, _ = compute_design_matrix(model.x_scaled, h, G, order=1, accuracy=4)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        kind="intermediates",
        x=x, y=y, h=h, G=G,
        x_scaled=model.x_scaled,
        L=np.asarray(prm["L"]), qin=np.asarray(prm["qin"]), qout=np.asarray(prm["qout"]),
        kdf=np.stack([np.asarray(k) for k in kd], axis=0),
        spec_ones=spec_ones, spec_y=spec_y,
        S=np.stack([np.asarray(s) for s in S], axis=0),
    )
    print(f"{name}: intermediates L={prm['L']}")


def main():
    fastlpr = _import_reference()
    from fastlpr import get_hlist

    rng = np.random.default_rng(2024)

    # 1-D, orders 0/1/2, real response (tests/e2e/test_e2e_lpr_1d.py shapes).
    n = 3000
    x1 = rng.random((n, 1))
    y1 = np.sin(2 * np.pi * x1[:, 0]) + 0.1 * rng.standard_normal(n)
    h1 = get_hlist(8, [0.02, 0.8])
    for order in (0, 1, 2):
        _lpr_case(fastlpr, f"lpr1d_o{order}", x1, y1, h1, {"order": order, "N": 256})

    # 1-D with a bandwidth far below the grid spacing: exercises the
    # "too small" filter of py/convolution.py:542-566.
    h1b = np.vstack([[1e-4], h1])
    _lpr_case(fastlpr, "lpr1d_o1_badh", x1, y1, h1b, {"order": 1, "N": 128})

    # 1-D complex response (tests/e2e/test_e2e_complex.py).
    yc = np.exp(2j * np.pi * x1[:, 0]) + 0.1 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    _lpr_case(fastlpr, "lpr1d_o1_complex", x1, yc, h1, {"order": 1, "N": 256})

    # 1-D non-power-of-two padding and fewer probes.
    _lpr_case(fastlpr, "lpr1d_o1_nopow2", x1, y1, h1,
              {"order": 1, "N": 200, "flag_power2": False, "num_dof_sample": 4})

    # 2-D, orders 0/1/2 (N >= 5000 keeps the linear GCV/DoF interpolation).
    n2 = 6000
    x2 = rng.random((n2, 2))
    y2 = np.sin(2 * np.pi * x2[:, 0]) * np.cos(2 * np.pi * x2[:, 1]) + 0.1 * rng.standard_normal(n2)
    hv = np.logspace(np.log10(0.02), np.log10(0.5), 6)
    h2 = np.column_stack([hv, hv])
    for order in (0, 1, 2):
        _lpr_case(fastlpr, f"lpr2d_o{order}", x2, y2, h2, {"order": order, "N": [48, 40]})

    # 2-D anisotropic bandwidth grid from get_hlist (Fortran ordering).
    h2a = get_hlist([3, 2], [[0.05, 0.4], [0.08, 0.3]])
    _lpr_case(fastlpr, "lpr2d_o1_aniso", x2, y2, h2a, {"order": 1, "N": [32, 32]})

    # 2-D heteroscedastic variance fit (examples/example_hetero.py pattern).
    sig = 0.05 + 0.1 * x2[:, 0]
    y2h = np.sin(2 * np.pi * x2[:, 0]) * np.cos(2 * np.pi * x2[:, 1]) + sig * rng.standard_normal(n2)
    from fastlpr import cv_fastlpr
    fastlpr.clear_fastlpr_caches()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        r_mean = cv_fastlpr(x2, y2h, h2, {"order": 1, "N": [32, 32]})
    res2 = (y2h - r_mean.yhat) ** 2
    _lpr_case(fastlpr, "lpr2d_o1_variance", x2, res2, h2,
              {"order": 1, "N": [32, 32], "y_type_out": "variance"})

    # 3-D order 1.
    n3 = 6000
    x3 = rng.random((n3, 3))
    y3 = np.sin(2 * np.pi * x3[:, 0]) + x3[:, 1] * x3[:, 2] + 0.1 * rng.standard_normal(n3)
    hv3 = np.array([0.1, 0.2, 0.4])
    h3 = np.column_stack([hv3, hv3, hv3])
    _lpr_case(fastlpr, "lpr3d_o1", x3, y3, h3, {"order": 1, "N": [16, 16, 16]})

    # KDE 1-D / 2-D / 3-D.
    xk1 = np.concatenate([rng.normal(-1, 0.3, (1500, 1)), rng.normal(1.5, 0.6, (1500, 1))])
    _kde_case(fastlpr, "kde1d", xk1, get_hlist(10, [0.05, 1.0]), {"N": 256})
    xk2 = rng.standard_normal((4000, 2)) * np.array([1.0, 0.5])
    hk = np.logspace(np.log10(0.05), np.log10(0.8), 6)
    _kde_case(fastlpr, "kde2d", xk2, np.column_stack([hk, hk]), {"N": [40, 40]})
    xk3 = rng.standard_normal((5000, 3))
    hk3 = np.array([0.1, 0.2, 0.4, 0.8])
    _kde_case(fastlpr, "kde3d", xk3, np.column_stack([hk3, hk3, hk3]), {"N": [16, 16, 16]})

    _intermediates_case(fastlpr, "inter2d_o1")
    interval_case(fastlpr)
    accuracy3d_cases(fastlpr)
    extrapolation_cases(fastlpr)
    batch_cases(fastlpr)
    accuracy_cases(fastlpr)
    cubic_cases(fastlpr)
    kernel_cases(fastlpr)


def interval_case(fastlpr):
    """Mean fit, variance fit of the squared residuals and the reference's
    fastlpr_interval (confidence and prediction) on the mean's grid."""
    from fastlpr import cv_fastlpr, get_hlist
    from fastlpr.confidence import fastlpr_interval

    rng = np.random.default_rng(77)
    n = 4000
    x = rng.random((n, 1))
    sig = 0.05 + 0.2 * x[:, 0]
    y = np.sin(2 * np.pi * x[:, 0]) + sig * rng.standard_normal(n)
    h = get_hlist(10, [0.02, 0.6])
    fastlpr.clear_fastlpr_caches()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        mu = cv_fastlpr(x, y, h, {"order": 1, "N": 256})
        res = (y - mu.yhat) ** 2
        var = cv_fastlpr(x, res, h, {"order": 1, "N": 256, "y_type_out": "variance", "dstd": 10})
    ci = fastlpr_interval(mu, var, 0.05, type="confidence")
    pi = fastlpr_interval(mu, var, 0.1, type="prediction")
    np.savez_compressed(os.path.join(HERE, "interval1d.npz"), kind="interval", x=x, y=y,
                        h=np.asarray(h),
                        ci=np.asarray(ci), pi=np.asarray(pi), mu_h=np.asarray(mu.h),
                        var_h=np.asarray(var.h), mu_values=np.asarray(mu.fpp_yhat.values),
                        var_values=np.asarray(var.fpp_yhat.values), s0=np.asarray(mu.s0))
    print(f"interval1d: N={n} h_mu={np.asarray(mu.h).ravel()} h_var={np.asarray(var.h).ravel()}")


def accuracy_cases(fastlpr):
    """Non-default accuracies: 0 (nearest-bin binning, nufftn_type1.py:442-516)
    and >= 7 (oversampling ratio 2 / 3 with Gaussian deconvolution,
    nufftn_type1.py:693-770)."""
    from fastlpr import get_hlist

    rng = np.random.default_rng(99)
    n = 3000
    x1 = rng.random((n, 1))
    y1 = np.sin(2 * np.pi * x1[:, 0]) + 0.1 * rng.standard_normal(n)
    h1 = get_hlist(6, [0.03, 0.6])
    _lpr_case(fastlpr, "lpr1d_o1_acc0", x1, y1, h1, {"order": 1, "N": 256, "accuracy": 0})
    _lpr_case(fastlpr, "lpr1d_o1_acc12", x1, y1, h1, {"order": 1, "N": 128, "accuracy": 12})
    n2 = 6000  # 2-D with n >= 5000: the reference interpolates GCV/DoF linearly
    x2 = rng.random((n2, 2))
    y2 = np.sin(2 * np.pi * x2[:, 0]) * np.cos(2 * np.pi * x2[:, 1]) + 0.1 * rng.standard_normal(n2)
    hv = np.logspace(np.log10(0.05), np.log10(0.5), 4)
    h2 = np.column_stack([hv, hv])
    _lpr_case(fastlpr, "lpr2d_o1_acc7", x2, y2, h2, {"order": 1, "N": [32, 32], "accuracy": 7})
    xk = rng.standard_normal((3000, 2))
    _kde_case(fastlpr, "kde2d_acc7", xk, h2, {"N": [32, 32], "accuracy": 7})


def accuracy3d_cases(fastlpr):
    """Accuracy >= 7 in 3-D (oversampling ratio 2 / 3 with Gaussian
    deconvolution on a 3-D grid, nufftn_type1.py:693-770).  The reference's
    response grids come out about 1e3 times too large on this path; the
    fixtures pin that behaviour, which the oracle and the GPU reproduce."""
    rng = np.random.default_rng(97)
    n = 20000
    x = rng.random((n, 3)) * np.array([1.0, 2.0, 0.5])
    y = np.sin(3 * x[:, 0]) + x[:, 1] * x[:, 2] + 0.1 * rng.standard_normal(n)
    hv = np.array([0.3, 0.6, 1.2])
    h = np.column_stack([hv, hv, hv])
    _lpr_case(fastlpr, "lpr3d_o1_acc7", x, y, h, {"order": 1, "N": [16, 14, 12], "accuracy": 7})
    xk = rng.standard_normal((8000, 3))
    _kde_case(fastlpr, "kde3d_acc12", xk, h, {"N": [16, 14, 12], "accuracy": 12})


def extrapolation_cases(fastlpr):
    """opts['xrange'] narrower than the data, so that points lie beyond the
    grid.  With the DoF on, the reference raises here: its finite-difference
    extrapolation of the probe fits (regression.py:1074) cannot broadcast
    the (bandwidth, probe) axes ("operands could not be broadcast
    together").  Without the DoF it returns the fit at the first bandwidth,
    the fitted values from the clamped linear interpolant
    (interp_optimized.py:60-215); these fixtures pin that."""
    from fastlpr import get_hlist

    rng = np.random.default_rng(123)
    n = 3000
    x1 = rng.random((n, 1))
    y1 = np.sin(2 * np.pi * x1[:, 0]) + 0.1 * rng.standard_normal(n)
    _lpr_case(fastlpr, "lpr1d_o1_xrange", x1, y1, get_hlist(3, [0.05, 0.3]),
              {"order": 1, "N": 128, "xrange": [[0.1, 0.85]], "calc_dof": False})
    n2 = 6000
    x2 = rng.random((n2, 2))
    y2 = np.sin(2 * np.pi * x2[:, 0]) * np.cos(2 * np.pi * x2[:, 1]) + 0.1 * rng.standard_normal(n2)
    hv = np.array([0.1, 0.2])
    _lpr_case(fastlpr, "lpr2d_o1_xrange", x2, y2, np.column_stack([hv, hv]),
              {"order": 1, "N": [40, 36], "xrange": [[0.1, 0.9], [0.05, 0.8]],
               "calc_dof": False})


def batch_cases(fastlpr):
    """Shared-data batch API (batch.py:139-760): the fields of
    precompute_shared, batch_evaluate_at_points at points inside and beyond
    the grid (RegularGridInterpolator, linear in 1-D and cubic otherwise,
    fill_value=None) and compute_gcv_scores_batch on given fitted grids and
    DoF.  (cv_fastlpr_batch itself stops at batch.py:417, unpacking three
    values from a four-value return.)"""
    from fastlpr import get_hlist
    from fastlpr.batch import (batch_evaluate_at_points, compute_gcv_scores_batch,
                               precompute_shared)

    rng = np.random.default_rng(321)
    for d, n, G, name in ((1, 2000, 128, "batch1d"), (2, 3000, [40, 36], "batch2d")):
        fastlpr.clear_fastlpr_caches()
        x = rng.random((n, d))
        y = np.sin(2 * np.pi * x[:, 0]) * (np.cos(np.pi * x[:, -1]) if d == 2 else 1.0)
        y = y + 0.1 * rng.standard_normal(n)
        hv = np.logspace(np.log10(0.06), np.log10(0.5), 5)
        h = np.column_stack([hv] * d)
        opts = {"order": 1, "N": G}
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            sh = precompute_shared(x, y, h, dict(opts))
            pts = np.vstack([rng.random((40, d)), rng.uniform(-0.2, 1.2, (20, d))])
            ev = batch_evaluate_at_points(sh, pts, [0, 2, 4])
            gshape = tuple(int(g) for g in sh.grid_shape)
            axes = np.meshgrid(*sh.grid_axes_raw, indexing="ij")
            m_all = np.stack([np.sin((1 + k) * axes[0]) + (axes[-1] ** 2 if d == 2 else 0.0)
                              for k in range(len(hv))], axis=-1)
            dof = np.linspace(5.0, 80.0, len(hv))
            sc, se = compute_gcv_scores_batch(sh, m_all, dof, 0.1 * dof, np.full(len(hv), 0.3))
        out = dict(kind="batch", x=x, y=y, h=h, opts=repr(opts),
                   x_scaled=np.asarray(sh.x_scaled), mean=np.asarray(sh.mean),
                   std=np.asarray(sh.std), bandwidths_filtered=np.asarray(sh.bandwidths_filtered),
                   grid_shape=np.asarray(sh.grid_shape), L=np.asarray(sh.kdf_params["L"]),
                   qin=np.asarray(sh.kdf_params["qin"]), qout=np.asarray(sh.kdf_params["qout"]),
                   eval_points=pts, eval_values=np.asarray(ev), m_all=m_all, dof=dof,
                   gcv_scores=np.asarray(sc), gcv_stderr=np.asarray(se))
        for k, ax in enumerate(sh.grid_axes_raw):
            out[f"axis{k}"] = np.asarray(ax)
            out[f"axis_scaled{k}"] = np.asarray(sh.grid_axes_scaled[k])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(f"{name}: N={n} d={d} H={len(hv)} eval {np.asarray(ev).shape}")


def cubic_cases(fastlpr):
    """2-D+ data with n < 5000, where the reference interpolates GCV and DoF
    with scipy's not-a-knot cubic spline (api.py:594-600, api.py:651-657).
    Kind 'lpr_cubic': scipy solves the spline system iteratively (gcrotmk,
    atol 1e-6), so GCV/DoF carry that solver's residual."""
    rng = np.random.default_rng(123)
    n = 2000
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(np.pi * x[:, 1]) + 0.2 * rng.standard_normal(n)
    hv = np.logspace(np.log10(0.04), np.log10(0.5), 6)
    _lpr_case(fastlpr, "lpr2d_o1_cubic", x, y, np.column_stack([hv, hv]), {"order": 1},
              extra={"kind": "lpr_cubic"})
    n3 = 3000
    x3 = rng.random((n3, 3))
    y3 = np.sin(2 * np.pi * x3[:, 0]) + x3[:, 1] * x3[:, 2] + 0.2 * rng.standard_normal(n3)
    h3 = np.logspace(np.log10(0.1), np.log10(0.6), 4)
    _lpr_case(fastlpr, "lpr3d_o1_cubic", x3, y3, np.column_stack([h3, h3, h3]),
              {"order": 1, "N": [16, 16, 16]}, extra={"kind": "lpr_cubic"})
    n0 = 1500
    x0 = rng.random((n0, 2))
    y0 = np.exp(-4 * ((x0[:, 0] - 0.5) ** 2 + (x0[:, 1] - 0.4) ** 2)) + 0.1 * rng.standard_normal(n0)
    h0 = np.logspace(np.log10(0.05), np.log10(0.4), 5)
    _lpr_case(fastlpr, "lpr2d_o0_cubic_gcv", x0, y0, np.column_stack([h0, h0]),
              {"order": 0, "N": [30, 24], "dof_interp_method": "linear"},
              extra={"kind": "lpr_cubic"})


def kernel_cases(fastlpr):
    """Non-Gaussian kernel_type values (kernel.py:159-431): radial kernels
    of ||u||, not separable over the axes in 2-D."""
    rng = np.random.default_rng(321)
    n = 3000
    x1 = rng.random((n, 1))
    y1 = np.sin(2 * np.pi * x1[:, 0]) + 0.1 * rng.standard_normal(n)
    h1 = np.logspace(np.log10(0.03), np.log10(0.5), 6)[:, None]
    _lpr_case(fastlpr, "lpr1d_o1_epan", x1, y1, h1,
              {"order": 1, "N": 256, "kernel_type": "epanechnikov"})
    _lpr_case(fastlpr, "lpr1d_o2_quartic", x1, y1, h1,
              {"order": 2, "N": 200, "kernel_type": "quartic"})
    n2 = 6000
    x2 = rng.random((n2, 2))
    y2 = np.sin(2 * np.pi * x2[:, 0]) * np.cos(np.pi * x2[:, 1]) + 0.1 * rng.standard_normal(n2)
    hv = np.logspace(np.log10(0.06), np.log10(0.5), 5)
    h2 = np.column_stack([hv, hv])
    _lpr_case(fastlpr, "lpr2d_o1_tricube", x2, y2, h2,
              {"order": 1, "N": [48, 40], "kernel_type": "tricube"})
    _lpr_case(fastlpr, "lpr2d_o0_uniform", x2, y2, h2,
              {"order": 0, "N": [40, 40], "kernel_type": "uniform"})
    _lpr_case(fastlpr, "lpr2d_o1_triweight", x2, y2, h2,
              {"order": 1, "N": [32, 36], "kernel_type": "triweight"})
    _lpr_case(fastlpr, "lpr2d_o1_gaussft", x2, y2, h2,
              {"order": 1, "N": [40, 40], "kernel_type": "gaussian_ft"})
    xk = rng.standard_normal((3000, 2))
    _kde_case(fastlpr, "kde2d_epan", xk, h2, {"N": [40, 40], "kernel_type": "epanechnikov"})


if __name__ == "__main__":
    if "--only-kernels" in sys.argv:
        kernel_cases(_import_reference())
    elif "--only-cubic" in sys.argv:
        cubic_cases(_import_reference())
    elif "--only-interval" in sys.argv:
        interval_case(_import_reference())
    elif "--only-accuracy" in sys.argv:
        accuracy_cases(_import_reference())
    elif "--only-accuracy3d" in sys.argv:
        accuracy3d_cases(_import_reference())
    elif "--only-extrapolation" in sys.argv:
        extrapolation_cases(_import_reference())
    elif "--only-batch" in sys.argv:
        batch_cases(_import_reference())
    else:
        main()
