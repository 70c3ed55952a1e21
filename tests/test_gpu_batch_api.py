"""Shared-data batch API (reference batch.py): the batch sweep on
precomputed spectra equals cv_fastlpr; evaluation at points and the GCV
helper are consistent with it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _data(seed=50, n=20000, d=2):
    rng = np.random.default_rng(seed)
    x = rng.random((n, d))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(np.pi * x[:, -1]) + 0.2 * rng.standard_normal(n)
    return x, y


@pytest.mark.parametrize("d,precision", [(1, "fp64"), (2, "fp32")])
def test_batch_sweep_equals_cv_fastlpr(cuda_ok, d, precision):
    import fastlpr_b200 as fl
    x, y = _data(d=d)
    hv = np.logspace(np.log10(0.02), np.log10(0.5), 8)
    h = np.column_stack([hv] * d)
    opts = {"order": 1, "N": 256 if d == 1 else [96, 96], "precision": precision}
    if d == 2:
        # the batch helpers default to the cubic spline in 2-D (batch.py:646);
        # linear here so that their values are the fit's own interpolation
        opts.update(interp_method="linear", gcv_interp_method="linear")
    ref = fl.cv_fastlpr(x, y, h, opts)
    shared = fl.precompute_shared(x, y, h, opts)
    assert shared.kdf_params["dh"] == 8 and np.allclose(shared.bandwidths_filtered, h)
    assert np.allclose(shared.x_scaled.std(axis=0, ddof=1), 1.0)
    out = fl.cv_fastlpr_batch(shared, return_all_grid_values=True)
    # (the FP64 spread accumulates with FP64 atomics: equal up to summation order)
    assert np.allclose(out.yhat, ref.yhat, rtol=0, atol=1e-12 * np.max(np.abs(ref.yhat)))
    assert np.allclose(out.gcv_yhat["gcv_m"], ref.gcv_yhat["gcv_m"], rtol=1e-10, atol=0)
    assert np.allclose(out.h, ref.h)
    grids = out.metadata["all_grid_values"]
    assert len(grids) == 8 and grids[0].shape == tuple(shared.grid_shape)
    sel = int(out.gcv_yhat["id1se"])
    assert np.array_equal(grids[sel], out.fpp_yhat.values)
    # a second sweep on the same shared data gives the same answer
    again = fl.cv_fastlpr_batch(shared)
    assert np.array_equal(again.yhat, out.yhat)
    # evaluation at the data points with the selected bandwidth is the fitted values
    vals = fl.batch_evaluate_at_points(shared, x, [sel, 0])
    assert vals.shape == (x.shape[0], 2)
    assert np.max(np.abs(vals[:, 0] - out.yhat)) <= 1e-12 * np.max(np.abs(out.yhat))
    # GCV helper: the reference's formula on the given fitted grids and DoF
    m_all = np.stack(grids, axis=-1)
    dof = out.gcv_yhat["dof"]
    sc, se = fl.compute_gcv_scores_batch(shared, m_all, dof, out.gcv_yhat["dof_stderr"],
                                         np.full(8, 0.1))
    yh = fl.batch_evaluate_at_points(shared, x)
    mse = np.mean((y[:, None] - yh) ** 2, axis=0)
    pen = 1.0 / np.maximum(np.clip(1 - dof / len(y), 0, 1), 0.01) ** 2
    assert np.allclose(sc, mse * pen, rtol=1e-10)
    assert np.allclose(se, mse * 0.1, rtol=1e-10)


@pytest.mark.parametrize("name", ["batch1d", "batch2d"])
def test_batch_api_matches_reference(cuda_ok, name):
    """precompute_shared's fields, batch_evaluate_at_points (inside and
    beyond the grid) and compute_gcv_scores_batch against the reference's
    own outputs (tests/golden/batch*.npz, made by running its batch.py).  In
    2-D the batch helpers default to scipy's cubic spline, whose iterative
    coefficient solve (gcrotmk, atol 1e-6) the GPU replaces by the exact
    one: inside the grid they agree to that residual, beyond it the values
    are checked against the oracle's exact spline."""
    import os

    import oracle
    import fastlpr_b200 as fl
    from conftest import GOLDEN, elem_rel_err, load_golden, rel_err
    z = load_golden(os.path.join(GOLDEN, name + ".npz"))
    d = z["x"].shape[1]
    opts = dict(z["opts"], precision="fp64")
    sh = fl.precompute_shared(z["x"], z["y"], z["h"], opts)
    np.testing.assert_allclose(sh.x_scaled, z["x_scaled"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(sh.mean, z["mean"], rtol=1e-14)
    np.testing.assert_allclose(sh.std, z["std"], rtol=1e-14)
    np.testing.assert_array_equal(sh.bandwidths_filtered, z["bandwidths_filtered"])
    np.testing.assert_array_equal(sh.grid_shape, z["grid_shape"])
    np.testing.assert_array_equal(sh.kdf_params["L"], z["L"])
    np.testing.assert_array_equal(sh.kdf_params["qin"], z["qin"])
    np.testing.assert_array_equal(sh.kdf_params["qout"], z["qout"])
    for k in range(d):
        np.testing.assert_allclose(sh.grid_axes_raw[k], z[f"axis{k}"], rtol=1e-14)
        np.testing.assert_allclose(sh.grid_axes_scaled[k], z[f"axis_scaled{k}"], rtol=0,
                                   atol=1e-13)
    pts = z["eval_points"]
    ev = fl.batch_evaluate_at_points(sh, pts, [0, 2, 4])
    axes = [z[f"axis{k}"] for k in range(d)]
    inside = np.all([(pts[:, k] >= axes[k][0]) & (pts[:, k] <= axes[k][-1]) for k in range(d)],
                    axis=0)
    if d == 1:
        assert rel_err(ev, z["eval_values"]) < 1e-9
    else:
        assert rel_err(ev[inside], z["eval_values"][inside]) < 2e-5
        want = oracle.lpr.batch_evaluate_at_points(z["x"], z["y"], z["h"], z["opts"], pts,
                                                   [0, 2, 4])
        assert rel_err(ev, want) < 1e-9
    sc, se = fl.compute_gcv_scores_batch(sh, z["m_all"], z["dof"], 0.1 * z["dof"],
                                         np.full(len(z["dof"]), 0.3))
    tol = 1e-12 if d == 1 else 2e-5
    assert elem_rel_err(sc, z["gcv_scores"]) < tol
    assert elem_rel_err(se, z["gcv_stderr"]) < tol
