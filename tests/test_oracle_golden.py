"""The CPU oracle reproduces the reference (run in its FP64 configuration by
tests/golden/make_golden.py) on every golden fixture."""
import os

import numpy as np
import pytest

import oracle
from conftest import elem_rel_err, golden_files, load_golden, rel_err


@pytest.mark.parametrize("path", golden_files("lpr"), ids=os.path.basename)
def test_oracle_lpr_matches_reference(path):
    z = load_golden(path)
    o = oracle.cv_fastlpr(z["x"], z["y"], z["h"], z["opts"])
    assert o["id1se"] == z["id1se"]
    assert o["idmin"] == z["idmin"]
    np.testing.assert_allclose(o["bandwidths"], z["bandwidths"], rtol=0, atol=0)
    assert rel_err(o["yhat"], z["yhat"]) < 1e-12
    assert rel_err(o["grid_values"], z["grid_values"]) < 1e-12
    assert elem_rel_err(o["gcv_m"], z["gcv_m"]) < 1e-10
    assert rel_err(o["gcv_sd"], z["gcv_sd"]) < 1e-10
    assert rel_err(o["dof_all"], z["dof"]) < 1e-11
    assert rel_err(o["s0"], z["s0"]) < 1e-12
    for k in range(len(z["h"][0])):
        np.testing.assert_allclose(o["axes_raw"][k], z[f"axis{k}"], rtol=1e-15)


@pytest.mark.parametrize("path", golden_files("kde"), ids=os.path.basename)
def test_oracle_kde_matches_reference(path):
    z = load_golden(path)
    o = oracle.cv_fastkde(z["x"], z["h"], z["opts"])
    assert o["id1se"] == z["id1se"]
    assert o["idmax"] == z["idmax"]
    assert rel_err(o["fhat_all"], z["fhat_all"]) < 1e-12
    assert elem_rel_err(o["lcv_m"], z["lcv_m"]) < 1e-12
    assert elem_rel_err(o["lcv_sd"], z["lcv_sd"]) < 1e-10


def test_oracle_intermediates_match_reference():
    z = load_golden(os.path.join(os.path.dirname(__file__), "golden", "inter2d_o1.npz"))
    G = z["G"]
    spectra, prm = oracle.kernel_spectra(z["x_scaled"], z["h"], G, 1)
    np.testing.assert_array_equal(prm["L"], z["L"])
    np.testing.assert_array_equal(prm["qin"], z["qin"])
    np.testing.assert_array_equal(prm["qout"], z["qout"])
    assert rel_err(np.stack(spectra), z["kdf"]) < 1e-13
    L, qin = prm["L"], prm["qin"]
    msp, tau, _ = oracle.lpr.spread_params(L, 4)
    xmod = oracle.knot_coordinates(z["x_scaled"], L, G, qin)
    grid = oracle.spread_grid(xmod, np.column_stack([np.ones(len(z["y"])), z["y"]]), L, msp, tau)
    spec = oracle.nufft_spectra(grid, len(z["y"]))
    assert rel_err(spec[0], z["spec_ones"]) < 1e-13
    assert rel_err(spec[1], z["spec_y"]) < 1e-13
    S = [oracle.lpr.convolve(np.moveaxis(spec[:1], 0, -1), k, prm["qout"], G)[..., 0] for k in spectra]
    assert rel_err(np.stack(S), z["S"][..., 0]) < 1e-12


# scipy's 'cubic' RegularGridInterpolator solves the spline system with
# gcrotmk (atol 1e-6, rtol 1e-5); the oracle solves it exactly, so GCV and
# DoF agree with the reference to that solver's residual, everything else
# to rounding.
CUBIC_SOLVER_TOL = 2e-5


@pytest.mark.parametrize("path", golden_files("lpr_cubic"), ids=os.path.basename)
def test_oracle_cubic_lpr_matches_reference(path):
    z = load_golden(path)
    o = oracle.cv_fastlpr(z["x"], z["y"], z["h"], z["opts"])
    assert o["id1se"] == z["id1se"]
    assert o["idmin"] == z["idmin"]
    assert rel_err(o["yhat"], z["yhat"]) < 1e-12
    assert rel_err(o["grid_values"], z["grid_values"]) < 1e-12
    assert rel_err(o["s0"], z["s0"]) < 1e-12
    assert elem_rel_err(o["gcv_m"], z["gcv_m"]) < CUBIC_SOLVER_TOL
    assert rel_err(o["gcv_sd"], z["gcv_sd"]) < CUBIC_SOLVER_TOL
    assert rel_err(o["dof_all"], z["dof"]) < CUBIC_SOLVER_TOL


def test_oracle_spline_is_scipys_exact_spline():
    """The oracle's cubic interpolation equals scipy's make_ndbspl solved
    directly (spsolve) on the same grid: the restatement is exact."""
    import scipy.sparse.linalg as ssl
    from scipy.interpolate._ndbspline import make_ndbspl

    from oracle import spline
    rng = np.random.default_rng(5)
    for shape in ((9,), (7, 12), (5, 6, 8)):
        axes = [np.sort(rng.uniform(-2, 3, g)) for g in shape]
        vals = rng.standard_normal(shape + (3,))
        pts = np.column_stack([rng.uniform(a[0] - 0.2, a[-1] + 0.2, 300) for a in axes])
        want = make_ndbspl(tuple(axes), vals, 3, solver=ssl.spsolve)(pts)
        got = spline.cubic_interp(axes, vals, pts)
        assert np.abs(got - want).max() < 1e-11 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("path", golden_files("batch"), ids=os.path.basename)
def test_oracle_batch_helpers_match_reference(path):
    """batch_evaluate_at_points (points inside and beyond the grid) and
    compute_gcv_scores_batch of the reference's shared-data batch API.  In
    2-D their default is scipy's cubic spline, whose coefficients scipy
    solves iteratively (gcrotmk, atol 1e-6); the oracle solves them exactly,
    so inside the grid the two agree to that solver's residual, and beyond
    it the extended end pieces magnify the residual (checked against the
    exact spline instead)."""
    z = load_golden(path)
    d = z["x"].shape[1]
    axes = [z[f"axis{k}"] for k in range(d)]
    ev = oracle.lpr.batch_evaluate_at_points(z["x"], z["y"], z["h"], z["opts"], z["eval_points"],
                                             [0, 2, 4])
    pts = z["eval_points"]
    inside = np.all([(pts[:, k] >= axes[k][0]) & (pts[:, k] <= axes[k][-1]) for k in range(d)],
                    axis=0)
    assert inside.sum() >= 30 and (~inside).sum() >= 5
    if d == 1:
        assert rel_err(ev, z["eval_values"]) < 1e-12
    else:
        assert rel_err(ev[inside], z["eval_values"][inside]) < CUBIC_SOLVER_TOL
    opts = dict(z["opts"])
    sc, se = oracle.lpr.compute_gcv_scores_batch(axes, z["x"], z["y"], z["m_all"], z["dof"],
                                                 0.1 * z["dof"], np.full(len(z["dof"]), 0.3),
                                                 opts)
    tol = 1e-12 if d == 1 else CUBIC_SOLVER_TOL
    assert elem_rel_err(sc, z["gcv_scores"]) < tol
    assert elem_rel_err(se, z["gcv_stderr"]) < tol
