"""GPU parity: the CUDA path through the C ABI against the reference (golden
fixtures made by running it) and against the CPU oracle.

Tolerances: the FP64 path must match within 1e-9 relative, the FP32 path
(FP32 grids/FFT/products, FP64 solve and reductions) within 1e-5 relative;
max-normalised for arrays, element-wise for GCV/LCV scores.
"""
import os

import numpy as np
import pytest

import oracle
from conftest import elem_rel_err, golden_files, load_golden, rel_err

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "fp32": 1e-5}


def _fastlpr():
    import fastlpr_b200
    return fastlpr_b200


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("path", golden_files("lpr"), ids=os.path.basename)
def test_lpr_matches_reference(cuda_ok, path, prec):
    z = load_golden(path)
    opts = dict(z["opts"], precision=prec)
    r = _fastlpr().cv_fastlpr(z["x"], z["y"], z["h"], opts)
    tol = TOL[prec]
    g = r.gcv_yhat
    np.testing.assert_array_equal(g["bandwidths"], z["bandwidths"])
    if prec == "fp32" and z["opts"].get("order") == 2:
        # FP32 grids: the 1e-5 bound holds for bandwidths of at least one grid
        # spacing; below it the local-quadratic systems are too ill-conditioned
        # for FP32 S/T planes (order 2 therefore defaults to FP64 grids).
        spacing = np.array([(z[f"axis{k}"][-1] - z[f"axis{k}"][0]) / (len(z[f"axis{k}"]) - 1)
                            / np.std(z["x"][:, k], ddof=1) for k in range(z["x"].shape[1])])
        ok = np.all(z["bandwidths"] >= spacing, axis=1)
        assert ok.sum() >= 3
        assert elem_rel_err(g["gcv_m"][ok], z["gcv_m"][ok]) < tol
        assert elem_rel_err(g["gcv_m"], z["gcv_m"]) < 1e-2
        assert g["id1se"] == z["id1se"]
        return
    assert rel_err(r.yhat, z["yhat"]) < tol
    assert rel_err(r.fpp_yhat.values, z["grid_values"]) < tol
    assert elem_rel_err(g["gcv_m"], z["gcv_m"]) < tol
    assert rel_err(g["gcv_sd"], z["gcv_sd"]) < max(tol, 1e-9) * 10
    assert rel_err(g["dof"], z["dof"]) < tol
    assert rel_err(r.s0, z["s0"]) < tol
    assert g["id1se"] == z["id1se"]
    assert g["idmin"] == z["idmin"]
    if not np.isnan(z["d_norm"]):
        assert abs(r.d - z["d_norm"]) / abs(z["d_norm"]) < tol
    for k in range(z["x"].shape[1]):
        np.testing.assert_allclose(r.grid[k], z[f"axis{k}"], rtol=1e-14)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("path", golden_files("kde"), ids=os.path.basename)
def test_kde_matches_reference(cuda_ok, path, prec):
    z = load_golden(path)
    k = _fastlpr().cv_fastkde(z["x"], z["h"], dict(z["opts"], precision=prec))
    tol = TOL[prec]
    assert rel_err(k.metadata["fhat_all"], z["fhat_all"]) < tol
    assert elem_rel_err(k.lcv["lcv_m"], z["lcv_m"]) < tol
    # max-normalised: at the smallest bandwidth every LOO density is clamped
    # and the reference's standard deviation is rounding noise (5e-13)
    assert rel_err(k.lcv["lcv_sd"], z["lcv_sd"]) < tol * 10
    assert k.lcv["id1se"] == z["id1se"]
    assert k.lcv["idmax"] == z["idmax"]
    for j in range(z["x"].shape[1]):
        ax = z[f"axis{j}"]
        np.testing.assert_allclose(k.grid[j], ax, rtol=1e-13, atol=1e-14 * np.max(np.abs(ax)))


def _spread_via_abi(x_scaled_ref, x_raw, cols, G, prec):
    """Call flpr_spread directly; returns the (C, L...) grid times n."""
    import torch
    from fastlpr_b200 import _lib, api
    n, d = x_raw.shape
    ctx = api._Ctx(torch.device("cuda", 0))
    stats = api._point_stats(ctx, ctx.upload(x_raw), n, d)
    geom = api._make_geom(stats, n, d, np.asarray(G), 4, True)
    dcols = [ctx.upload(np.ascontiguousarray(c)) for c in cols.T]
    spec_dt = torch.float32 if prec == _lib.FLPR_PREC_F32 else torch.float64
    C = 1 + len(dcols)
    grid = ctx.empty((C, int(np.prod(geom.L))), dtype=spec_dt)
    ws = ctx.ws(ctx.lib.flpr_spread_ws(d, n, _lib.ivec(geom.L), geom.msp, C, prec))
    dx = ctx.upload(x_raw)
    _lib.check(ctx.lib.flpr_spread(d, n, dx.data_ptr(), _lib.dvec(geom.kmap.ravel()),
                                   _lib.ivec(geom.L), geom.msp, _lib.dvec(geom.tau), C, 1,
                                   _lib.pvec([c.data_ptr() for c in dcols]), grid.data_ptr(), prec,
                                   ws.data_ptr(), ws.numel(), ctx.stream), "spread")
    torch.cuda.synchronize()
    return grid.double().cpu().numpy().reshape((C,) + tuple(geom.L)) * n, geom


@pytest.mark.parametrize("d,G", [(1, [300]), (2, [48, 40]), (3, [12, 16, 10])])
def test_spread_kernel_matches_oracle(cuda_ok, d, G):
    from fastlpr_b200 import _lib
    rng = np.random.default_rng(10 + d)
    n = 4000
    x = rng.random((n, d)) * 2.0 - 0.3
    vals = np.column_stack([np.sin(3 * x[:, 0]), rng.standard_normal(n)])
    for prec, tol in ((_lib.FLPR_PREC_F64, 1e-12), (_lib.FLPR_PREC_F32, 2e-7)):
        g, geom = _spread_via_abi(None, x, vals, G, prec)
        xs = (x - geom.mean) / geom.std - geom.center
        xmod = oracle.knot_coordinates(xs, geom.L, np.asarray(G), geom.qin)
        ref = oracle.spread_grid(xmod, np.column_stack([np.ones(n), vals]), geom.L, geom.msp,
                                 geom.tau)
        for c in range(ref.shape[0]):
            assert rel_err(g[c], ref[c]) < tol, (prec, c)


@pytest.mark.parametrize("d,G,flag_power2", [(1, [300], True), (2, [48, 40], True),
                                              (2, [50, 33], False), (3, [12, 16, 10], True)])
def test_device_knot_map_equals_host_geometry(cuda_ok, d, G, flag_power2):
    # flpr_knot_map repeats the host geometry's arithmetic on the device
    # statistics: the knot maps must be the same bits (the spread that reads
    # them is enqueued before the host has the statistics)
    import torch
    from fastlpr_b200 import _lib, api
    rng = np.random.default_rng(30 + d)
    n = 5000
    x = rng.random((n, d)) * np.arange(1, d + 1) * 3.7 - 1.1
    ctx = api._Ctx(torch.device("cuda:0"))
    dx = ctx.upload(x)
    st_dev = api._point_stats_dev(ctx, dx, n, d)
    stats = st_dev.cpu().numpy().reshape(4, d)
    G = np.asarray(G)
    geom = api._make_geom(stats, n, d, G, 4, flag_power2)
    L, qin, _ = api._grid_params(G, flag_power2)
    ks, r0, hx = api._knot_consts(G, L, qin)
    kmap = ctx.empty(9 * d)
    ctx.check(ctx.lib.flpr_knot_map(d, n, st_dev.data_ptr(), _lib.dvec(ks), _lib.dvec(r0),
                                    _lib.dvec(hx), kmap.data_ptr(), ctx.stream), "knot_map")
    np.testing.assert_array_equal(kmap.cpu().numpy().reshape(d, 9), geom.kmap)


@pytest.mark.parametrize("d,G", [(2, [64, 64]), (3, [24, 20, 24])])
def test_fp32_spread_is_deterministic(cuda_ok, d, G):
    # the fixed-point accumulators make the grid independent of the order in
    # which points reach a tile (that order comes from atomics)
    from fastlpr_b200 import _lib
    rng = np.random.default_rng(7)
    x = rng.random((20000, d))
    v = rng.standard_normal((20000, 3))
    a, _ = _spread_via_abi(None, x, v, G, _lib.FLPR_PREC_F32)
    b, _ = _spread_via_abi(None, x, v, G, _lib.FLPR_PREC_F32)
    np.testing.assert_array_equal(a, b)


def _compare_to_oracle(r, o, tol):
    assert rel_err(r.yhat, o["yhat"]) < tol
    assert elem_rel_err(r.gcv_yhat["gcv_m"], o["gcv_m"]) < tol
    assert rel_err(r.gcv_yhat["dof"], o["dof_all"]) < tol
    assert r.gcv_yhat["id1se"] == o["id1se"]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_multi_response_and_aggregation(cuda_ok, prec):
    rng = np.random.default_rng(21)
    n = 4000
    x = rng.random((n, 1))
    y = np.column_stack([np.sin(2 * np.pi * x[:, 0]), np.cos(3 * x[:, 0])])
    y = y + 0.1 * rng.standard_normal(y.shape)
    h = oracle.get_hlist(6, [0.03, 0.5])
    for agg in ("first", "average", "sum"):
        opts = {"order": 1, "N": 128, "gcv_selection": agg}
        o = oracle.cv_fastlpr(x, y, h, opts)
        r = _fastlpr().cv_fastlpr(x, y, h, dict(opts, precision=prec))
        _compare_to_oracle(r, o, TOL[prec])
        assert r.yhat.shape == (n, 2)


def test_random_matrix_and_dstd_options(cuda_ok):
    rng = np.random.default_rng(22)
    n = 3000
    x = rng.random((n, 1))
    y = np.sin(2 * np.pi * x[:, 0]) + 0.2 * rng.standard_normal(n)
    h = oracle.get_hlist(7, [0.02, 0.6])
    rm = rng.standard_normal((n, 5))
    opts = {"order": 2, "N": 200, "random_matrix": rm, "dstd": 1.0}
    o = oracle.cv_fastlpr(x, y, h, opts)
    r = _fastlpr().cv_fastlpr(x, y, h, dict(opts, precision="fp64"))
    _compare_to_oracle(r, o, 1e-9)


@pytest.mark.parametrize("order", [0, 1, 2])
def test_fast_path_without_dof(cuda_ok, order):
    rng = np.random.default_rng(23)
    n = 3000
    x = rng.random((n, 2))
    y = x[:, 0] * np.sin(4 * x[:, 1]) + 0.05 * rng.standard_normal(n)
    h = np.array([[0.3, 0.3], [0.1, 0.1], [0.6, 0.6]])
    opts = {"order": order, "N": [40, 40], "calc_dof": False}
    o = oracle.cv_fastlpr(x, y, h, opts)
    r = _fastlpr().cv_fastlpr(x, y, h, dict(opts, precision="fp64"))
    assert rel_err(r.yhat, o["yhat"]) < 1e-9
    assert rel_err(r.s0, o["s0"]) < 1e-9
    assert np.isnan(r.dof)


def test_metric_shape_against_oracle(cuda_ok):
    """2-D local-linear GCV sweep with the metric's shape at a size the oracle
    finishes quickly (N=1e5, grid 128^2, 8 bandwidths)."""
    rng = np.random.default_rng(0)
    n = 100_000
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.1 * rng.standard_normal(n)
    hv = np.logspace(np.log10(0.005), np.log10(0.5), 8)
    h = np.column_stack([hv, hv])
    opts = {"order": 1, "N": [128, 128]}
    o = oracle.cv_fastlpr(x, y, h, opts)
    for prec in ("fp64", "fp32"):
        r = _fastlpr().cv_fastlpr(x, y, h, dict(opts, precision=prec))
        _compare_to_oracle(r, o, TOL[prec])


def test_fp32_and_fp64_paths_agree_at_full_metric_size(cuda_ok):
    """Size-independent check at N=1e6, grid 512^2, 32 bandwidths: the FP32
    path stays within 1e-5 of the FP64 path and selects the same bandwidth."""
    rng = np.random.default_rng(0)
    n = 1_000_000
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.1 * rng.standard_normal(n)
    hv = np.logspace(np.log10(0.005), np.log10(0.5), 32)
    h = np.column_stack([hv, hv])
    opts = {"order": 1, "N": [512, 512]}
    r64 = _fastlpr().cv_fastlpr(x, y, h, dict(opts, precision="fp64"))
    r32 = _fastlpr().cv_fastlpr(x, y, h, dict(opts, precision="fp32"))
    assert rel_err(r32.yhat, r64.yhat) < 1e-5
    assert elem_rel_err(r32.gcv_yhat["gcv_m"], r64.gcv_yhat["gcv_m"]) < 1e-5
    assert r32.gcv_yhat["id1se"] == r64.gcv_yhat["id1se"]
    # a constant response is reproduced up to the ridge lambda = 1e-6 max diag S,
    # which weighs most where the local moment matrices are small (edges)
    rc = _fastlpr().cv_fastlpr(x, np.full(n, 2.5), h[::8], dict(opts, precision="fp64"))
    assert np.median(np.abs(rc.yhat - 2.5)) < 2e-5
    assert np.max(np.abs(rc.yhat - 2.5)) < 1e-3


def test_interpolant_and_predict(cuda_ok):
    rng = np.random.default_rng(24)
    n = 2000
    x = rng.random((n, 1))
    y = np.sin(2 * np.pi * x[:, 0]) + 0.1 * rng.standard_normal(n)
    fl = _fastlpr()
    r = fl.cv_fastlpr(x, y, fl.get_hlist(5, [0.05, 0.5]), {"order": 1, "N": 128})
    xn = np.linspace(0, 1, 50).reshape(-1, 1)
    p = fl.fastlpr_predict(r, xn)
    ref = oracle.linear_interp(r.grid, r.fpp_yhat.values, xn)
    assert rel_err(p, ref) < 1e-14
    assert np.allclose(r.fpp_yhat(x), r.yhat)


@pytest.mark.parametrize("d,G", [(1, [256]), (2, [64, 48]), (3, [16, 16, 12])])
def test_dual_form_reductions_match_pointwise(cuda_ok, d, G):
    """GCV/Hutchinson sums from the adjoint deposits equal the point-wise
    interpolation of every (bandwidth, channel)."""
    rng = np.random.default_rng(30 + d)
    n = 20000
    x = rng.random((n, d))
    y = np.sin(2 * np.pi * x[:, 0]) + 0.2 * rng.standard_normal(n)
    hv = np.array([0.05, 0.15, 0.5])
    h = np.column_stack([hv] * d)
    opts = {"order": 1, "N": G, "precision": "fp64"}
    a = _fastlpr().cv_fastlpr(x, y, h, opts)
    b = _fastlpr().cv_fastlpr(x, y, h, dict(opts, _direct_reduce=True))
    assert elem_rel_err(a.gcv_yhat["gcv_m"], b.gcv_yhat["gcv_m"]) < 1e-11
    assert rel_err(a.gcv_yhat["dof"], b.gcv_yhat["dof"]) < 1e-11
    assert rel_err(a.yhat, b.yhat) < 1e-14


@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("G", [[48, 40], [64, 64], [200, 120]])
def test_fused_2d_path_matches_cufft_path_and_oracle(cuda_ok, order, G):
    """The fused column/row-pass FFT + solve kernels (2-D FP32) agree with the
    cuFFT-based product/C2R/crop path and with the oracle."""
    rng = np.random.default_rng(40 + order)
    n = 20000
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.1 * rng.standard_normal(n)
    hv = np.array([0.04, 0.08, 0.2, 0.5])
    h = np.column_stack([hv, 0.8 * hv])
    opts = {"order": order, "N": G, "precision": "fp32"}
    from fastlpr_b200 import _lib
    import fastlpr_b200.api as api
    L, qin, qout = api._grid_params(np.array(G), True)
    assert _lib.load().flpr_lpr2d_fused_supported(_lib.ivec(G), _lib.ivec(L), _lib.ivec(qout[0]),
                                                  4, order, 11) == 1
    fused = _fastlpr().cv_fastlpr(x, y, h, opts)
    plain = _fastlpr().cv_fastlpr(x, y, h, dict(opts, _no_fused=True))
    o = oracle.cv_fastlpr(x, y, h, {"order": order, "N": G})
    tol = 1e-5 if order < 2 else 1e-4
    for r in (fused, plain):
        assert rel_err(r.yhat, o["yhat"]) < tol
        assert elem_rel_err(r.gcv_yhat["gcv_m"], o["gcv_m"]) < tol
        assert rel_err(r.gcv_yhat["dof"], o["dof_all"]) < tol
        assert rel_err(r.s0, o["s0"]) < 1e-5
    assert rel_err(fused.yhat, plain.yhat) < tol


def test_fused_2d_band_classes_match_oracle(cuda_ok):
    """1024-point row and column transforms (grid 512 x 400) over bandwidths
    whose kernel spectra end anywhere from the first 32 frequencies to the
    whole band (the per-axis band limits skip columns and products) agree
    with the oracle."""
    rng = np.random.default_rng(77)
    n = 200000
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.1 * rng.standard_normal(n)
    # standardised units: 0.01 still covers more than 4 points at n = 2e5,
    # so every bandwidth takes the fused FP32 path
    hv = np.logspace(np.log10(0.01), np.log10(0.6), 8)
    h = np.column_stack([hv, 1.1 * hv])
    opts = {"order": 1, "N": [512, 400], "precision": "fp32"}
    r = _fastlpr().cv_fastlpr(x, y, h, opts)
    assert r.metadata.get("fp64_bandwidths", 0) == 0
    o = oracle.cv_fastlpr(x, y, h, {"order": 1, "N": [512, 400]})
    assert rel_err(r.yhat, o["yhat"]) < 1e-5
    assert elem_rel_err(r.gcv_yhat["gcv_m"], o["gcv_m"]) < 1e-5
    assert rel_err(r.gcv_yhat["dof"], o["dof_all"]) < 1e-5


@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("G", [[100, 60], [200, 160], [400, 300]])
def test_fused_2d_fp64_passes_match_cufft_path_and_oracle(cuda_ok, order, G):
    """The fused column/row passes in FP64 (transform lengths 256 to 1024)
    agree with the cuFFT-plane FP64 path to rounding and with the oracle
    within the FP64 bound."""
    rng = np.random.default_rng(60 + order)
    n = 30000
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.1 * rng.standard_normal(n)
    hv = np.array([0.03, 0.08, 0.2, 0.5])
    h = np.column_stack([hv, 0.8 * hv])
    opts = {"order": order, "N": G, "precision": "fp64"}
    fused = _fastlpr().cv_fastlpr(x, y, h, opts)
    plain = _fastlpr().cv_fastlpr(x, y, h, dict(opts, _no_fused=True))
    assert rel_err(fused.yhat, plain.yhat) < 1e-11
    assert elem_rel_err(fused.gcv_yhat["gcv_m"], plain.gcv_yhat["gcv_m"]) < 1e-11
    o = oracle.cv_fastlpr(x, y, h, {"order": order, "N": G})
    assert fused.gcv_yhat["id1se"] == o["id1se"]
    assert rel_err(fused.yhat, o["yhat"]) < 1e-9
    assert elem_rel_err(fused.gcv_yhat["gcv_m"], o["gcv_m"]) < 1e-9
    assert rel_err(fused.gcv_yhat["dof"], o["dof_all"]) < 1e-9
    assert rel_err(fused.s0, o["s0"]) < 1e-9


@pytest.mark.parametrize("n,G", [(50000, [256, 256]), (300000, [200, 160])])
def test_order2_2d_default_fp64_moment_planes_match_oracle(cuda_ok, n, G):
    """2-D local quadratic at the default precision: FP32 value channels on
    the fused path with the moment planes S and the solves in FP64 (the
    sparse bandwidths wholly in FP64); every output within the FP32 bound of
    the oracle."""
    rng = np.random.default_rng(n)
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * (1.3 * x[:, 0] + 0.4 * x[:, 1])) + 0.1 * rng.standard_normal(n)
    hv = np.logspace(np.log10(0.005), np.log10(0.5), 24)
    h = np.column_stack([hv, hv])
    opts = {"order": 2, "N": G}
    r = _fastlpr().cv_fastlpr(x, y, h, opts)
    assert r.metadata["precision"] == "fp32"
    assert r.metadata["moment_planes"] == "fp64"
    o = oracle.cv_fastlpr(x, y, h, opts, workers=8)
    assert r.gcv_yhat["id1se"] == o["id1se"]
    assert rel_err(r.yhat, o["yhat"]) < 1e-5
    assert rel_err(r.fpp_yhat.values, o["grid_values"]) < 1e-5
    assert elem_rel_err(r.gcv_yhat["gcv_m"], o["gcv_m"]) < 1e-5
    assert rel_err(r.gcv_yhat["dof"], o["dof_all"]) < 1e-5
    assert rel_err(r.s0, o["s0"]) < 1e-5


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_validation_rejects_nonfinite(cuda_ok, bad):
    """NaN/Inf inputs raise the reference's ValueError (checked on the device)."""
    fl = _fastlpr()
    x = np.random.default_rng(0).random((200, 1))
    y = np.sin(x[:, 0])
    word = "NaN" if np.isnan(bad) else "Inf"
    xb = x.copy()
    xb[3, 0] = bad
    with pytest.raises(ValueError, match=f"Input x contains {word}"):
        fl.cv_fastlpr(xb, y, [[0.2]], {"order": 1})
    yb = y.copy()
    yb[4] = bad
    with pytest.raises(ValueError, match=f"Response y contains {word}"):
        fl.cv_fastlpr(x, yb, [[0.2]], {"order": 1})
    with pytest.raises(ValueError, match=f"Input x contains {word}"):
        fl.cv_fastkde(xb, [[0.2]])


@pytest.mark.parametrize("L,ratio", [([64], 2), ([48], 3), ([16, 12], 2), ([9, 8, 6], 3)])
def test_oversample_crop_matches_oracle(cuda_ok, L, ratio):
    """flpr_oversample_crop on the FFT of a random ratio*L grid against the
    oracle's crop + deconvolution; the oracle's full spectrum X enters the
    reference through real(ifft(K X)), so the device half spectrum must hold
    the Hermitian part (X[f] + conj(X[-f])) / 2."""
    import torch
    from fastlpr_b200 import _lib
    rng = np.random.default_rng(sum(L) + ratio)
    L = np.array(L)
    Li = L * ratio
    d = len(L)
    C, n = 2, 1000
    tau = np.pi * 7 / (L * L * ratio * (ratio - 0.5))
    big = rng.standard_normal((C,) + tuple(Li))
    X = oracle.lpr.nufft_spectra_oversampled(big, n, L, ratio, tau)
    conjneg = np.conj(X)
    for ax in range(1, d + 1):
        conjneg = np.roll(np.flip(conjneg, axis=ax), 1, axis=ax)
    herm = 0.5 * (X + conjneg)
    want = herm[..., :L[-1] // 2 + 1]
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    spec_in = torch.from_numpy(np.fft.rfftn(big, axes=tuple(range(1, d + 1))) / n).to(dev)
    spec_in = torch.view_as_real(spec_in.contiguous()).contiguous()
    out = torch.empty((C,) + want.shape[1:] + (2,), dtype=torch.float64, device=dev)
    _lib.check(lib.flpr_oversample_crop(d, _lib.ivec(L), _lib.ivec(Li), C, _lib.dvec(tau), ratio,
                                        spec_in.data_ptr(), out.data_ptr(), _lib.FLPR_PREC_F64,
                                        None), "oversample_crop")
    torch.cuda.synchronize()
    got = torch.view_as_complex(out).cpu().numpy()
    assert rel_err(got, want) < 1e-13


# scipy's cubic RegularGridInterpolator (the reference) solves the spline
# system iteratively (gcrotmk, atol 1e-6, rtol 1e-5); the GPU and the oracle
# solve it exactly.  Against the reference, GCV/DoF therefore hold to that
# solver's residual; against the oracle, to the usual precision bounds.
CUBIC_SOLVER_TOL = 2e-5


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("path", golden_files("lpr_cubic"), ids=os.path.basename)
def test_cubic_lpr_matches_reference_and_oracle(cuda_ok, path, prec):
    z = load_golden(path)
    opts = dict(z["opts"], precision=prec)
    r = _fastlpr().cv_fastlpr(z["x"], z["y"], z["h"], opts)
    tol = TOL[prec]
    g = r.gcv_yhat
    assert g["id1se"] == z["id1se"]
    assert g["idmin"] == z["idmin"]
    assert rel_err(r.yhat, z["yhat"]) < tol
    assert rel_err(r.fpp_yhat.values, z["grid_values"]) < tol
    assert rel_err(r.s0, z["s0"]) < tol
    assert elem_rel_err(g["gcv_m"], z["gcv_m"]) < max(tol, CUBIC_SOLVER_TOL)
    assert rel_err(g["dof"], z["dof"]) < max(tol, CUBIC_SOLVER_TOL)
    o = oracle.cv_fastlpr(z["x"], z["y"], z["h"], z["opts"])
    assert elem_rel_err(g["gcv_m"], o["gcv_m"]) < tol
    assert rel_err(g["gcv_sd"], o["gcv_sd"]) < tol * 10
    assert rel_err(g["dof"], o["dof_all"]) < tol


@pytest.mark.parametrize("shape", [(11,), (9, 14), (6, 7, 5)])
def test_spline_kernels_match_oracle(cuda_ok, shape):
    """flpr_spline_prefilter + flpr_spline_eval against the oracle's exact
    not-a-knot spline, points inside and beyond the grid."""
    import torch
    from fastlpr_b200 import _lib, spline
    from oracle import spline as ospl
    rng = np.random.default_rng(len(shape))
    d = len(shape)
    axes = [np.linspace(-1.0 + a, 2.0 + 0.5 * a, g) for a, g in enumerate(shape)]
    nval = 3
    vals = rng.standard_normal(shape + (nval,))
    pts = np.column_stack([rng.uniform(a[0] - 0.3, a[-1] + 0.3, 500) for a in axes])
    want = ospl.cubic_interp(axes, vals, pts)            # (n, nval)
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    tabs = spline.tables(axes, dev)
    M = int(np.prod(shape))
    coef = torch.from_numpy(np.ascontiguousarray(np.moveaxis(vals, -1, 0).reshape(nval, M))).to(dev)
    _lib.check(lib.flpr_spline_prefilter(d, _lib.ivec(shape), nval, 1, tabs.lu.data_ptr(),
                                         coef.data_ptr(), None), "spline_prefilter")
    dx = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    out = torch.empty((nval, pts.shape[0]), dtype=torch.float64, device=dev)
    _lib.check(lib.flpr_spline_eval(d, pts.shape[0], dx.data_ptr(), tabs.axes.data_ptr(),
                                    _lib.ivec(shape), nval, coef.data_ptr(), out.data_ptr(),
                                    None), "spline_eval")
    torch.cuda.synchronize()
    got = out.cpu().numpy().T
    assert rel_err(got, want) < 1e-12
    # coefficients themselves, prefiltered with the channels innermost
    c2 = torch.from_numpy(np.ascontiguousarray(vals.reshape(M, nval))).to(dev)
    _lib.check(lib.flpr_spline_prefilter(d, _lib.ivec(shape), 1, nval, tabs.lu.data_ptr(),
                                         c2.data_ptr(), None), "spline_prefilter")
    torch.cuda.synchronize()
    assert rel_err(c2.cpu().numpy().reshape(vals.shape), ospl.coefficients(axes, vals)) < 1e-12


def test_cubic_output_interpolant_matches_oracle(cuda_ok):
    """interp_method='cubic': the final yhat and fpp_yhat use the spline."""
    from oracle import spline as ospl
    rng = np.random.default_rng(77)
    n = 6000
    x = rng.random((n, 2))
    y = np.cos(3 * x[:, 0]) + x[:, 1] ** 2 + 0.1 * rng.standard_normal(n)
    hv = np.array([0.08, 0.15, 0.3])
    r = _fastlpr().cv_fastlpr(x, y, np.column_stack([hv, hv]),
                              {"order": 1, "N": [40, 36], "interp_method": "cubic"})
    gv = r.fpp_yhat.values
    assert rel_err(r.yhat, ospl.cubic_interp(r.grid, gv, x)) < 1e-12
    newp = np.column_stack([rng.uniform(-0.1, 1.1, 200), rng.uniform(0, 1, 200)])
    assert rel_err(r.fpp_yhat(newp), ospl.cubic_interp(r.grid, gv, newp)) < 1e-12
    lin = _fastlpr().cv_fastlpr(x, y, np.column_stack([hv, hv]), {"order": 1, "N": [40, 36]})
    assert lin.gcv_yhat["id1se"] == r.gcv_yhat["id1se"]
    np.testing.assert_allclose(lin.fpp_yhat.values, gv, rtol=1e-12)


@pytest.mark.parametrize("kernel,d", [("tricube", 2), ("uniform", 1), ("epanechnikov", 3),
                                      ("gaussian", 2)])
def test_radial_kernel_spectra_match_oracle(cuda_ok, kernel, d):
    """flpr_kernel_spectra (full-plane moment spectra of a radial kernel)
    against the oracle's compute_kernel_fourier restatement."""
    import torch
    from fastlpr_b200 import api
    rng = np.random.default_rng(d)
    n = 500
    x = rng.random((n, d)) * 3 - 1
    G = np.array([20, 14, 9][:d])
    bw = np.column_stack([np.array([0.15, 0.4, 0.9])] * d)
    order = 1
    ctx = api._Ctx(torch.device("cuda", 0))
    stats = api._point_stats(ctx, ctx.upload(x), n, d)
    geom = api._make_geom(stats, n, d, G, 4, True)
    powers = oracle.lpr.element_powers(d, order)
    K = api._kernel_spectra_full(ctx, geom, bw, powers, api._KERNEL_IDS[kernel])
    xs = (x - geom.mean) / geom.std - geom.center
    spectra, prm = oracle.kernel_spectra(xs, bw, G, order, kernel_type=kernel)
    np.testing.assert_array_equal(prm["L"], geom.L)
    half = int(geom.L[-1]) // 2 + 1
    K = K.cpu().numpy()
    K = K[..., 0] + 1j * K[..., 1]
    for e, pw in enumerate(powers):
        got = K[e].reshape((bw.shape[0],) + tuple(geom.L[:-1]) + (half,))
        want = np.moveaxis(spectra[e], -1, 0)[..., :half]
        assert rel_err(got, want) < 1e-12, (kernel, pw)


@pytest.mark.parametrize("prec", [0, 1])
def test_conv2d_sep_matches_full_inverse(cuda_ok, prec):
    """flpr_conv2d_sep (column pass shared per (channel, h, axis-0 power),
    then row passes) equals flpr_conv (full 2-D inverse per product) on the
    same spectra, factors and product list; more jobs and products than one
    chunk holds."""
    import torch
    from fastlpr_b200 import _lib, api
    rng = np.random.default_rng(31 + prec)
    G = np.array([40, 36])
    L, qin, qout = api._grid_params(G, True)
    C, H, npow = 6, 10, 5
    L1h = int(L[1]) // 2 + 1
    dev = torch.device("cuda", 0)
    cdt = torch.complex64 if prec == _lib.FLPR_PREC_F32 else torch.complex128
    # spectra of real grids and factors of real sequences, as in a fit (the
    # half-spectrum inverses assume Hermitian symmetry)
    spec = torch.from_numpy(np.fft.rfft2(rng.standard_normal((C, int(L[0]), int(L[1])))))
    spec = spec.to(cdt).to(dev)
    F = torch.from_numpy(np.concatenate(
        [np.fft.fft(rng.standard_normal((H * npow, int(La))), axis=1).ravel() for La in L])).to(dev)
    prods = [(c, h, (a, b)) for c in range(C) for h in range(H)
             for a in range(npow) for b in range(npow) if a + b < npow]
    rng.shuffle(prods)
    lib = _lib.load()
    ctx = api._Ctx(dev)
    args = (_lib.ivec([p[0] for p in prods]), _lib.ivec([p[1] for p in prods]),
            _lib.ivec([v for p in prods for v in p[2]]))
    rdt = torch.float32 if prec == _lib.FLPR_PREC_F32 else torch.float64
    outs = []
    for sep in (True, False):
        out = torch.empty((len(prods), int(np.prod(G))), dtype=rdt, device=dev)
        if sep:
            ws = ctx.ws(lib.flpr_conv2d_sep_ws(ctx.handle, _lib.ivec(G), _lib.ivec(L),
                                               len(prods), prec))
            st = lib.flpr_conv2d_sep(ctx.handle, _lib.ivec(G), _lib.ivec(L), _lib.ivec(qout[0]),
                                     H, npow, spec.data_ptr(), F.data_ptr(), len(prods), *args,
                                     0.37, 0, out.data_ptr(), prec, ws.data_ptr(), ws.numel(),
                                     ctx.stream)
        else:
            ws = ctx.ws(lib.flpr_conv_ws(ctx.handle, 2, _lib.ivec(L), len(prods), prec))
            st = lib.flpr_conv(ctx.handle, 2, _lib.ivec(G), _lib.ivec(L), _lib.ivec(qout[0]), H,
                               npow, spec.data_ptr(), F.data_ptr(), len(prods), *args, 0.37, 0,
                               out.data_ptr(), prec, ws.data_ptr(), ws.numel(), ctx.stream)
        _lib.check(st, "conv")
        outs.append(out)
    torch.cuda.synchronize()
    a, b = outs[0].double().cpu().numpy(), outs[1].double().cpu().numpy()
    assert rel_err(a, b) < (1e-5 if prec == _lib.FLPR_PREC_F32 else 1e-12)


@pytest.mark.parametrize("dual,cplx,R,agg", [(1, 0, 10, "first"), (0, 0, 10, "first"),
                                             (1, 1, 10, "first"), (0, 0, 1, "first"),
                                             (1, 0, 10, "average"), (0, 1, 6, "sum")])
def test_device_gcv_select_matches_host(cuda_ok, dual, cplx, R, agg):
    """flpr_gcv_select (GCV, DoF and the 1-SE choice on the device) equals
    the host formulas (_gcv_from_sums, _one_se_rule) on the same reductions."""
    import torch
    from fastlpr_b200 import _lib, api
    rng = np.random.default_rng(dual * 7 + cplx * 3 + R)
    H, n = 17, 5000
    dy = 2 if agg != "first" else 1
    ny = dy * (2 if cplx else 1)
    C = ny + R
    bw = np.column_stack([np.logspace(-2, -0.3, H)] * 2)
    bw[5] = bw[6]  # a tie in the bandwidth sums
    rss_true = rng.uniform(50, 80, (H, ny))
    tr = np.clip(rng.uniform(-20, 900, (R, H)), -10, None)
    pp = rng.uniform(4000, 6000, max(R, 1))
    pdot = tr * pp[:R, None] / n
    if R > 1:
        pdot[0, 3] = np.nan
    if dual:
        sq = np.concatenate([rng.uniform(900, 1000, ny), pp[:R]])
        dots = np.zeros((C, H))
        dots[ny:] = pdot
        dots[:ny] = rng.uniform(100, 200, (ny, H))
        quad = rss_true - sq[None, :ny] + 2.0 * dots[:ny].T
        packed = np.concatenate([sq, dots.ravel(), quad.ravel()])
        rss_h = sq[None, :ny] - 2.0 * dots[:ny].T + quad
        pp_h = sq[ny:]
    else:
        Rm = max(R, 1)
        pd_full = np.zeros((Rm, H))
        pd_full[:R] = pdot
        packed = np.concatenate([rss_true.ravel(), pd_full.ravel(), pp[:Rm]])
        rss_h, pp_h = rss_true, pp[:R]
    opts = {"gcv_selection": agg, "dstd": 0.5}
    want = api._gcv_from_sums(n, rss_h, pdot, pp_h, dy, bool(cplx), opts)
    wsel = api._one_se_rule(want["gcv_m"], want["gcv_sd"], bw, prefer_smaller=True, dstd=0.5)
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    dp = torch.from_numpy(packed).to(dev)
    hs = torch.from_numpy(np.sum(bw, axis=1)).to(dev)
    out = torch.empty(4 * H, dtype=torch.float64, device=dev)
    sel = torch.empty(1, dtype=torch.int32, device=dev)
    agg_id = {"first": 0, "average": 1, "sum": 2}[agg]
    _lib.check(lib.flpr_gcv_select(H, ny, R, dual, cplx, agg_id, float(n), 0.5, dp.data_ptr(),
                                   hs.data_ptr(), out.data_ptr(), sel.data_ptr(), None),
               "gcv_select")
    g4 = out.cpu().numpy().reshape(4, H)
    for k, key in enumerate(("gcv_m", "gcv_sd", "dof", "dof_stderr")):
        np.testing.assert_allclose(g4[k], want[key], rtol=1e-13, atol=1e-13, err_msg=key)
    assert int(sel.cpu()[0]) == wsel



@pytest.mark.parametrize("d,order,n", [(2, 1, 20000), (2, 0, 20000), (1, 1, 500)])
def test_sparse_bandwidths_take_fp64_planes(cuda_ok, d, order, n):
    """Few points per kernel (bandwidths below the grid spacing on sparse
    data): the FP32 path evaluates those bandwidths with FP64 planes from
    the exact fixed-point spread (same lambda over the whole list) and stays
    within 1e-5 of the oracle; the rest of the list stays FP32."""
    rng = np.random.default_rng(60 + 3 * d + order)
    x = rng.random((n, d))
    y = np.sin(2 * np.pi * x[:, 0]) * (np.cos(2 * np.pi * x[:, -1]) if d == 2 else 1.0)
    y = y + 0.1 * rng.standard_normal(n)
    hv = np.logspace(np.log10(0.005), np.log10(0.5), 12)
    h = np.column_stack([hv] * d)
    opts = {"order": order, "N": [256, 256] if d == 2 else 1024}
    o = oracle.cv_fastlpr(x, y, h, opts)
    r = _fastlpr().cv_fastlpr(x, y, h, opts)
    assert r.metadata["precision"] == "fp32"
    assert 0 < r.metadata["fp64_bandwidths"] < len(h)
    _compare_to_oracle(r, o, TOL["fp32"])
    assert rel_err(r.s0, o["s0"]) < TOL["fp32"]
    # the explicit FP64 path agrees with both
    r64 = _fastlpr().cv_fastlpr(x, y, h, dict(opts, precision="fp64"))
    _compare_to_oracle(r64, o, TOL["fp64"])


@pytest.mark.parametrize("d,G,prec", [(1, [300], 0), (2, [64, 48], 0), (2, [64, 48], 1),
                                      (2, [512, 512], 0)])
def test_sorted_deposits_match_pointwise_deposits(cuda_ok, d, G, prec):
    """flpr_deposit_sorted (from the spread's tile-sorted records, exact
    fixed point, shared-memory windows) equals flpr_deposit (one FP64
    atomic per point, corner and channel) and is bitwise reproducible."""
    import torch
    from fastlpr_b200 import _lib, api
    rng = np.random.default_rng(70 + d + prec)
    n = 50000 if G[0] < 512 else 1_000_000
    x = rng.random((n, d)) * np.arange(1, d + 1) - 0.4
    cols = np.column_stack([np.sin(3 * x[:, 0]), rng.standard_normal((n, 3))])
    ctx = api._Ctx(torch.device("cuda", 0))
    dx = ctx.upload(x)
    stats = api._point_stats(ctx, dx, n, d)
    geom = api._make_geom(stats, n, d, np.asarray(G), 4, True)
    dcols = [ctx.upload(np.ascontiguousarray(c)) for c in cols.T]
    C = 1 + len(dcols)
    spec_dt = torch.float32 if prec == _lib.FLPR_PREC_F32 else torch.float64
    grid = ctx.empty((C, int(np.prod(geom.L))), dtype=spec_dt)
    ws = ctx.ws(ctx.lib.flpr_spread_ws(d, n, _lib.ivec(geom.L), geom.msp, C, prec))
    _lib.check(ctx.lib.flpr_spread(d, n, dx.data_ptr(), _lib.dvec(geom.kmap.ravel()),
                                   _lib.ivec(geom.L), geom.msp, _lib.dvec(geom.tau), C, 1,
                                   _lib.pvec([c.data_ptr() for c in dcols]), grid.data_ptr(), prec,
                                   ws.data_ptr(), ws.numel(), ctx.stream), "spread")
    axes = api._raw_axes(geom, {})
    ax = _lib.dvec(api._axes_arg(axes))
    M, Cv, npair = int(np.prod(G)), C - 1, (2 ** d) * (2 ** d + 1) // 2
    outs = []
    for rep in range(2):
        Q, B, sq = ctx.empty((M, Cv)), ctx.empty((M, npair)), ctx.empty(Cv)
        ws2 = ctx.ws(ctx.lib.flpr_deposit_sorted_ws(d, n, _lib.ivec(geom.L), geom.msp, C))
        _lib.check(ctx.lib.flpr_deposit_sorted(d, n, dx.data_ptr(), _lib.ivec(geom.L), geom.msp,
                                               C, 1, _lib.pvec([c.data_ptr() for c in dcols]),
                                               ws.data_ptr(), ws.numel(), ax,
                                               _lib.ivec(G), _lib.ivec(api._node0_cells(geom)),
                                               Q.data_ptr(), B.data_ptr(), sq.data_ptr(),
                                               ws2.data_ptr(), ws2.numel(), ctx.stream),
                   "deposit_sorted")
        outs.append((Q, B, sq))
    Qr, Br, sqr = ctx.empty((M, Cv)), ctx.empty((M, npair)), ctx.empty(Cv)
    _lib.check(ctx.lib.flpr_deposit(d, n, dx.data_ptr(), ax, _lib.ivec(G), Cv,
                                    _lib.pvec([c.data_ptr() for c in dcols]), Qr.data_ptr(),
                                    Br.data_ptr(), sqr.data_ptr(), ctx.stream), "deposit")
    torch.cuda.synchronize()
    for a, b in zip(outs[0], outs[1]):
        assert torch.equal(a, b)                     # bitwise reproducible
    for a, b in zip(outs[0], (Qr, Br, sqr)):
        assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < 1e-12


def test_fp32_fit_is_bitwise_reproducible(cuda_ok):
    """Spread and deposits sum exactly in fixed point: the whole FP32 fit
    repeats bit for bit."""
    rng = np.random.default_rng(81)
    n = 200000
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.1 * rng.standard_normal(n)
    hv = np.logspace(np.log10(0.01), np.log10(0.4), 6)
    h = np.column_stack([hv, hv])
    opts = {"order": 1, "N": [128, 128], "precision": "fp32"}
    a = _fastlpr().cv_fastlpr(x, y, h, opts)
    b = _fastlpr().cv_fastlpr(x, y, h, opts)
    np.testing.assert_array_equal(a.yhat, b.yhat)
    np.testing.assert_array_equal(a.gcv_yhat["gcv_m"], b.gcv_yhat["gcv_m"])
    np.testing.assert_array_equal(a.gcv_yhat["dof"], b.gcv_yhat["dof"])
