"""Host-side logic of fastlpr_b200 that needs no GPU: bandwidth grids, input
validation, grid geometry, knot constants, selection and GCV assembly."""
import numpy as np
import pytest

import oracle
from fastlpr_b200 import api, get_hlist


def test_get_hlist_matches_oracle_and_known_values():
    h = get_hlist(5, [0.1, 1.0])
    np.testing.assert_allclose(h[:, 0], np.logspace(-1, 0, 5))
    h2 = get_hlist([3, 2], [[0.1, 1.0], [0.2, 2.0]])
    assert h2.shape == (6, 2)
    # first axis varies fastest (MATLAB ndgrid order)
    np.testing.assert_allclose(h2[:3, 1], 0.2)
    np.testing.assert_allclose(h2[3:, 1], 2.0)
    np.testing.assert_array_equal(h2, oracle.get_hlist([3, 2], [[0.1, 1.0], [0.2, 2.0]]))
    np.testing.assert_array_equal(get_hlist(1, [0.5, 0.5]), np.array([[0.5]]))
    lin = get_hlist(5, [0.5, 1.0], spacing=np.linspace)
    np.testing.assert_allclose(np.diff(lin[:, 0]), 0.125)
    with pytest.raises(ValueError):
        get_hlist([2, 2], [[0.1, 1.0]])


def test_nonfinite_messages_match_reference():
    """NaN is reported before Inf, x before y, with the reference's wording."""
    names = [("Input x", 0), ("Response y", 1)]
    api._raise_nonfinite(np.array([False, False, False, False]), names, "cv_fastlpr")
    with pytest.raises(ValueError, match="Input x contains NaN values"):
        api._raise_nonfinite(np.array([True, True, False, False]), names, "cv_fastlpr")
    with pytest.raises(ValueError, match="Input x contains Inf values"):
        api._raise_nonfinite(np.array([False, True, True, False]), names, "cv_fastlpr")
    with pytest.raises(ValueError, match="Response y contains Inf values.*cv_fastlpr"):
        api._raise_nonfinite(np.array([False, False, False, True]), names, "cv_fastlpr")


def test_validation_shapes_and_options():
    rng = np.random.default_rng(1)
    x = rng.random((30, 1))
    y = rng.random(30)
    with pytest.raises(ValueError):
        api.cv_fastlpr(x, y[:20], [[0.2]])
    with pytest.raises(ValueError):
        api.cv_fastlpr(x, np.zeros((30, 1, 1)), [[0.2]])
    for order in (-1, 3, 5):
        with pytest.raises(ValueError):
            api.cv_fastlpr(x, y, [[0.2]], {"order": order})
    for h in ([[-0.1]], [[0.0]], [[0.1], [-0.2]]):
        with pytest.raises(ValueError):
            api.cv_fastlpr(x, y, h)
    with pytest.raises(ValueError):
        api.cv_fastlpr(x, y, [[0.2, 0.3]])
    with pytest.raises(ValueError):
        api.cv_fastlpr(rng.random((40, 11)), rng.random(40), [[0.2] * 11])
    with pytest.raises(ValueError):
        api.cv_fastkde(np.array([[1.0]]))
    with pytest.raises(ValueError):
        api.cv_fastlpr(np.zeros((0, 1)), np.zeros(0), [[0.2]])


def test_unsupported_paths_raise_not_implemented():
    rng = np.random.default_rng(2)
    x = rng.random((50, 4))
    with pytest.raises(NotImplementedError):
        api.cv_fastlpr(x, rng.random(50), [[0.3] * 4], {"calc_dof": False})
    x1 = rng.random((50, 1))
    with pytest.raises(NotImplementedError):
        api.cv_fastlpr(x1, rng.random(50), [[0.3]], {"accuracy": 13})
    # the reference calls kernel_function without options: polynomial fails there
    with pytest.raises(ValueError, match="Polynomial"):
        api.cv_fastlpr(x1, rng.random(50), [[0.3]], {"kernel_type": "polynomial"})
    with pytest.raises(ValueError, match="Unknown kernel type"):
        api.cv_fastlpr(x1, rng.random(50), [[0.3]], {"kernel_type": "cauchy"})


@pytest.mark.parametrize("G,p2", [(np.array([64]), True), (np.array([512, 512]), True),
                                  (np.array([200]), False), (np.array([16, 24, 9]), True)])
def test_grid_params_match_oracle(G, p2):
    L, qin, qout = api._grid_params(G, p2)
    Lo, qino, qouto = oracle.grid_params(G, p2)
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(qin, qino)
    np.testing.assert_array_equal(qout, qouto)


@pytest.mark.parametrize("d", [1, 2, 3])
def test_knot_constants_reproduce_oracle_knots(d):
    """The per-axis constants handed to the spread kernel reproduce the
    oracle's knot coordinates bit for bit when applied in the same order."""
    rng = np.random.default_rng(3 + d)
    n = 5000
    x = rng.random((n, d)) * np.array([1.0, 3.0, 0.5])[:d] + np.array([-2.0, 5.0, 0.1])[:d]
    G = np.array([64, 40, 16])[:d]
    stats = np.stack([x.min(0), x.max(0), x.mean(0), ((x - x.mean(0)) ** 2).sum(0)])
    geom = api._make_geom(stats, n, d, G, 4, True)
    xs = (x - geom.mean) / geom.std - geom.center
    xmod_o = oracle.knot_coordinates(xs, geom.L, G, geom.qin)
    for a in range(d):
        mean, std, center, lo, scale, ks, r0, shift, hx = geom.kmap[a]
        v = (x[:, a] - mean) / std - center
        xn = (v - lo) / scale * ks + r0
        xn = np.mod(xn + 0.5, 1.0) - 0.5
        k = np.mod((xn + shift) * (2 * np.pi), 2 * np.pi)
        np.testing.assert_array_equal(k, xmod_o[:, a])
        assert hx == 2 * np.pi / geom.L[a]
    np.testing.assert_allclose(geom.lo, xs.min(0), rtol=0, atol=1e-15)


@pytest.mark.parametrize("d,order", [(1, 0), (1, 1), (1, 2), (2, 1), (2, 2), (3, 1)])
def test_element_powers_match_oracle(d, order):
    assert api._element_powers(d, order) == oracle.lpr.element_powers(d, order)
    assert api._design_powers(d, order) == oracle.design_powers(d, order)


def test_one_se_rule_cases():
    bw = np.array([[0.1], [0.2], [0.3], [0.4]])
    s = np.array([3.0, 1.0, 1.05, 2.0])
    e = np.array([0.1, 0.1, 0.1, 0.1])
    assert api._one_se_rule(s, e, bw, True, dstd=0.0) == 1
    assert api._one_se_rule(s, e, bw, True, dstd=1.0) == 2
    assert api._one_se_rule(np.array([np.nan, 2.0, 1.0, np.inf]), e, bw, True, 0.0) == 2
    with pytest.raises(ValueError):
        api._one_se_rule(np.array([np.nan, np.nan]), e[:2], bw[:2], True)
    ll = np.array([-10.0, -5.0, -5.5, -20.0])
    assert api._one_se_rule(ll, np.array([1.0, 1.0, 1.0, 1.0]), bw, False, 1.0) == 2
    for _ in range(20):
        rng = np.random.default_rng(_)
        sc = rng.random(7)
        er = rng.random(7) * 0.2
        hb = rng.random((7, 2))
        for pref in (True, False):
            assert api._one_se_rule(sc, er, hb, pref, 1.0) == oracle.one_se_rule(sc, er, hb, pref, 1.0)


def test_gcv_from_sums_matches_oracle_formulas():
    rng = np.random.default_rng(5)
    n, H, R = 1000, 6, 10
    p = rng.standard_normal((n, R))
    phat = rng.standard_normal((n, H, R)) * 0.1 + p[:, None, :] * rng.random((1, H, 1))
    y = rng.standard_normal((n, 1))
    yhat = y[:, None, :] + 0.3 * rng.standard_normal((n, H, 1))
    rss = np.sum((y[:, None, :] - yhat) ** 2, axis=0)  # (H, 1)
    pdot = np.einsum("nr,nhr->rh", p, phat)
    pp = np.sum(p * p, axis=0)
    out = api._gcv_from_sums(n, rss, pdot, pp, 1, False, {"gcv_selection": "first"})
    tr = np.clip(n * pdot / pp[:, None], 0, n)
    pen = 1.0 / np.maximum(np.clip(1 - tr / n, 0, 1), 0.01) ** 2
    np.testing.assert_allclose(out["dof"], tr.mean(0))
    np.testing.assert_allclose(out["gcv_m"], rss[:, 0] / n * pen.mean(0))
    np.testing.assert_allclose(out["gcv_sd"], rss[:, 0] / n * pen.std(0, ddof=1))


@pytest.mark.parametrize("G", [4, 5, 6, 9, 33, 200])
def test_spline_band_lu_solves_collocation(G):
    """The 7-column LU rows that flpr_spline_prefilter consumes solve the
    not-a-knot collocation system (forward / back substitution as the
    device does it)."""
    from oracle import spline as ospl
    from fastlpr_b200 import spline
    ax = np.linspace(-0.4, 2.2, G)
    T = spline.band_lu(ax)
    A = ospl.collocation(ax)
    b = np.random.default_rng(G).standard_normal(G)
    y = np.zeros(G)
    for i in range(G):
        y[i] = b[i] - sum(T[i, 3 - k] * y[i - k] for k in (1, 2, 3) if i - k >= 0)
    x = np.zeros(G)
    for i in range(G - 1, -1, -1):
        x[i] = (y[i] - sum(T[i, 3 + k] * x[i + k] for k in (1, 2, 3) if i + k < G)) * T[i, 3]
    np.testing.assert_allclose(x, np.linalg.solve(A, b), rtol=0, atol=1e-13)
    for i in range(G):
        for c in range(7):
            if not 0 <= i + c - 3 < G:
                assert T[i, c] == 0.0


def test_interp_method_resolution():
    m = api._check_interp_methods({}, 2, 1000)
    assert m == {"gcv": "cubic", "dof": "cubic", "output": "linear"}
    assert api._check_interp_methods({}, 2, 5000)["gcv"] == "linear"
    assert api._check_interp_methods({}, 1, 100)["dof"] == "linear"
    m = api._check_interp_methods({"dof_interp_method": "linear", "interp_method": "cubic"}, 3, 100)
    assert m == {"gcv": "cubic", "dof": "linear", "output": "cubic"}
    with pytest.raises(NotImplementedError):
        api._check_interp_methods({"gcv_interp_method": "quintic"}, 2, 100)
    with pytest.raises(ValueError):
        api._check_interp_methods({"N": [3, 10]}, 2, 100)
    from fastlpr_b200 import spline
    with pytest.raises(ValueError):
        spline.band_lu(np.array([0.0, 1.0, 1.0, 2.0]))


def test_bandwidth_filter_bound_matches_exact_sums():
    # the "too small bandwidth" test (convolution.py:542-605) decided from
    # the largest-term bound agrees with the decision from the exact sums
    from types import SimpleNamespace
    rng = np.random.default_rng(0)
    for _ in range(200):
        d = int(rng.integers(1, 4))
        G = rng.integers(3, 600, size=d)
        hi = rng.uniform(0.5, 3.0, size=d)
        lo = -hi * rng.uniform(0.9, 1.1, size=d)
        geom = SimpleNamespace(d=d, G=G, lo=lo, hi=hi)
        bw = np.exp(rng.uniform(np.log(1e-4), np.log(2.0), size=(40, d)))
        exact = np.prod(api._kernel_sums_host(geom, bw), axis=0) / api.SQRT_2PI
        fast = api._separable_kernel_sums(geom, bw, api.SQRT_2PI)
        np.testing.assert_array_equal(fast < api.EPS * 10, exact < api.EPS * 10)
        assert np.all(fast <= exact * (1 + 1e-12))


@pytest.mark.parametrize("dy,cplx", [(1, False), (3, False), (1, True), (2, True)])
def test_result_layout_matches_channel_rows(dy, cplx):
    # the output stage downloads fitted values / residuals / grid values in
    # the result's layout: (k,) or (k, dy), complex from real/imaginary row
    # pairs; the same arrays as assembling them from the channel rows
    import torch
    rng = np.random.default_rng(dy)
    k = 37
    rows = rng.standard_normal(((2 if cplx else 1) * dy, k))
    got = api._result_layout(torch.from_numpy(rows), dy, cplx).numpy()
    ref = rows[0::2] + 1j * rows[1::2] if cplx else rows
    ref = ref[0] if dy == 1 else ref.T
    assert got.shape == ref.shape and got.dtype == ref.dtype
    np.testing.assert_array_equal(got, ref)


def test_plan_segments_cut_issue_order_by_staged_bytes():
    # the captured graphs of a plan cover consecutive parts of the issue
    # order, the first about 1/8 of the staged response bytes
    import torch

    from fastlpr_b200.plan import LprPlan, _Problem

    rng = np.random.default_rng(3)
    sizes = rng.integers(1000, 100000, 40)
    stub = type("Stub", (), {})()
    stub.prop = None
    stub.probs = []
    for n in sizes:
        p = _Problem()
        p.staging = torch.empty((1, int(n)), dtype=torch.float64)
        stub.probs.append(p)
    stub.order = sorted(range(len(sizes)), key=lambda i: -sizes[i])
    segs = LprPlan._segment_order(stub)
    assert len(segs) == 4
    assert [i for sg in segs for i in sg] == stub.order
    total = float(sizes.sum())
    first = float(sum(sizes[i] for i in segs[0]))
    assert first - sizes[segs[0][-1]] < total / 8 <= first
    # few problems, or a learned proposal chain: one graph
    stub.order = stub.order[:5]
    assert LprPlan._segment_order(stub) == [stub.order]
    stub.order = sorted(range(len(sizes)), key=lambda i: -sizes[i])
    stub.prop = object()
    assert LprPlan._segment_order(stub) == [stub.order]


def test_plan_checks_new_responses_against_the_plan():
    # new responses must keep each problem's shape and real/complex kind; a
    # 1 x n row is taken as a column (as cv_fastlpr takes it)
    from fastlpr_b200.plan import LprPlan, _Problem

    stub = type("Stub", (), {})()
    stub.probs = []
    for shape, cplx in (((5, 1), False), ((4, 2), False), ((3, 1), True)):
        p = _Problem()
        p.su = type("Setup", (), {})()
        p.su.y_arr = np.zeros(shape, dtype=complex if cplx else float)
        p.su.y_is_complex = cplx
        stub.probs.append(p)
    good = [np.arange(5.0), np.ones((4, 2)), np.ones(3) * (1 + 2j)]
    arrs = LprPlan._check_y(stub, good)
    assert [a.shape for a in arrs] == [(5, 1), (4, 2), (3, 1)]
    row = [np.arange(5.0)[None, :], np.ones((4, 2)), np.ones(3) * 1j]
    assert LprPlan._check_y(stub, row)[0].shape == (5, 1)
    with pytest.raises(ValueError, match="expected 3 responses"):
        LprPlan._check_y(stub, good[:2])
    with pytest.raises(ValueError, match="differs from the planned"):
        LprPlan._check_y(stub, [np.arange(6.0), good[1], good[2]])
    with pytest.raises(ValueError, match="real and complex"):
        LprPlan._check_y(stub, [good[0], good[1], np.ones(3)])
