"""LprPlan / cv_fastlpr_many: many fits in one captured CUDA graph give the
same results as separate cv_fastlpr calls (the same kernels run; FP64
atomics make the last bits order dependent, hence rtol 1e-12 / the FP32
bound), including replays with new responses."""
import os

import numpy as np
import pytest

import oracle
from conftest import elem_rel_err, rel_err

pytestmark = pytest.mark.gpu


def _problems(seed=0):
    """A small mix of the batched workload's kinds: 1-D and 2-D, orders
    0-2, complex responses, uneven n, a variance fit, a radial kernel and a
    2-D fit with n < 5000 (cubic GCV/DoF)."""
    rng = np.random.default_rng(seed)
    out = []
    hv = np.logspace(np.log10(0.02), np.log10(0.5), 8)
    for k, (d, n, order, cplx) in enumerate([(1, 30000, 1, False), (1, 2000, 0, False),
                                             (1, 12000, 2, True), (2, 20000, 1, False),
                                             (2, 6000, 0, True), (2, 8000, 2, False),
                                             (1, 60000, 1, True), (2, 3000, 1, False)]):
        x = rng.random((n, d))
        f = np.sin(2 * np.pi * x[:, 0]) * (np.cos(np.pi * x[:, 1]) if d == 2 else 1.0)
        if cplx:
            y = np.exp(2j * np.pi * x[:, 0]) + 0.1 * (rng.standard_normal(n)
                                                       + 1j * rng.standard_normal(n))
        else:
            y = f + 0.1 * rng.standard_normal(n)
        h = np.column_stack([hv] * d)
        opts = {"order": order, "N": 256 if d == 1 else [48, 40]}
        out.append((x, y, h, opts))
    x = rng.random((5000, 1))
    out.append((x, np.exp(np.sin(4 * x[:, 0])) + 0.2 * rng.random(5000), hv[:, None],
                {"order": 1, "N": 200, "y_type_out": "variance"}))
    x = rng.random((7000, 2))
    out.append((x, np.cos(3 * x[:, 0]) + 0.1 * rng.standard_normal(7000),
                np.column_stack([hv[2:], hv[2:]]), {"order": 1, "N": [40, 40],
                                                    "kernel_type": "epanechnikov"}))
    return out


def _same(a, b, tol):
    np.testing.assert_array_equal(a.gcv_yhat["bandwidths"], b.gcv_yhat["bandwidths"])
    assert a.gcv_yhat["id1se"] == b.gcv_yhat["id1se"]
    assert rel_err(a.yhat, b.yhat) < tol
    assert elem_rel_err(a.gcv_yhat["gcv_m"], b.gcv_yhat["gcv_m"]) < tol
    assert rel_err(a.gcv_yhat["dof"], b.gcv_yhat["dof"]) < tol
    assert rel_err(a.fpp_yhat.values, b.fpp_yhat.values) < tol
    assert rel_err(a.s0, b.s0) < tol
    if a.d is not None:
        assert abs(a.d - b.d) <= tol * abs(b.d)


def _tol(opts):
    # order 2 runs in FP64 (bound 1e-9), the rest in FP32 (bound 1e-5); the
    # same kernels run, so the differences are far smaller than either
    return 1e-9 if opts.get("order", 0) == 2 else 1e-6


@pytest.mark.parametrize("graph", [True, False])
def test_plan_matches_single_fits(cuda_ok, graph):
    import fastlpr_b200
    probs = _problems()
    plan = fastlpr_b200.LprPlan(probs, graph=graph, streams=4)
    if graph:
        # ten problems: captured as several graphs, staged and replayed in turn
        assert len(plan.segs) > 1
        assert sorted(i for sg in plan.segs for i in sg.idx) == list(range(len(probs)))
    got = plan.run()
    for (x, y, h, o), g in zip(probs, got):
        ref = fastlpr_b200.cv_fastlpr(x, y, h, o)
        _same(g, ref, _tol(o))
    # new responses on the same designs
    rng = np.random.default_rng(9)
    ys = []
    for (x, y, h, o) in probs:
        if np.iscomplexobj(y):
            ys.append(y * np.exp(0.3j))
        elif o.get("y_type_out") == "variance":
            ys.append(y * (1.0 + 0.2 * rng.random(y.shape)))
        else:
            ys.append(y + 0.05 * rng.standard_normal(y.shape))
    got2 = plan.run(ys)
    for (x, y, h, o), y2, g in zip(probs, ys, got2):
        ref = fastlpr_b200.cv_fastlpr(x, y2, h, o)
        _same(g, ref, _tol(o))


def test_plan_replay_is_reproducible(cuda_ok):
    """Replaying with y unchanged reproduces the first run."""
    import fastlpr_b200
    probs = _problems(1)[:4]
    plan = fastlpr_b200.LprPlan(probs)
    a = plan.run()
    b = plan.run([p[1] for p in probs])
    for ra, rb in zip(a, b):
        _same(ra, rb, 1e-12)


def test_segmented_plan_rejects_nonfinite_response_of_last_part(cuda_ok):
    # a NaN in a problem of the last captured graph is caught like one in
    # the first; the next finite run fits all problems again
    import fastlpr_b200
    probs = _problems()
    plan = fastlpr_b200.LprPlan(probs, streams=4)
    assert len(plan.segs) > 1
    last = plan.segs[-1].idx[-1]
    bad = [p[1].copy() for p in probs]
    bad[last][3] = np.nan
    with pytest.raises(ValueError, match="NaN or Inf"):
        plan.run(bad)
    with pytest.raises(ValueError, match="NaN or Inf"):
        plan.run()
    got = plan.run([p[1] for p in probs])
    for (x, y, h, o), g in zip(probs, got):
        _same(g, fastlpr_b200.cv_fastlpr(x, y, h, o), _tol(o))
    # after close() the host threads start again for the next run, and the
    # results of the earlier run stay as they were
    plan.close()
    again = plan.run()
    for a, b in zip(got, again):
        _same(a, b, 1e-12)


def test_plan_rejects_nonfinite_responses_and_recovers(cuda_ok):
    # the NaN/Inf check of new responses runs on the device and raises after
    # the replay (api.py:310-323 raises the same error); the next run with
    # finite responses gives the results of a fresh fit
    import fastlpr_b200
    probs = _problems()[:4]
    plan = fastlpr_b200.LprPlan(probs)
    bad = [p[1].copy() for p in probs]
    bad[2][17] = np.nan
    with pytest.raises(ValueError, match="NaN or Inf"):
        plan.run(bad)
    bad[2][17] = 0.0
    bad[3][5] = np.inf
    with pytest.raises(ValueError, match="NaN or Inf"):
        plan.run(bad)
    # the rejected responses are still on the device: a run without new
    # responses must refuse them too
    with pytest.raises(ValueError, match="NaN or Inf"):
        plan.run()
    out = plan.run([p[1] for p in probs])
    for (x, y, h, opts), r in zip(probs, out):
        _same(r, fastlpr_b200.cv_fastlpr(x, y, h, opts), _tol(opts))


def test_cv_fastlpr_many_matches_oracle(cuda_ok):
    import fastlpr_b200
    probs = _problems(2)[:3]
    got = fastlpr_b200.cv_fastlpr_many([(x, y, h, dict(o, precision="fp64"))
                                        for (x, y, h, o) in probs])
    for (x, y, h, o), g in zip(probs, got):
        z = oracle.cv_fastlpr(x, y, h, o)
        assert g.gcv_yhat["id1se"] == z["id1se"]
        assert rel_err(g.yhat, z["yhat"]) < 1e-9
        assert elem_rel_err(g.gcv_yhat["gcv_m"], z["gcv_m"]) < 1e-9


def test_spread_item_size_does_not_change_results(cuda_ok):
    """The autotuned spread work-item size only regroups the work: the
    fixed-point spread is exact and order-independent, so the FP32 fit is
    bitwise the same for every setting."""
    import fastlpr_b200
    from fastlpr_b200 import autotune
    rng = np.random.default_rng(4)
    x = rng.random((40000, 2))
    y = np.sin(4 * x[:, 0]) + 0.1 * rng.standard_normal(40000)
    hv = np.logspace(-1.7, -0.5, 6)
    h = np.column_stack([hv, hv])
    saved = autotune.get_params()
    outs = []
    try:
        for ip in (1024, 8192):
            autotune.set_params({"spread_item_points": ip})
            outs.append(fastlpr_b200.cv_fastlpr(x, y, h, {"order": 1, "N": [96, 80],
                                                          "precision": "fp32",
                                                          "calc_dof": False}))
    finally:
        autotune.set_params(saved)
    np.testing.assert_array_equal(outs[0].fpp_yhat.values, outs[1].fpp_yhat.values)


def test_tune_fit_applies_a_candidate(cuda_ok, tmp_path, monkeypatch):
    monkeypatch.setenv("FASTLPR_B200_CACHE", str(tmp_path / "c.json"))
    from fastlpr_b200 import autotune
    rng = np.random.default_rng(5)
    x = rng.random((20000, 2))
    y = np.cos(3 * x[:, 1]) + 0.1 * rng.standard_normal(20000)
    hv = np.logspace(-1.5, -0.5, 4)
    saved = autotune.get_params()
    try:
        rec = autotune.tune_fit(x, y, np.column_stack([hv, hv]), {"order": 1, "N": [64, 64]})
        assert rec["best"]["spread_item_points"] in autotune.ITEM_POINTS
        assert autotune.get_params()["spread_item_points"] == rec["best"]["spread_item_points"]
        assert os.path.exists(tmp_path / "c.json")
    finally:
        autotune.set_params(saved)


def _learned_problems(seed=70):
    """Data sets for the learned search in a plan: 1-D and 2-D, orders 0-2,
    uneven n, the canonical bandwidth list; plus a complex response (the
    network does not serve it: full sweep) and a plain full-sweep problem."""
    from fastlpr_b200 import learned
    rng = np.random.default_rng(seed)
    out = []
    for k, (d, n, order) in enumerate([(1, 40000, 1), (2, 120000, 1), (1, 9000, 2),
                                       (2, 30000, 0), (1, 70000, 0), (2, 60000, 1)]):
        x = rng.random((n, d))
        f = np.sin(2 * np.pi * (1 + k % 3) * x[:, 0]) * (np.cos(np.pi * x[:, 1]) if d == 2 else 1)
        y = f + (0.05 + 0.1 * k) * rng.standard_normal(n)
        h = np.column_stack([learned.HGRID] * d)
        out.append((x, y, h, {"order": order, "N": 512 if d == 1 else [96, 96],
                              "bandwidth_search": "learned"}))
    x = rng.random((20000, 1))
    y = np.exp(2j * np.pi * x[:, 0]) + 0.1 * rng.standard_normal(20000)
    out.append((x, y, np.column_stack([learned.HGRID]), {"order": 1, "N": 256,
                                                         "bandwidth_search": "learned"}))
    x = rng.random((15000, 2))
    out.append((x, np.cos(3 * x[:, 0]) + 0.1 * rng.standard_normal(15000),
                np.column_stack([learned.HGRID[::3]] * 2), {"order": 1, "N": [64, 64]}))
    return out


def test_plan_learned_search_matches_single_fits(cuda_ok):
    """The learned search inside the graph (proposal chain for all problems
    in one batch, windows chosen and evaluated on the device) gives each
    problem the single-fit learned search's window, choice and outputs;
    replays with new responses agree with fresh single fits too."""
    import fastlpr_b200
    probs = _learned_problems()
    plan = fastlpr_b200.LprPlan(probs, streams=4)
    try:
        for run in range(2):
            ys = [p[1] for p in probs] if run == 0 else [
                (p[1] * 1.3 + 0.2) if not np.iscomplexobj(p[1]) else p[1] * np.exp(0.4j)
                for p in probs]
            got = plan.run(ys)
            for (x, _, h, o), y, g in zip(probs, ys, got):
                ref = fastlpr_b200.cv_fastlpr(x, y, h, o)
                gs, rs = g.metadata["bandwidth_search"], ref.metadata["bandwidth_search"]
                assert gs.get("mode") == rs.get("mode")
                assert gs.get("accepted") == rs.get("accepted")
                assert gs.get("windows") == rs.get("windows")
                if gs.get("mode") == "learned" and "proposal_index" in rs:
                    assert abs(gs["proposal_index"] - rs["proposal_index"]) < 1e-4
                _same(g, ref, _tol(o))
        learned_count = sum(1 for r in got if r.metadata["bandwidth_search"].get("accepted"))
        assert learned_count >= 4
    finally:
        plan.close()
