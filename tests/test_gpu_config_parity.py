"""GPU parity at the sizes of the benchmarked configurations, against the
CPU oracle on identical inputs (the same helpers print the ``parity`` object
of the benchmark line).

- the benchmark workload itself: N = 1e6, grid 512^2 (padded 1024^2, so the
  fused FP32 column/row-pass kernels run their widest instantiation), all 32
  bandwidths, the data set the benchmark fits;
- the 1-D local-linear configuration at full size (N = 1e5, grid 1024, 20 h);
- the 2-D local-quadratic heteroscedastic configuration at full size
  (N = 2e6, grid 512^2), mean and variance fits, on six of its 32
  bandwidths (smallest, largest, the full sweep's choice and neighbours);
- the 3-D KDE configuration (grid 128^3, 16 h) at N = 1e6;
- 16 problems of the batched workload through LprPlan.

Tolerances: FP32 path 1e-5, FP64 path 1e-9 relative (max-normalised for
arrays, element-wise for GCV/LCV scores), and the same selected bandwidth.
"""
import os

import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu

WORKERS = os.cpu_count() or 1


def _assert_ok(p):
    assert p["same_bandwidth"], p
    assert p["max_rel_err"] <= p["tol"], p


@pytest.fixture(scope="module")
def metric_oracle():
    _, o, _ = bench.cpu_fit(bench.replica_seed(0), workers=WORKERS)
    return o


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_benchmark_workload_matches_oracle(cuda_ok, metric_oracle, prec):
    import torch

    import fastlpr_b200
    x, y, h, opts = bench.workload(bench.replica_seed(0))
    dev = torch.device("cuda", 0)
    r = fastlpr_b200.cv_fastlpr_device(torch.from_numpy(x).to(dev), torch.from_numpy(y).to(dev),
                                       h, dict(opts, precision=prec, device=str(dev)))
    _assert_ok(bench.lpr_parity(r, metric_oracle, bench.TOL[prec]))
    # the public host-array entry point gives the same fit
    e = fastlpr_b200.cv_fastlpr(x, y, h, dict(opts, precision=prec))
    _assert_ok(bench.lpr_parity(e, metric_oracle, bench.TOL[prec]))


def test_lpr1d_config_matches_oracle(cuda_ok):
    import torch
    p = bench.parity_lpr1d(torch.device("cuda", 0), WORKERS)
    assert p["precision"] == "fp32"
    _assert_ok(p)


def test_hetero2d_config_mean_and_variance_match_oracle(cuda_ok):
    import torch
    p = bench.parity_hetero2d(torch.device("cuda", 0), WORKERS)
    assert len(p["bandwidths"]) == 6 and p["bandwidths"][0] == 0 and p["bandwidths"][-1] == 31
    _assert_ok(p["mean"])
    _assert_ok(p["variance"])


def test_kde3d_config_matches_oracle(cuda_ok):
    import torch
    p = bench.parity_kde3d(torch.device("cuda", 0), WORKERS)
    assert p["precision"] == "fp32"
    _assert_ok(p)


def test_batched_sample_matches_oracle(cuda_ok):
    import fastlpr_b200
    probs = bench.batched_sample(16)
    assert {o["order"] for (_, _, _, o) in probs} == {0, 1, 2}
    assert any(np.iscomplexobj(y) for (_, y, _, _) in probs)
    plan = fastlpr_b200.LprPlan(probs)
    try:
        res = plan.run()
    finally:
        plan.close()
    p = bench.parity_batched(res, probs, WORKERS)
    assert set(p) == {"fp32", "fp64"}
    for q in p.values():
        assert q["all_same_bandwidth"] and q["ok"], p
