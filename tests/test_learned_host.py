"""Host-side checks of the learned bandwidth proposal: the CPU oracle of the
network (checked against finite differences), the feature summary and the
search-window logic.  No GPU needed."""
import numpy as np
import pytest

from oracle import mlp as om
from fastlpr_b200 import learned


def test_bf16_rounding_known_values():
    vals = np.array([1.0, 1.00390625, 1.001953125, 1.005859375, -3.14159, 0.0], np.float32)
    r = om.to_bf16(vals)
    assert r[0] == 1.0
    assert r[1] == 1.0                       # 1 + 2^-8 is a tie: to even
    assert r[2] == 1.0                       # below half an ulp
    assert r[3] == 1.0078125                 # above half an ulp
    assert abs(r[4] - (-3.140625)) < 1e-7
    assert r[5] == 0.0


def test_oracle_backward_matches_finite_differences():
    dims = [7, 5, 4, 1]
    rng = np.random.default_rng(3)
    params = learned.init_params(dims, seed=1).astype(np.float64)
    params += 0.05 * rng.standard_normal(params.shape)
    x = rng.standard_normal((6, dims[0]))
    dout = rng.standard_normal((6, 1))
    g = om.backward_exact(params, dims, x, dout)
    eps = 1e-6
    num = np.empty_like(params)
    for i in range(params.size):
        p1, p2 = params.copy(), params.copy()
        p1[i] += eps
        p2[i] -= eps
        num[i] = (np.sum(dout * om.forward_exact(p1, dims, x)) -
                  np.sum(dout * om.forward_exact(p2, dims, x))) / (2 * eps)
    assert np.max(np.abs(g - num)) < 1e-6 * max(1.0, np.max(np.abs(num)))


def test_oracle_rounded_backward_close_to_exact():
    dims = [16, 32, 32, 1]
    rng = np.random.default_rng(4)
    params = learned.init_params(dims, seed=2)
    x = rng.standard_normal((40, dims[0])).astype(np.float32)
    dout = rng.standard_normal((40, 1)).astype(np.float32)
    out, hs = om.forward(params, dims, x)
    g16 = om.backward(params, dims, hs, dout)
    g64 = om.backward_exact(params, dims, x, dout)
    assert np.max(np.abs(g16 - g64)) < 0.05 * np.max(np.abs(g64))


def test_oracle_adam_first_step():
    p = np.array([1.0, -2.0], np.float32)
    g = np.array([0.5, -0.25], np.float32)
    z = np.zeros(2, np.float32)
    p1, m1, v1 = om.adam(p, g, z, z, lr=0.1, b1=0.9, b2=0.999, eps=1e-8, wd=0.0, step=1)
    # first bias-corrected step moves every parameter by lr against the gradient sign
    assert np.allclose(p1, p - 0.1 * np.sign(g), atol=1e-6)


def test_bin_moments_oracle_counts():
    rng = np.random.default_rng(5)
    x = rng.random((1000, 2))
    y = rng.standard_normal(1000)
    b = om.bin_moments(x, y)
    assert b.shape == (3, 4096)
    assert b[0].sum() == 1000
    assert np.isclose(b[1].sum(), y.sum())
    assert np.isclose(b[2].sum(), (y * y).sum())
    # the maximum of each axis lands in its last bin
    assert b[0].reshape(64, 64)[63].sum() >= 1 and b[0].reshape(64, 64)[:, 63].sum() >= 1


@pytest.mark.parametrize("d", [1, 2])
def test_summarize_shapes_and_invariants(d):
    rng = np.random.default_rng(6 + d)
    n = 50000
    x = rng.random((n, d))
    y = np.sin(2 * np.pi * 3 * x[:, 0]) + 0.2 * rng.standard_normal(n)
    f = learned.summarize(om.bin_moments(x, y), d, n, order=1)
    assert f.shape == (learned.FEATURE_DIM,) and f.dtype == np.float32
    assert np.all(np.isfinite(f))
    dens = f[0:64]
    assert abs(dens.mean() - 1.0) < 1e-6           # normalised count averages to one
    assert f[411 + 1] == 1.0 and f[414 + d - 1] == 1.0
    if d == 1:
        assert np.all(f[192:384] == 0.0)
    # the pooled within-cell variance of the standardised response tracks the noise share
    noise_share = 0.04 / (0.5 + 0.04)
    assert 0.5 * noise_share < f[408] < 2.5 * noise_share


def test_curve_target_parabola():
    i = np.arange(32)
    g = np.exp(0.01 * (i - 12.3) ** 2)
    assert abs(learned.curve_target(g) - 12.3) < 0.05
    assert learned.curve_target(np.exp(-0.1 * i)) == 31.0


def test_window_logic():
    lh = np.log(learned.HGRID)
    w = learned.refine_window(10.2, lh)
    assert list(w) == [8, 9, 10, 11, 12]
    assert list(learned.refine_window(0.3, lh)) == [0, 1, 2, 3, 4]
    assert list(learned.refine_window(31.0, lh)) == [27, 28, 29, 30, 31]
    assert learned.accept_window(w, 2, 32)
    assert not learned.accept_window(w, 0, 32)
    assert learned.accept_window(np.arange(5), 0, 32)          # at the start of the list
    assert learned.accept_window(np.arange(27, 32), 4, 32)     # at the end of the list
    iso = np.column_stack([learned.HGRID, learned.HGRID])
    assert learned.isotropic_log_h(iso) is not None
    assert learned.isotropic_log_h(np.column_stack([learned.HGRID, 2 * learned.HGRID])) is None
    assert learned.isotropic_log_h(iso[::-1]) is None
