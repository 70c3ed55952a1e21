"""GPU checks of the learned bandwidth proposal: the BF16 tensor-core GEMM,
the network's forward / backward / Adam kernels against the CPU oracle
(which applies the same BF16 roundings), the binned moment sums, training,
and the learned search of cv_fastlpr including its fallback."""
import numpy as np
import pytest
import torch

from oracle import mlp as om

pytestmark = pytest.mark.gpu


def _lib():
    from fastlpr_b200 import _lib as L
    return L, L.load()


def _bf16(a, dev="cuda"):
    return torch.tensor(np.asarray(a, np.float32), device=dev).to(torch.bfloat16)


@pytest.mark.parametrize("a_trans", [0, 1])
@pytest.mark.parametrize("b_nk", [0, 1])
@pytest.mark.parametrize("epi", ["plain", "bias_relu", "mask"])
def test_gemm_layouts_and_epilogues(cuda_ok, a_trans, b_nk, epi):
    L, lib = _lib()
    rng = np.random.default_rng(10 + 4 * a_trans + 2 * b_nk)
    M, N, K = 77, 130, 45                       # ragged against the 64 x 64 x 32 tiles
    A = om.to_bf16(rng.standard_normal((M, K)))
    B = om.to_bf16(rng.standard_normal((K, N)))
    bias = rng.standard_normal(N).astype(np.float32)
    mask = om.to_bf16(rng.standard_normal((M, N)))
    dA = _bf16(A.T.copy() if a_trans else A)
    dB = _bf16(B.T.copy() if b_nk else B)
    lda = M if a_trans else K
    ldb = K if b_nk else N
    C32 = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    C16 = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda")
    db = torch.tensor(bias, device="cuda") if epi == "bias_relu" else None
    dm = _bf16(mask) if epi == "mask" else None
    L.check(lib.flpr_mlp_gemm(M, N, K, dA.data_ptr(), lda, a_trans, dB.data_ptr(), ldb, b_nk,
                              db.data_ptr() if db is not None else None,
                              1 if epi == "bias_relu" else 0,
                              dm.data_ptr() if dm is not None else None, N,
                              C32.data_ptr(), C16.data_ptr(), N,
                              torch.cuda.current_stream().cuda_stream))
    ref = A.astype(np.float64) @ B.astype(np.float64)
    if epi == "bias_relu":
        ref = np.maximum(ref + bias, 0.0)
    if epi == "mask":
        ref = np.where(mask > 0, ref, 0.0)
    got = C32.cpu().numpy()
    scale = np.max(np.abs(ref)) + 1e-30
    assert np.max(np.abs(got - ref)) / scale < 1e-5
    assert np.max(np.abs(C16.float().cpu().numpy() - ref)) / scale < 1e-2


def _net(dims, seed):
    from fastlpr_b200 import learned
    return learned.init_params(dims, seed) + 0.02 * np.random.default_rng(seed).standard_normal(
        learned.init_params(dims, seed).shape).astype(np.float32)


def test_forward_backward_match_oracle(cuda_ok):
    L, lib = _lib()
    dims = [40, 64, 48, 3]
    params = _net(dims, 11)
    rng = np.random.default_rng(12)
    B = 100
    x = rng.standard_normal((B, dims[0])).astype(np.float32)
    dout = rng.standard_normal((B, dims[-1])).astype(np.float32)
    dims_c = L.ivec(dims)
    nl = len(dims) - 1
    assert lib.flpr_mlp_param_count(nl, dims_c) == params.size
    s = torch.cuda.current_stream().cuda_stream
    p32 = torch.tensor(params, device="cuda")
    p16 = p32.to(torch.bfloat16)
    x16 = _bf16(x)
    ws = torch.empty(lib.flpr_mlp_ws(nl, dims_c, B), dtype=torch.uint8, device="cuda")
    out = torch.empty((B, dims[-1]), dtype=torch.float32, device="cuda")
    L.check(lib.flpr_mlp_fwd(nl, dims_c, p16.data_ptr(), p32.data_ptr(), B, x16.data_ptr(),
                             out.data_ptr(), ws.data_ptr(), ws.numel(), s))
    ref_out, hs = om.forward(params, dims, x)
    assert np.max(np.abs(out.cpu().numpy() - ref_out)) / np.max(np.abs(ref_out)) < 1e-2
    grad = torch.empty(params.size, dtype=torch.float32, device="cuda")
    dd = torch.tensor(dout, device="cuda")
    L.check(lib.flpr_mlp_bwd(nl, dims_c, p16.data_ptr(), B, x16.data_ptr(), dd.data_ptr(),
                             grad.data_ptr(), ws.data_ptr(), ws.numel(), s))
    ref_g = om.backward(params, dims, hs, dout)
    g = grad.cpu().numpy()
    # every parameter block within BF16-level agreement of the oracle
    o = 0
    for l in range(nl):
        for size in (dims[l + 1] * dims[l], dims[l + 1]):
            blk, rblk = g[o:o + size], ref_g[o:o + size]
            assert np.max(np.abs(blk - rblk)) <= 2e-2 * np.max(np.abs(rblk)) + 1e-6, (l, size)
            o += size
    # and it points along the gradient of the unrounded network (whose exact
    # form is checked against finite differences); BF16 activations and
    # gradients alone move it by a few percent in norm
    exact = om.backward_exact(params.astype(np.float64), dims, om.to_bf16(x), dout)
    cos = float(g @ exact) / (np.linalg.norm(g) * np.linalg.norm(exact))
    assert cos > 0.99


def test_adam_step_matches_oracle(cuda_ok):
    L, lib = _lib()
    rng = np.random.default_rng(13)
    n = 1000
    p, g = rng.standard_normal(n).astype(np.float32), rng.standard_normal(n).astype(np.float32)
    m, v = (0.1 * rng.standard_normal(n)).astype(np.float32), rng.random(n).astype(np.float32)
    dp, dg, dm, dv = (torch.tensor(a, device="cuda") for a in (p, g, m, v))
    p16 = torch.empty(n, dtype=torch.bfloat16, device="cuda")
    L.check(lib.flpr_mlp_step(n, dp.data_ptr(), p16.data_ptr(), dg.data_ptr(), dm.data_ptr(),
                              dv.data_ptr(), 1e-3, 0.9, 0.999, 1e-8, 1e-4, 7,
                              torch.cuda.current_stream().cuda_stream))
    rp, rm, rv = om.adam(p, g, m, v, 1e-3, 0.9, 0.999, 1e-8, 1e-4, 7)
    assert np.allclose(dp.cpu().numpy(), rp, rtol=1e-5, atol=1e-6)
    assert np.allclose(dm.cpu().numpy(), rm, rtol=1e-5, atol=1e-7)
    assert np.allclose(dv.cpu().numpy(), rv, rtol=1e-5, atol=1e-7)
    assert np.array_equal(p16.float().cpu().numpy(), om.to_bf16(dp.cpu().numpy()))


@pytest.mark.parametrize("d", [1, 2])
def test_bin_moments_match_oracle(cuda_ok, d):
    L, lib = _lib()
    rng = np.random.default_rng(20 + d)
    n = 300000
    x = rng.random((n, d)) * np.array([2.0, 0.5][:d]) - 0.3
    y = np.cos(3 * x[:, 0]) + 0.1 * rng.standard_normal(n)
    dx = torch.tensor(x, device="cuda")
    dy = torch.tensor(y, device="cuda")
    stats = torch.tensor(np.concatenate([x.min(0), x.max(0)]), device="cuda")
    out = torch.empty((3, 4096), dtype=torch.float64, device="cuda")
    L.check(lib.flpr_bin_moments(d, n, dx.data_ptr(), dy.data_ptr(), stats.data_ptr(),
                                 out.data_ptr(), torch.cuda.current_stream().cuda_stream))
    got = out.cpu().numpy()
    ref = om.bin_moments(x, y)
    assert np.array_equal(got[0], ref[0])
    assert np.max(np.abs(got[1:] - ref[1:])) < 1e-4 * np.max(np.abs(ref[1:]))


def test_training_reduces_loss(cuda_ok):
    from fastlpr_b200 import learned
    rng = np.random.default_rng(30)
    dims = [32, 64, 64, 1]
    X = rng.standard_normal((2048, 32)).astype(np.float32)
    w = rng.standard_normal(32).astype(np.float32) / np.sqrt(32)
    T = np.tanh(X @ w)[:, None].astype(np.float32)
    net = learned.BandwidthMLP(device="cuda", dims=dims, seed=3)
    x16 = net._inputs(X)
    t = torch.tensor(T, device="cuda")
    first = float(net.train_step(x16, t, lr=1e-3).item())
    for _ in range(300):
        last = net.train_step(x16, t, lr=1e-3)
    assert float(last.item()) < 0.1 * first


def _problem(seed, n=200000):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * 2 * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.3 * rng.standard_normal(n)
    return x, y


def _constant_net(t):
    """A network whose output is the proposal t for every input: zero
    weights, the last bias set (the biases are added in FP32)."""
    from fastlpr_b200 import learned
    base = learned.BandwidthMLP(device="cuda")
    p = np.zeros(base.nparams, np.float32)
    p[-1] = (t - learned.T_CENTER) / learned.T_SCALE
    return learned.BandwidthMLP(device="cuda", params=p)


def test_learned_search_window_walk_and_fallback(cuda_ok, monkeypatch):
    """A proposal on the minimum is accepted at once; a far proposal walks its
    window to the minimum; with walking disabled it falls back to the full
    sweep, whose result comes back unchanged."""
    import fastlpr_b200
    import fastlpr_b200.api as api
    from fastlpr_b200 import learned
    x, y = _problem(40)
    h = np.column_stack([learned.HGRID, learned.HGRID])
    opts = {"order": 1, "N": [128, 128]}
    full = fastlpr_b200.cv_fastlpr(x, y, h, opts)
    best = int(np.argmin(full.gcv_yhat["gcv_m"]))
    assert 4 < best < 27
    lopts = dict(opts, bandwidth_search="learned")
    # on the minimum: one window
    net = _constant_net(float(best))
    monkeypatch.setattr(learned, "default_model", lambda device: net)
    res = fastlpr_b200.cv_fastlpr(x, y, h, lopts)
    bs = res.metadata["bandwidth_search"]
    assert bs["accepted"] is True and len(bs["windows"]) == 1
    assert bs["windows"][0] == list(range(best - 2, best + 3))
    assert abs(bs["proposal_index"] - best) < 1e-5
    assert len(res.gcv_yhat["bandwidths"]) == 5
    assert np.allclose(res.h, full.h)
    assert res.gcv_yhat["gcv_m"].min() <= 1.01 * full.gcv_yhat["gcv_m"].min()
    # the window's outputs equal the full sweep's at the same bandwidths
    w = bs["windows"][0]
    assert np.allclose(res.gcv_yhat["gcv_m"], full.gcv_yhat["gcv_m"][w], rtol=1e-9)
    # far away: the window walks toward the minimum
    far = 0.0 if best > 15 else 31.0
    net = _constant_net(far)
    monkeypatch.setattr(learned, "default_model", lambda device: net)
    monkeypatch.setattr(api, "_MAX_WALKS", 10)
    res = fastlpr_b200.cv_fastlpr(x, y, h, lopts)
    bs = res.metadata["bandwidth_search"]
    assert bs["accepted"] is True and len(bs["windows"]) > 1
    assert np.allclose(res.h, full.h)
    # no walking: the full sweep runs and gives the plain result
    monkeypatch.setattr(api, "_MAX_WALKS", 0)
    res = fastlpr_b200.cv_fastlpr(x, y, h, lopts)
    assert res.metadata["bandwidth_search"]["accepted"] is False
    assert np.array_equal(res.yhat, full.yhat)
    # (the adjoint deposits use FP64 atomics: equal up to summation order)
    assert np.allclose(res.gcv_yhat["gcv_m"], full.gcv_yhat["gcv_m"], rtol=1e-12, atol=0.0)


@pytest.mark.parametrize("d", [1, 2])
def test_device_features_match_host_summary(cuda_ok, d):
    """flpr_learned_features equals learned.summarize on the same binned
    sums (float32 features) and the network's standardised BF16 inputs."""
    from fastlpr_b200 import learned
    L, lib = _lib()
    net = learned.default_model(torch.device("cuda"))
    s = torch.cuda.current_stream().cuda_stream
    bins, metas, want = [], [], []
    for k, (n, order) in enumerate([(300000, 1), (5000, 0), (20000, 2)]):
        rng = np.random.default_rng(50 + 3 * d + k)
        x = rng.random((n, d)) ** (1 + k)
        y = np.sin(5 * x[:, 0]) + (0.5 + k) * rng.standard_normal(n)
        dx, dy = torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda")
        st = torch.tensor(np.concatenate([x.min(0), x.max(0)]), device="cuda")
        b = torch.empty((3, 4096), dtype=torch.float64, device="cuda")
        L.check(lib.flpr_bin_moments(d, n, dx.data_ptr(), dy.data_ptr(), st.data_ptr(),
                                     b.data_ptr(), s))
        bins.append(b)
        metas.append((d, order, n))
        want.append(learned.summarize(b.cpu().numpy(), d, n, order))
    B = len(bins)
    db = torch.stack(bins)
    meta = torch.tensor(np.asarray(metas, np.int32), device="cuda")
    feat = torch.empty((B, learned.FEATURE_DIM), dtype=torch.float32, device="cuda")
    x16 = torch.empty((B, learned.FEATURE_DIM), dtype=torch.bfloat16, device="cuda")
    L.check(lib.flpr_learned_features(B, db.data_ptr(), meta.data_ptr(), net.fmean.data_ptr(),
                                      net.fstd.data_ptr(), feat.data_ptr(), x16.data_ptr(), s))
    got = feat.cpu().numpy()
    want = np.stack(want)
    np.testing.assert_allclose(got, want, rtol=2e-6, atol=1e-7)
    ref16 = net._inputs(want).float().cpu().numpy()
    diff = np.abs(x16.float().cpu().numpy() - ref16)
    # a feature within an ulp of a BF16 rounding boundary may round the other way
    assert np.mean(diff == 0) > 0.995
    assert np.max(diff) <= 2 ** -7 * np.maximum(np.abs(ref16), 1e-3).max()


def test_device_window_matches_host(cuda_ok):
    """flpr_learned_window equals learned.refine_window for proposals all
    over (and beyond) the canonical grid and lists of several lengths."""
    from fastlpr_b200 import learned
    L, lib = _lib()
    rng = np.random.default_rng(60)
    B = 200
    raw = rng.uniform(-2.5, 2.5, B).astype(np.float32)
    raw[:5] = (np.array([0, 3, 15.5, 28, 31]) - learned.T_CENTER) / learned.T_SCALE
    lists = [np.log(np.logspace(np.log10(rng.uniform(0.002, 0.02)),
                                np.log10(rng.uniform(0.2, 0.9)), int(rng.integers(5, 40))))
             for _ in range(B)]
    prop = learned.DeviceProposal(learned.default_model(torch.device("cuda")),
                                  [(2, 1, 1000)] * B, lists, "cuda")
    out = torch.tensor(raw, device="cuda")
    L.check(lib.flpr_learned_window(B, out.data_ptr(), learned.T_SCALE, learned.T_CENTER,
                                    len(learned.HGRID), prop.loggrid.data_ptr(), prop.lmax,
                                    prop.nlist.data_ptr(), prop.logh.data_ptr(), learned.REFINE,
                                    prop.lo.data_ptr(), prop.t.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream))
    lo = prop.lo.cpu().numpy()
    t = prop.t.cpu().numpy()
    for b in range(B):
        tb = float(np.float64(raw[b]) * learned.T_SCALE + learned.T_CENTER)
        assert t[b] == tb
        assert lo[b] == learned.refine_window(tb, lists[b])[0], b


def test_copy_rows_from_device_start(cuda_ok):
    L, lib = _lib()
    src = torch.arange(7 * 24, dtype=torch.float64, device="cuda").reshape(7, 24)
    dst = torch.zeros((3, 24), dtype=torch.float64, device="cuda")
    start = torch.tensor([4], dtype=torch.int32, device="cuda")
    L.check(lib.flpr_copy_rows(src.data_ptr(), dst.data_ptr(), 24 * 8, 3, start.data_ptr(),
                               torch.cuda.current_stream().cuda_stream))
    assert torch.equal(dst, src[4:7])


def test_trained_network_gains_over_full_sweep(cuda_ok):
    """The shipped network on held-out seeded problems (seeds the training
    never saw): its walked five-bandwidth search evaluates far fewer than the
    32 bandwidths of the sweep, is accepted in most cases, keeps every choice
    within 1% of the swept GCV optimum, and beats a fixed mid-sweep proposal."""
    import os
    from fastlpr_b200 import learned
    from fastlpr_b200 import train_bandwidth_mlp as T
    assert os.path.exists(learned.WEIGHTS_PATH), "trained network missing"
    net = learned.BandwidthMLP.load(learned.WEIGHTS_PATH, "cuda")
    feats, curves, meta = T.generate(24, seed0=77_000_000, log_every=0)
    prop = net.predict(feats)
    res = [T.search_on_curve(p, g) for p, g in zip(prop, curves)]
    fixed = [T.search_on_curve(15.5, g) for g in curves]
    ratio = np.array([r[0] / g.min() for r, g in zip(res, curves)])
    accepted = np.array([r[1] for r in res])
    evaluated = np.array([r[2] for r in res])
    assert np.all(ratio <= 1.01)
    assert accepted.mean() >= 0.6
    assert evaluated.mean() < 16
    assert evaluated.mean() < np.mean([f[2] for f in fixed])
