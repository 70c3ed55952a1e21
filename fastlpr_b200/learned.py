"""Learned bandwidth proposal for ``cv_fastlpr``.

The reference sweeps every bandwidth of the list (api.py:645-741).  Here a
small MLP reads binned moment summaries of the data set and proposes where
the GCV minimum lies on a canonical sweep; ``cv_fastlpr`` with option
``bandwidth_search='learned'`` then evaluates only the five bandwidths of
the list around the proposal and accepts the result when its GCV minimum is
interior to that window (or at an end of the whole list).  Otherwise it runs
the full sweep, which stays the fallback and the reference score.

Everything runs on the GPU through the C ABI: ``flpr_bin_moments`` for the
summaries, ``flpr_mlp_fwd/bwd/step`` (BF16 tensor-core products with FP32
accumulation) for inference and training.  PyTorch only holds the buffers.

Input summary (``FEATURE_DIM`` = 416 values):

* per axis (two slots; the second is zero for 1-D data): 64-bin histograms
  of the normalised count (64 n_b / n), the mean of the standardised
  response and the mean of its square;
* 12 lag-roughness values of the cell means (mean squared difference of the
  standardised cell means at lags 2^k / 4096 of the data range, k = 0..11),
  raw and with the expected noise contribution removed;
* the pooled within-cell variance of the standardised response (a noise
  estimate) and its logarithm;
* log10(n) / 6, the order one-hot (3) and the dimension one-hot (2).

Target: the position of the GCV minimum on the canonical sweep ``HGRID``
(32 log-spaced isotropic bandwidths in [0.005, 0.5], z-units), as a
fractional index refined by a parabola through the three lowest points.
"""
from __future__ import annotations

import os
import threading
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib

FEATURE_DIM = 416
DIMS = (FEATURE_DIM, 256, 256, 256, 1)
CELLS = 4096
NLAGS = 12
HGRID = np.logspace(np.log10(0.005), np.log10(0.5), 32)
REFINE = 5
T_CENTER, T_SCALE = 15.5, 9.0
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                            "bandwidth_mlp.npz")


def bins_per_axis(d: int) -> int:
    return 4096 if d == 1 else 64


# ---------------------------------------------------------------- summaries

def bin_moments(dx: torch.Tensor, dy: torch.Tensor, d_stats: torch.Tensor, n: int, d: int,
                stream) -> torch.Tensor:
    """(3, 4096) count, sum y, sum y^2 per cell (flpr_bin_moments), on the device."""
    lib = _lib.load()
    out = torch.empty((3, CELLS), dtype=torch.float64, device=dx.device)
    _lib.check(lib.flpr_bin_moments(d, n, dx.data_ptr(), dy.data_ptr(), d_stats.data_ptr(),
                                    out.data_ptr(), stream), "flpr_bin_moments")
    return out


def _aggregate_axis(a: np.ndarray, d: int, axis: int) -> np.ndarray:
    """Per-axis 64-bin marginal of a 4096-cell field."""
    if d == 1:
        return a.reshape(64, 64).sum(axis=1)
    g = a.reshape(64, 64)
    return g.sum(axis=1 - axis)


def summarize(bins: np.ndarray, d: int, n: int, order: int) -> np.ndarray:
    """Feature vector (FEATURE_DIM,) float32 of one data set from its binned sums."""
    cnt, sy, syy = (np.asarray(b, dtype=np.float64) for b in bins)
    N = max(cnt.sum(), 1.0)
    ybar = sy.sum() / N
    var = max(syy.sum() / N - ybar * ybar, 0.0)
    sd = np.sqrt(var) if var > 0 else 1.0
    sz = (sy - cnt * ybar) / sd
    szz = (syy - 2.0 * ybar * sy + cnt * ybar * ybar) / (sd * sd)
    f = np.zeros(FEATURE_DIM, dtype=np.float64)
    for a in range(d):
        c = _aggregate_axis(cnt, d, a)
        s1 = _aggregate_axis(sz, d, a)
        s2 = _aggregate_axis(szz, d, a)
        with np.errstate(invalid="ignore", divide="ignore"):
            mean = np.where(c > 0, s1 / np.maximum(c, 1.0), 0.0)
            msq = np.where(c > 0, s2 / np.maximum(c, 1.0), 0.0)
        f[192 * a:192 * a + 64] = 64.0 * c / N
        f[192 * a + 64:192 * a + 128] = mean
        f[192 * a + 128:192 * a + 192] = msq
    ok = cnt >= 2
    dof = np.sum(cnt[ok] - 1.0)
    within = np.sum(szz[ok] - sz[ok] ** 2 / cnt[ok]) / dof if dof > 0 else 0.0
    within = max(within, 0.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        mu = np.where(cnt > 0, sz / np.maximum(cnt, 1.0), np.nan)
        inv = np.where(cnt > 0, 1.0 / np.maximum(cnt, 1.0), np.nan)
    field = mu.reshape((4096,) if d == 1 else (64, 64))
    finv = inv.reshape(field.shape)
    for k in range(NLAGS):
        lag = 2 ** k
        if d == 2:
            if lag < 64:
                continue
            lag //= 64
        raw, cor = [], []
        for a in range(d):
            lo = [slice(None)] * d
            hi = [slice(None)] * d
            lo[a] = slice(0, field.shape[a] - lag)
            hi[a] = slice(lag, None)
            diff = field[tuple(hi)] - field[tuple(lo)]
            noise = within * (finv[tuple(hi)] + finv[tuple(lo)])
            good = np.isfinite(diff)
            if np.any(good):
                r = float(np.mean(diff[good] ** 2))
                raw.append(r)
                cor.append(r - float(np.mean(noise[good])))
        if raw:
            f[384 + k] = np.mean(raw)
            f[384 + NLAGS + k] = np.mean(cor)
    f[408] = within
    f[409] = np.log10(within + 1e-6) / 3.0
    f[410] = np.log10(max(n, 1)) / 6.0
    f[411 + int(order)] = 1.0
    f[414 + (d - 1)] = 1.0
    return f.astype(np.float32)


def dataset_features(dx: torch.Tensor, y_col: torch.Tensor, d_stats: torch.Tensor, n: int,
                     d: int, order: int, stream) -> np.ndarray:
    """Features of one data set already on the device (synchronises)."""
    b = bin_moments(dx, y_col, d_stats, n, d, stream)
    return summarize(b.cpu().numpy(), d, n, order)


def curve_target(gcv: np.ndarray) -> float:
    """Fractional index of the minimum of a GCV curve (parabola through the
    three lowest points of log GCV around the discrete minimum)."""
    g = np.log(np.maximum(np.asarray(gcv, dtype=np.float64), 1e-300))
    finite = np.isfinite(g)
    if not np.any(finite):
        return T_CENTER
    g = np.where(finite, g, np.inf)
    i = int(np.argmin(g))
    if 0 < i < len(g) - 1 and np.isfinite(g[i - 1]) and np.isfinite(g[i + 1]):
        den = g[i - 1] - 2.0 * g[i] + g[i + 1]
        if den > 0:
            return float(i + np.clip(0.5 * (g[i - 1] - g[i + 1]) / den, -0.5, 0.5))
    return float(i)


# ---------------------------------------------------------------- network

def init_params(dims: Sequence[int], seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases, packed as the C ABI expects."""
    rng = np.random.default_rng(seed)
    parts = []
    for l in range(len(dims) - 1):
        n_in, n_out = dims[l], dims[l + 1]
        std = np.sqrt(2.0 / n_in) if l < len(dims) - 2 else np.sqrt(1.0 / n_in)
        parts.append((rng.standard_normal((n_out, n_in)) * std).ravel())
        parts.append(np.zeros(n_out))
    return np.concatenate(parts).astype(np.float32)


class BandwidthMLP:
    """The proposal network: FP32 master parameters, BF16 compute copy and
    Adam moments on the device; feature standardisation folded in front."""

    def __init__(self, device=None, dims: Sequence[int] = DIMS, params: Optional[np.ndarray] = None,
                 fmean: Optional[np.ndarray] = None, fstd: Optional[np.ndarray] = None,
                 seed: int = 0):
        self.lib = _lib.load()
        self.device = torch.device(device if device is not None else "cuda")
        self.dims = [int(v) for v in dims]
        self.nl = len(self.dims) - 1
        self._dims_c = _lib.ivec(self.dims)
        self.nparams = int(self.lib.flpr_mlp_param_count(self.nl, self._dims_c))
        if self.nparams <= 0:
            raise ValueError(f"bad network dims {self.dims}")
        if params is None:
            params = init_params(self.dims, seed)
        if params.size != self.nparams:
            raise ValueError(f"parameter vector has {params.size} entries, expected {self.nparams}")
        self.p32 = torch.tensor(np.asarray(params, np.float32), device=self.device)
        self.p16 = torch.empty(self.nparams, dtype=torch.bfloat16, device=self.device)
        self.grad = torch.zeros(self.nparams, dtype=torch.float32, device=self.device)
        self.m = torch.zeros_like(self.grad)
        self.v = torch.zeros_like(self.grad)
        self.step_count = 0
        fm = np.zeros(self.dims[0], np.float32) if fmean is None else np.asarray(fmean, np.float32)
        fs = np.ones(self.dims[0], np.float32) if fstd is None else np.asarray(fstd, np.float32)
        self.fmean = torch.tensor(fm, device=self.device)
        self.fstd = torch.tensor(np.where(fs > 0, fs, 1.0).astype(np.float32), device=self.device)
        self._ws = {}
        self._refresh_bf16()

    @property
    def stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _refresh_bf16(self):
        _lib.check(self.lib.flpr_to_bf16(self.nparams, self.p32.data_ptr(), self.p16.data_ptr(),
                                         self.stream), "flpr_to_bf16")

    def _workspace(self, batch: int) -> torch.Tensor:
        ws = self._ws.get(batch)
        if ws is None:
            nb = int(self.lib.flpr_mlp_ws(self.nl, self._dims_c, batch))
            ws = torch.empty(max(nb, 256), dtype=torch.uint8, device=self.device)
            self._ws = {batch: ws}
        return ws

    def _inputs(self, feats) -> torch.Tensor:
        x = torch.as_tensor(feats, dtype=torch.float32, device=self.device)
        if x.dim() == 1:
            x = x[None, :]
        x = ((x - self.fmean) / self.fstd).contiguous()
        x16 = torch.empty(x.shape, dtype=torch.bfloat16, device=self.device)
        _lib.check(self.lib.flpr_to_bf16(x.numel(), x.data_ptr(), x16.data_ptr(), self.stream),
                   "flpr_to_bf16")
        return x16

    def forward_raw(self, x16: torch.Tensor) -> torch.Tensor:
        """Network output (batch,) for BF16 standardised inputs."""
        B = int(x16.shape[0])
        ws = self._workspace(B)
        out = torch.empty((B, self.dims[-1]), dtype=torch.float32, device=self.device)
        _lib.check(self.lib.flpr_mlp_fwd(self.nl, self._dims_c, self.p16.data_ptr(),
                                         self.p32.data_ptr(), B, x16.data_ptr(), out.data_ptr(),
                                         ws.data_ptr(), ws.numel(), self.stream), "flpr_mlp_fwd")
        return out[:, 0]

    def predict(self, feats) -> np.ndarray:
        """Proposed fractional index on HGRID for each feature row."""
        y = self.forward_raw(self._inputs(feats))
        return (y.cpu().numpy().astype(np.float64) * T_SCALE + T_CENTER)

    def train_step(self, x16: torch.Tensor, target: torch.Tensor, lr: float,
                   weight_decay: float = 0.0) -> torch.Tensor:
        """One Adam step on a batch (x16 BF16 standardised inputs, target in
        network units); returns the batch loss as a device tensor."""
        B = int(x16.shape[0])
        ws = self._workspace(B)
        out = torch.empty((B, 1), dtype=torch.float32, device=self.device)
        _lib.check(self.lib.flpr_mlp_fwd(self.nl, self._dims_c, self.p16.data_ptr(),
                                         self.p32.data_ptr(), B, x16.data_ptr(), out.data_ptr(),
                                         ws.data_ptr(), ws.numel(), self.stream), "flpr_mlp_fwd")
        dout = torch.empty_like(out)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        _lib.check(self.lib.flpr_mlp_mse(B, out.data_ptr(), target.data_ptr(), dout.data_ptr(),
                                         loss.data_ptr(), self.stream), "flpr_mlp_mse")
        _lib.check(self.lib.flpr_mlp_bwd(self.nl, self._dims_c, self.p16.data_ptr(), B,
                                         x16.data_ptr(), dout.data_ptr(), self.grad.data_ptr(),
                                         ws.data_ptr(), ws.numel(), self.stream), "flpr_mlp_bwd")
        self.step_count += 1
        _lib.check(self.lib.flpr_mlp_step(self.nparams, self.p32.data_ptr(), self.p16.data_ptr(),
                                          self.grad.data_ptr(), self.m.data_ptr(),
                                          self.v.data_ptr(), lr, 0.9, 0.999, 1e-8, weight_decay,
                                          self.step_count, self.stream), "flpr_mlp_step")
        return loss

    def save(self, path: str, **extra) -> None:
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez_compressed(path, dims=np.asarray(self.dims), params=self.p32.cpu().numpy(),
                            fmean=self.fmean.cpu().numpy(), fstd=self.fstd.cpu().numpy(),
                            **extra)

    @classmethod
    def load(cls, path: str, device=None) -> "BandwidthMLP":
        z = np.load(path)
        return cls(device=device, dims=[int(v) for v in z["dims"]], params=z["params"],
                   fmean=z["fmean"], fstd=z["fstd"])


_default = {}
_default_lock = threading.Lock()


def default_model(device: torch.device) -> BandwidthMLP:
    """The shipped trained network (cached per device)."""
    key = str(device)
    with _default_lock:
        if key not in _default:
            if not os.path.exists(WEIGHTS_PATH):
                raise FileNotFoundError(
                    f"no trained bandwidth network at {WEIGHTS_PATH}; run "
                    "python -m fastlpr_b200.train_bandwidth_mlp")
            _default[key] = BandwidthMLP.load(WEIGHTS_PATH, device)
        return _default[key]


# ---------------------------------------------------------------- search

def isotropic_log_h(bandwidths: np.ndarray) -> Optional[np.ndarray]:
    """log h per row when every row is isotropic and rows increase strictly;
    None otherwise (the learned search then falls back to the full sweep)."""
    bw = np.asarray(bandwidths, dtype=np.float64)
    if bw.ndim != 2 or bw.shape[0] < REFINE:
        return None
    if bw.shape[1] > 1 and not np.allclose(bw, bw[:, :1], rtol=1e-12, atol=0.0):
        return None
    lh = np.log(bw[:, 0])
    if not np.all(np.diff(lh) > 0):
        return None
    return lh


def refine_window(proposal: float, log_h: np.ndarray) -> np.ndarray:
    """Indices of the REFINE bandwidths of the list nearest to the proposal."""
    lg = np.log(HGRID)
    t = float(np.clip(proposal, 0.0, len(HGRID) - 1))
    i0 = int(np.floor(t))
    i1 = min(i0 + 1, len(HGRID) - 1)
    target = lg[i0] + (t - i0) * (lg[i1] - lg[i0])
    c = int(np.argmin(np.abs(log_h - target)))
    lo = int(np.clip(c - REFINE // 2, 0, len(log_h) - REFINE))
    return np.arange(lo, lo + REFINE)


def accept_window(window: np.ndarray, idmin: int, nlist: int) -> bool:
    """The window's GCV minimum is trusted when it is interior to the window,
    or sits at an end of the whole list."""
    g = int(window[idmin])
    return (0 < idmin < len(window) - 1) or g == 0 or g == nlist - 1


# ---------------------------------------------------------------- device chain

class DeviceProposal:
    """The proposal chain of B data sets on the device, without a host round
    trip: binned sums (filled per data set by ``bin_moments``), feature
    vectors and their standardised BF16 copy (``flpr_learned_features``), the
    network (``flpr_mlp_fwd``, one batch for all data sets) and the window
    start of the local sweep in each data set's own bandwidth list
    (``flpr_learned_window``).  Every buffer lives as long as this object, so
    the chain can be captured in a CUDA graph and replayed."""

    def __init__(self, model: "BandwidthMLP", metas, log_hs, device):
        """metas: (d, order, n) per data set; log_hs: each data set's log
        bandwidths.  The small tables go up with non-blocking copies on the
        current stream (no host wait)."""
        self.lib = _lib.load()
        self.model = model
        self.device = torch.device(device)
        B = len(metas)
        self.B = B
        dev = self.device

        def up(a):
            return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().to(dev, non_blocking=True)

        self.bins = torch.zeros((B, 3, CELLS), dtype=torch.float64, device=dev)
        self.meta = up(np.asarray(metas, dtype=np.int32).reshape(B, 3))
        self.lmax = max(REFINE, max(len(v) for v in log_hs))
        lh = np.zeros((B, self.lmax))
        for i, v in enumerate(log_hs):
            lh[i, :len(v)] = v
        self.logh = up(lh)
        self.nlist = up(np.asarray([len(v) for v in log_hs], dtype=np.int32))
        self.loggrid = up(np.log(HGRID))
        self.x16 = torch.empty((B, model.dims[0]), dtype=torch.bfloat16, device=dev)
        self.out = torch.empty((B, model.dims[-1]), dtype=torch.float32, device=dev)
        self.lo = torch.zeros(B, dtype=torch.int32, device=dev)
        self.t = torch.zeros(B, dtype=torch.float64, device=dev)
        # the fused tensor-core inference kernel when the network's shape
        # allows it (the shipped one does), else the layer-by-layer products
        self.fused = bool(self.lib.flpr_mlp_infer_supported(model.nl, model._dims_c))
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        nb = 0 if self.fused else int(self.lib.flpr_mlp_ws(model.nl, model._dims_c, B))
        self.ws = torch.empty(max(nb, 256), dtype=torch.uint8, device=dev)

    def enqueue(self, stream) -> None:
        """Features, network and window starts of every data set (their
        binned sums must be in ``bins``)."""
        m, lib = self.model, self.lib
        _lib.check(lib.flpr_learned_features(self.B, self.bins.data_ptr(), self.meta.data_ptr(),
                                             m.fmean.data_ptr(), m.fstd.data_ptr(), None,
                                             self.x16.data_ptr(), stream),
                   "flpr_learned_features")
        if self.fused:
            _lib.check(lib.flpr_mlp_infer(m.nl, m._dims_c, m.p16.data_ptr(), m.p32.data_ptr(),
                                          self.B, self.x16.data_ptr(), self.out.data_ptr(),
                                          self.status.data_ptr(), stream), "flpr_mlp_infer")
        else:
            _lib.check(lib.flpr_mlp_fwd(m.nl, m._dims_c, m.p16.data_ptr(), m.p32.data_ptr(),
                                        self.B, self.x16.data_ptr(), self.out.data_ptr(),
                                        self.ws.data_ptr(), self.ws.numel(), stream),
                       "flpr_mlp_fwd")
        _lib.check(lib.flpr_learned_window(self.B, self.out.data_ptr(), T_SCALE, T_CENTER,
                                           len(HGRID), self.loggrid.data_ptr(), self.lmax,
                                           self.nlist.data_ptr(), self.logh.data_ptr(), REFINE,
                                           self.lo.data_ptr(), self.t.data_ptr(), stream),
                   "flpr_learned_window")
