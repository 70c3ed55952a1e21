"""Drop-in ``cv_fastlpr`` / ``cv_fastkde`` on the B200.

The host keeps the reference API (api.py:167-1184 of the reference package):
argument handling, validation, option defaults, bandwidth-candidate
handling, 1-SE selection and output assembly run here in Python on O(H)
scalars.  Everything that touches the N points or the grids runs in the
CUDA library through its C ABI (``_lib``):

  point statistics -> spread {1, y, probes} -> R2C FFT -> per-axis kernel
  spectra -> multiply + C2R + crop (S, T planes) -> FP64 solve ->
  interpolation + GCV/Hutchinson reductions -> final interpolation.
"""
from __future__ import annotations

import copy
import math
import time
import warnings
from types import SimpleNamespace
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib, spline
from .bandwidth import get_hlist
from .interpolant import GridInterpolant
from .structures import KDEOutput, RegressionOutput

SQRT_2PI = math.sqrt(2.0 * math.pi)

# kernel_type names (kernel.py:159-431) -> flpr_kernel_spectra ids; the two
# Gaussians factor over the axes and use the per-axis path
_KERNEL_IDS = {"gaussian": 0, "gauss": 0, "normal": 0, "gaussian_ft": 1, "normal_ft": 1,
               "epan": 2, "epanechnikov": 2, "tricube": 3, "quartic": 4, "biweight": 4,
               "triweight": 5, "uniform": 6, "rectangular": 6}
_SUPPORTED_KERNEL_NAMES = ("gaussian, gauss, normal, gaussian_ft, normal_ft, epanechnikov, epan, "
                           "tricube, quartic, biweight, triweight, uniform, rectangular")


def _kernel_id(opts) -> int:
    kt = str(opts.get("kernel_type", "gaussian")).lower()
    if kt in ("poly", "polynomial"):
        # compute_kernel_fourier passes no options to kernel_function
        raise ValueError('Polynomial kernel requires opt["order"] to be specified')
    if kt not in _KERNEL_IDS:
        raise ValueError(f"Unknown kernel type: {opts.get('kernel_type')}. "
                         f"Supported types: {_SUPPORTED_KERNEL_NAMES}")
    return _KERNEL_IDS[kt]
EPS = float(np.finfo(float).eps)


# ---------------------------------------------------------------------------
# Option handling (reference utils/__init__.py:18-56, helpers.py:31-92)
# ---------------------------------------------------------------------------
def set_defaults(options=None, **kwargs) -> Dict[str, object]:
    result = dict(options) if options is not None else {}
    for k, v in kwargs.items():
        result.setdefault(k, v)
    return result


def _as_column_matrix(x) -> np.ndarray:
    arr = np.asarray(x)
    if arr.ndim == 1:
        arr = arr[:, None]
    if arr.ndim != 2:
        raise ValueError("Input must be a 1D or 2D array.")
    if np.iscomplexobj(arr):
        cc = np.any(arr.imag != 0, axis=0)
        arr = np.column_stack([arr.real, arr.imag[:, cc]]) if np.any(cc) else arr.real
    return arr.astype(float, copy=False)


def _finite_flags(tensors) -> torch.Tensor:
    """Device-side NaN/Inf scan: [any NaN, any Inf] per tensor, in order."""
    out = []
    for t in tensors:
        out.append(torch.isnan(t).any())
        out.append(torch.isinf(t).any())
    return torch.stack(out)


def _raise_nonfinite(flags: np.ndarray, names, fn: str) -> None:
    """ValueError for the first NaN, then Inf, per input (api.py:310-323)."""
    for k, (what, _) in enumerate(names):
        if flags[2 * k]:
            raise ValueError(f"{what} contains NaN values. Please remove or impute NaN values "
                             f"before calling {fn}.")
        if flags[2 * k + 1]:
            raise ValueError(f"{what} contains Inf values. Please remove or handle Inf values "
                             f"before calling {fn}.")


def _default_hrange(points: np.ndarray) -> np.ndarray:
    scale = np.std(points, axis=0, ddof=1)
    scale[scale == 0] = 1.0
    return np.column_stack((0.1 * scale, 1.0 * scale))


def _prepare_bandwidths(h, dims, options, default_range) -> np.ndarray:
    """api.py:32-70.  default_range may be a callable (evaluated only when h is None)."""
    if h is None:
        dh = options.get("dh", None)
        if dh is None:
            dh = 20 if dims == 1 else [20] * dims
        if callable(default_range):
            default_range = default_range()
        bw = get_hlist(dh, default_range)
    else:
        a = np.asarray(h, dtype=float)
        if a.ndim == 0:
            bw = np.full((1, dims), a.item())
        elif a.ndim == 1:
            if a.size != dims:
                raise ValueError("Scalar bandwidth must match the number of dimensions.")
            bw = a.reshape(1, -1)
        else:
            if a.shape[1] != dims:
                raise ValueError(
                    "Bandwidth array must have the same dimensionality as the input data.")
            bw = a.reshape(-1, dims)
    if not np.all(np.isfinite(bw)):
        raise ValueError("Bandwidth values must be finite (no NaN or Inf).")
    if np.any(bw <= 0):
        raise ValueError("Bandwidth values must be strictly positive. "
                         f"Found non-positive values: {bw[bw <= 0]}")
    return bw


def _one_se_rule(scores, errs, bandwidths, prefer_smaller: bool, dstd: float = 1.0) -> int:
    """1-SE bandwidth selection (api.py:73-164)."""
    valid = np.isfinite(scores)
    if not np.any(valid):
        raise ValueError(
            "All GCV scores are NaN or Inf. Regression failed for all bandwidths. "
            "Try: (1) Use larger bandwidth h, (2) Increase grid points, "
            "(3) Check for data quality issues")
    vi = np.where(valid)[0]
    vs, ve = scores[valid], errs[valid]
    if prefer_smaller:
        b = int(np.argmin(vs))
        thr = vs[b] + dstd * ve[b]
        cm = vs <= thr
        ci = vi[cm]
        if len(ci) == 0:
            return int(vi[b])
        sums = np.sum(bandwidths[ci], axis=1)
        tie = np.where(sums == sums.max())[0]
        return int(ci[tie[int(np.argmin(vs[cm][tie]))]])
    b = int(np.argmax(vs))
    thr = vs[b] - dstd * ve[b]
    cm = vs >= thr
    ci = vi[cm]
    if len(ci) == 0:
        return int(vi[b])
    sums = np.sum(bandwidths[ci], axis=1)
    return int(ci[np.argmax(sums)])


# ---------------------------------------------------------------------------
# Device context
# ---------------------------------------------------------------------------
def _device(options) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("fastlpr_b200 needs a CUDA device (no CPU fallback)")
    dev = options.get("device", None) if options else None
    if dev is None:
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device(dev)


class _Ctx:
    """Device, stream, library handle and workspace helpers for one call."""

    def __init__(self, device: torch.device):
        self.device = device
        self.index = device.index if device.index is not None else torch.cuda.current_device()
        self.lib = _lib.load()
        self.handle = _lib.handle(self.index)
        self.stream = torch.cuda.current_stream(device).cuda_stream

    def empty(self, shape, dtype=torch.float64):
        return torch.empty(shape, dtype=dtype, device=self.device)

    def zeros(self, shape, dtype=torch.float64):
        return torch.zeros(shape, dtype=dtype, device=self.device)

    def ws(self, nbytes: int):
        return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=self.device)

    def upload(self, arr: np.ndarray, dtype=torch.float64):
        t = torch.from_numpy(np.ascontiguousarray(arr))
        if t.dtype != dtype:
            t = t.to(dtype)
        if t.numel() * t.element_size() >= _STAGE_MIN_BYTES and not t.is_pinned():
            # a large pageable array: copied into page-locked memory by a few
            # host threads, then uploaded asynchronously (a pageable upload
            # is staged by the driver at a fraction of the link's rate)
            t = _pinned_copy(t)
        # asynchronous from page-locked memory (stream-ordered before every kernel
        # that reads it; the call returns only after the results are on the host;
        # the caching host allocator keeps the pages until the copy is done)
        return t.to(self.device, non_blocking=True)

    def check(self, status: int, what: str):
        _lib.check(status, what)


_STAGE_MIN_BYTES = 4 << 20
_stage_pool = None


def _pinned_copy(t: torch.Tensor) -> torch.Tensor:
    """A page-locked copy of a contiguous CPU tensor, made in chunks by a
    thread pool (numpy's copies release the GIL)."""
    global _stage_pool
    if _stage_pool is None:
        from concurrent.futures import ThreadPoolExecutor
        import os
        _stage_pool = ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1)))
    out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    src, dst = t.numpy().reshape(-1), out.numpy().reshape(-1)
    n = src.size
    step = max(1 << 18, -(-n // _stage_pool._max_workers))
    bounds = [(a, min(n, a + step)) for a in range(0, n, step)]

    def piece(ab):
        np.copyto(dst[ab[0]:ab[1]], src[ab[0]:ab[1]])

    list(_stage_pool.map(piece, bounds))
    return out


def _to_host(t: torch.Tensor) -> torch.Tensor:
    """Asynchronous copy of a device tensor into fresh pinned host memory."""
    out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    out.copy_(t, non_blocking=True)
    return out


class _PhaseEvents:
    """Optional CUDA-event timing of the pipeline phases (milliseconds per
    phase, accumulated into ``timings``)."""

    def __init__(self, timings):
        self.timings = timings
        self.events = []

    def mark(self, name):
        if self.timings is None:
            return
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.events.append((name, e, time.perf_counter()))

    def finish(self):
        if self.timings is None or len(self.events) < 2:
            return
        self.events[-1][1].synchronize()
        for (_, a, ta), (name, b, tb) in zip(self.events[:-1], self.events[1:]):
            self.timings[name] = self.timings.get(name, 0.0) + a.elapsed_time(b)
            key = "host_" + name
            self.timings[key] = self.timings.get(key, 0.0) + 1000.0 * (tb - ta)
        self.events = []


# Probe matrices: MT19937(seed).standard_normal((n, R)) fills the matrix in
# row-major order, so the probes for n points are the first n rows of any
# larger draw.  One (R, n_max) device matrix per (device, R, seed) serves
# every n <= n_max.
_PROBE_CACHE: Dict[Tuple[int, int, int], torch.Tensor] = {}


def _probes(ctx: _Ctx, n: int, R: int, seed, random_matrix) -> Tuple[torch.Tensor, int]:
    """Hutchinson probes p = MT19937(seed).standard_normal((n, R)) as an
    (R, n) float64 device tensor, rows contiguous (regression.py:1182-1194)."""
    if random_matrix is not None:
        p = np.asarray(random_matrix, dtype=float)
        if p.ndim == 1:
            p = p[:, None]
        if p.shape[0] != n:
            raise ValueError(f"random_matrix has wrong shape: expected ({n}, *), got {p.shape}")
        return ctx.upload(np.ascontiguousarray(p.T)), p.shape[1]
    key = (ctx.index, R, int(seed))
    t = _PROBE_CACHE.get(key)
    if t is None or t.shape[1] < n:
        p = np.random.Generator(np.random.MT19937(seed)).standard_normal((n, R))
        t = ctx.upload(np.ascontiguousarray(p.T))
        if len(_PROBE_CACHE) > 8:
            _PROBE_CACHE.clear()
        _PROBE_CACHE[key] = t
    return t[:, :n], R


def clear_fastlpr_caches() -> None:
    """Drop cached probe matrices (the reference's clear_fastlpr_caches)."""
    _PROBE_CACHE.clear()


# ---------------------------------------------------------------------------
# Grid geometry: everything derived on the host from the point statistics
# ---------------------------------------------------------------------------
@dataclass
class _Geom:
    n: int
    d: int
    G: np.ndarray
    L: np.ndarray
    qin: np.ndarray
    qout: np.ndarray
    msp: int
    tau: np.ndarray
    kmap: np.ndarray          # (d, 9), knot spacing 2 pi / L (no oversampling)
    lo: np.ndarray            # scaled kernel grid min (= centred data min)
    hi: np.ndarray
    mean: np.ndarray
    std: np.ndarray
    center: np.ndarray
    xmin: np.ndarray
    xmax: np.ndarray
    accuracy: int = 4

    @property
    def M(self) -> int:
        return int(np.prod(self.G))


def _grid_params(G: np.ndarray, flag_power2: bool):
    """convolution.py:389-409."""
    if flag_power2:
        L = 2 ** np.ceil(np.log2(2 * G - 1)).astype(int)
    else:
        L = G + 2
    qin = np.zeros((2, len(G)), dtype=int)
    qout = np.zeros((2, len(G)), dtype=int)
    qin[0] = (L - G) // 2
    qin[1] = qin[0] + G - 1
    qout[0] = np.ceil((L - G) / 2).astype(int)
    qout[1] = qout[0] + G - 1
    return L, qin, qout


def _point_stats_dev(ctx: _Ctx, dx: torch.Tensor, n: int, d: int) -> torch.Tensor:
    """(4 d) device statistics: minimum, maximum, mean, M2 per axis."""
    out = ctx.empty(4 * d)
    ws = ctx.ws(ctx.lib.flpr_point_stats_ws(d, n))
    ctx.check(ctx.lib.flpr_point_stats(d, n, dx.data_ptr(), out.data_ptr(), ws.data_ptr(),
                                       ws.numel(), ctx.stream), "flpr_point_stats")
    return out


def _point_stats(ctx: _Ctx, dx: torch.Tensor, n: int, d: int) -> np.ndarray:
    return _point_stats_dev(ctx, dx, n, d).cpu().numpy().reshape(4, d)


def _knot_consts(G: np.ndarray, L: np.ndarray, qin: np.ndarray):
    """Per-axis constants of the knot mapping that depend on the grid only:
    the knot range ks and start r0 of convolution.py:190-208 and the knot
    spacing hx = 2 pi / L."""
    d = len(G)
    ks, r0, hx = np.empty(d), np.empty(d), np.empty(d)
    for a in range(d):
        idx_range = np.linspace(-0.5, 0.5 - 1 / L[a], L[a])
        if G[a] != L[a]:
            ks[a] = idx_range[qin[1, a]] - idx_range[qin[0, a]]
            r0[a] = idx_range[qin[0, a]]
        else:
            ks[a] = idx_range[-1] - idx_range[0]
            r0[a] = -0.5
        hx[a] = 2 * np.pi / L[a]
    return ks, r0, hx


def _make_geom(stats: np.ndarray, n: int, d: int, G: np.ndarray, accuracy: int,
               flag_power2: bool) -> _Geom:
    xmin, xmax, mean, m2 = stats[0].copy(), stats[1].copy(), stats[2].copy(), stats[3].copy()
    std = np.sqrt(m2 / (n - 1)) if n > 1 else np.full(d, np.nan)
    std[std == 0] = 1.0
    xs_min = (xmin - mean) / std                        # model.py:58-68
    xs_max = (xmax - mean) / std
    center = (xs_max + xs_min) / 2
    lo = xs_min - center
    hi = xs_max - center
    L, qin, qout = _grid_params(G, flag_power2)
    kmap = np.zeros((d, 9))
    ks_all, r0_all, hx_all = _knot_consts(G, L, qin)       # convolution.py:190-208
    for a in range(d):
        scale = hi[a] - lo[a]
        if scale == 0:
            scale = 1.0
        ks, r0 = ks_all[a], r0_all[a]

        def chain(v):
            xn = (np.float64(v) - lo[a]) / scale * ks + r0
            xn = xn + 0.5
            xn = np.mod(xn, 1.0)
            return xn - 0.5

        kmin = (chain(lo[a]) + chain(hi[a])) * 0.5 - 0.5       # nufftn_type1.py:164-166
        shift = -0.5 - kmin
        hx = 2 * np.pi / L[a]
        kmap[a] = [mean[a], std[a], center[a], lo[a], scale, ks, r0, shift, hx]
    msp, tau, _, _ = _spread_params(L, kmap, accuracy)
    return _Geom(n=n, d=d, G=G, L=L, qin=qin, qout=qout, msp=msp, tau=tau, kmap=kmap, lo=lo,
                 hi=hi, mean=mean, std=std, center=center, xmin=xmin, xmax=xmax,
                 accuracy=int(accuracy))


def _design_powers(d: int, order: int) -> List[Tuple[int, ...]]:
    """Polynomial term exponents (design_matrix_optimized.py:30-76)."""
    if order == 0:
        return [(0,) * d]
    out = []
    for tot in range(order + 1):
        if d == 1:
            out.append((tot,))
        elif d == 2:
            for px in range(tot, -1, -1):
                out.append((px, tot - px))
        else:
            for px in range(tot, -1, -1):
                for py in range(tot - px, -1, -1):
                    out.append((px, py, tot - px - py))
    return out


def _element_powers(d: int, order: int) -> List[Tuple[int, ...]]:
    """Exponents of every packed S element (column-major lower triangle)."""
    pw = _design_powers(d, order)
    if order == 0:
        return pw
    nt = len(pw)
    return [tuple(a + b for a, b in zip(pw[i], pw[j])) for j in range(nt) for i in range(j, nt)]


def _kernel_factors(ctx: _Ctx, geom: _Geom, bw: np.ndarray, npow: int):
    """Per-axis kernel spectra F and the a=0 grid sums (convolution.py:318-652)."""
    H = bw.shape[0]
    d = geom.d
    dh = ctx.upload(np.ascontiguousarray(bw))
    nF = int(sum(H * npow * int(geom.L[a]) for a in range(d)))
    F = ctx.empty((nF, 2))
    sum0 = ctx.empty((d, H))
    ws = ctx.ws(ctx.lib.flpr_kernel_factors_ws(ctx.handle, d, _lib.ivec(geom.L), H, npow))
    ctx.check(ctx.lib.flpr_kernel_factors(ctx.handle, d, _lib.ivec(geom.G), _lib.ivec(geom.L),
                                          _lib.dvec(geom.lo), _lib.dvec(geom.hi), H,
                                          dh.data_ptr(), npow, F.data_ptr(), sum0.data_ptr(),
                                          ws.data_ptr(), ws.numel(), ctx.stream),
              "flpr_kernel_factors")
    return F, sum0


def _kernel_sums_host(geom: _Geom, bw: np.ndarray) -> np.ndarray:
    """(d, H) grid sums of the order-0 kernel factor exp(-u^2/2)/h on
    linspace(lo, hi, G) per axis: the same values flpr_kernel_factors returns
    in d_sum0, formed on the host so the filter needs no device round trip."""
    out = np.empty((geom.d, bw.shape[0]))
    for a in range(geom.d):
        G = int(geom.G[a])
        g = np.linspace(geom.lo[a], geom.hi[a], G)
        u = g[None, :] / bw[:, a:a + 1]
        out[a] = np.sum(np.exp(-0.5 * (u * u)) / bw[:, a:a + 1], axis=1)
    return out


def _separable_kernel_sums(geom: _Geom, bw: np.ndarray, norm: float) -> np.ndarray:
    """Per-bandwidth kernel sums for the "too small bandwidth" test
    (convolution.py:542-605), exact where the test is close: every term of
    the positive grid sums is at most their total, so where the product of
    the largest terms already clears twice the threshold (10 eps) the
    bandwidth stays and that product stands in for the sum; only the others
    get the exact sums."""
    peak = np.ones(bw.shape[0])
    for a in range(geom.d):
        g = np.linspace(geom.lo[a], geom.hi[a], int(geom.G[a]))
        u = np.min(np.abs(g)) / bw[:, a]
        peak = peak * (np.exp(-0.5 * (u * u)) / bw[:, a])
    sums = peak / norm
    low = np.where(sums < EPS * 20)[0]
    if len(low):
        sums[low] = np.prod(_kernel_sums_host(geom, bw[low]), axis=0) / norm
    return sums


class _Kernel:
    """Kernel spectra of one bandwidth list: per-axis factors F (Gaussian
    kernels, flpr_kernel_factors) or full-plane spectra K of every moment
    element (radial kernels, flpr_kernel_spectra), with the inverse-FFT scale
    of the convolutions that use them."""

    def __init__(self, kid: int, data: torch.Tensor, H: int, npow: int, scale: float,
                 elems: Optional[Dict[Tuple[int, ...], int]] = None):
        self.kid, self.data, self.H, self.npow, self.scale = kid, data, H, npow, scale
        self.elems = elems

    @property
    def separable(self) -> bool:
        return self.elems is None

    def data_ptr(self) -> int:
        return self.data.data_ptr()


def _kernel_spectra_full(ctx, geom, bw, powers, kid):
    """(len(powers), H, half) complex128 spectra of the radial kernel's
    moment planes (convolution.py:318-652 with kernel.py:159-431)."""
    H, d = bw.shape[0], geom.d
    L = geom.L
    half = int(np.prod(L[:-1])) * (int(L[-1]) // 2 + 1)
    dh = ctx.upload(np.ascontiguousarray(bw))
    K = ctx.empty((len(powers), H, half, 2))
    nitems = len(powers) * H
    ws = ctx.ws(ctx.lib.flpr_kernel_spectra_ws(ctx.handle, d, _lib.ivec(L), nitems))
    ctx.check(ctx.lib.flpr_kernel_spectra(ctx.handle, d, _lib.ivec(geom.G), _lib.ivec(L),
                                          _lib.dvec(geom.lo), _lib.dvec(geom.hi), kid, H,
                                          dh.data_ptr(), len(powers),
                                          _lib.ivec([v for p in powers for v in p]),
                                          K.data_ptr(), ws.data_ptr(), ws.numel(), ctx.stream),
              "flpr_kernel_spectra")
    return K


def _make_kernel(ctx, geom, bw, npow, kid) -> Tuple[_Kernel, Optional[np.ndarray]]:
    """Kernel spectra for bw; for radial kernels also the order-0 plane sums
    (the DC terms of their spectra), else None."""
    Lprod = float(np.prod(geom.L.astype(float)))
    if kid in (0, 1):
        F, _ = _kernel_factors(ctx, geom, bw, npow)
        scale = (1.0 / SQRT_2PI if kid == 0 else 1.0) / Lprod
        return _Kernel(kid, F, bw.shape[0], npow, scale), None
    powers = _element_powers(geom.d, (npow - 1) // 2)
    uniq = sorted(set(powers), key=powers.index)
    K = _kernel_spectra_full(ctx, geom, bw, uniq, kid)
    sums = K[uniq.index((0,) * geom.d), :, 0, 0].cpu().numpy()
    return _Kernel(kid, K, bw.shape[0], npow, 1.0 / Lprod, {p: i for i, p in enumerate(uniq)}), sums


def _filter_bandwidths(ctx, geom, bw, npow, kid: int = 0):
    """Kernel spectra with the "too small bandwidth" filter of convolution.py:542-605."""
    kern, sums = _make_kernel(ctx, geom, bw, npow, kid)
    if sums is None:
        sums = _separable_kernel_sums(geom, bw, SQRT_2PI if kid == 0 else 1.0)
    ihbad = np.abs(sums) < EPS * 10
    keep = np.where(~ihbad)[0]
    if np.any(ihbad) and not np.all(ihbad):
        warnings.warn(f"{int(np.sum(ihbad))} bandwidth(s) are too small for this grid and "
                      "will be removed", stacklevel=3)
        bw = bw[keep]
        kern, _ = _make_kernel(ctx, geom, bw, npow, kid)
        keep = np.arange(bw.shape[0])
    elif np.all(ihbad):
        d = geom.d
        hs = (4.0 / (d + 2) / geom.n) ** (1.0 / (d + 4))
        warnings.warn(f"All bandwidths too small. Using Silverman's rule: h = {hs:.4f}",
                      stacklevel=3)
        bw = np.array([[hs] * d])
        kern, _ = _make_kernel(ctx, geom, bw, npow, kid)
        keep = np.array([0])
        ihbad = np.array([False])
    return kern, bw, keep, ihbad


def _spread_params(L: np.ndarray, kmap: np.ndarray, accuracy: int):
    """(msp, tau (d,), ratio, kmap) of the spreading at one accuracy
    (kernel.py:97-156): ratio 1/2/3 for accuracy <= 6 / <= 11 / above, Msp =
    accuracy taps, tau = pi Msp / (L^2 ratio (ratio - 1/2)); accuracy 0 is
    nearest-bin binning (nufftn_type1.py:442-516): one tap of weight 1, given
    to the kernel as Msp = 0 with an infinite tau.  The knot grid spacing is
    2 pi / (ratio L)."""
    ratio = 1 if accuracy <= 6 else (2 if accuracy <= 11 else 3)
    msp = int(accuracy)
    if accuracy == 0:
        tau = np.full(len(L), np.inf)
    else:
        tau = (np.pi * msp) / (L * L * ratio * (ratio - 0.5))
    if kmap is not None:
        kmap = kmap.copy()
        kmap[:, 8] = 2 * np.pi / (ratio * np.asarray(L, dtype=float))
    return msp, tau, ratio, kmap


def _spread_fft(ctx: _Ctx, geom: _Geom, dx: torch.Tensor, cols: List[torch.Tensor], prec: int,
                ev=None, accuracy: Optional[int] = None, ones: bool = True,
                kmap_dev: Optional[torch.Tensor] = None, keep: Optional[dict] = None):
    """Spread {1 (if ones), cols...} at `accuracy` and transform: returns the
    (C, L.., L_last/2+1) spectra.  Oversampled accuracies spread on the
    ratio*L grid and keep its central deconvolved L frequencies.  kmap_dev:
    the knot maps on the device (flpr_knot_map; accuracy <= 6 only), in
    which case `geom` needs only d, n, L and accuracy.  keep (a dict, FP32
    without oversampling): receives the spread workspace and its arguments,
    from which _grid64 forms the exact FP64 grid later."""
    d, n = geom.d, geom.n
    acc = geom.accuracy if accuracy is None else int(accuracy)
    msp, tau, ratio, kmap = _spread_params(geom.L, None if kmap_dev is not None else geom.kmap,
                                           acc)
    Lsp = (geom.L * ratio).astype(int)
    C = (1 if ones else 0) + len(cols)
    cells = int(np.prod(Lsp))
    real_dt = torch.float32 if prec == _lib.FLPR_PREC_F32 else torch.float64
    grid = ctx.empty((C, cells), dtype=real_dt)
    ws = ctx.ws(ctx.lib.flpr_spread_ws(d, n, _lib.ivec(Lsp), msp, C, prec))
    chans = _lib.pvec([c.data_ptr() for c in cols])
    if kmap_dev is not None:
        if ratio != 1:
            raise ValueError("device knot maps serve accuracies up to 6")
        hx = 2 * np.pi / (ratio * np.asarray(geom.L, dtype=float))
        ctx.check(ctx.lib.flpr_spread_dkmap(d, n, dx.data_ptr(), kmap_dev.data_ptr(),
                                            _lib.dvec(hx), _lib.ivec(Lsp), msp, _lib.dvec(tau),
                                            C, 1 if ones else 0, chans, grid.data_ptr(), prec,
                                            ws.data_ptr(), ws.numel(), ctx.stream),
                  "flpr_spread_dkmap")
    else:
        ctx.check(ctx.lib.flpr_spread(d, n, dx.data_ptr(), _lib.dvec(kmap.ravel()),
                                      _lib.ivec(Lsp), msp, _lib.dvec(tau), C, 1 if ones else 0,
                                      chans, grid.data_ptr(), prec, ws.data_ptr(), ws.numel(),
                                      ctx.stream), "flpr_spread")
    if keep is not None and ratio == 1:
        keep.update(ws=ws, d=d, n=n, L=Lsp.copy(), msp=msp, C=C, prec=prec)
    del ws
    if ev is not None:
        ev.mark("spread")
    half = cells // int(Lsp[-1]) * (int(Lsp[-1]) // 2 + 1)
    spec = ctx.empty((C, half, 2), dtype=real_dt)
    ws = ctx.ws(ctx.lib.flpr_forward_fft_ws(ctx.handle, d, _lib.ivec(Lsp), C, prec))
    ctx.check(ctx.lib.flpr_forward_fft(ctx.handle, d, _lib.ivec(Lsp), C, grid.data_ptr(),
                                       spec.data_ptr(), prec, ws.data_ptr(), ws.numel(),
                                       ctx.stream), "flpr_forward_fft")
    if ratio > 1:
        del grid, ws
        Lc = int(np.prod(geom.L))
        half_o = Lc // int(geom.L[-1]) * (int(geom.L[-1]) // 2 + 1)
        out = ctx.empty((C, half_o, 2), dtype=real_dt)
        ctx.check(ctx.lib.flpr_oversample_crop(d, _lib.ivec(geom.L), _lib.ivec(Lsp), C,
                                               _lib.dvec(tau), ratio, spec.data_ptr(),
                                               out.data_ptr(), prec, ctx.stream),
                  "flpr_oversample_crop")
        spec = out
    if ev is not None:
        ev.mark("fft")
    return spec


def _node0_cells(geom) -> List[int]:
    """Spreading cell of raw-grid node 0 per axis (where x = min lands: the
    knot map at xs = lo), the window hint of flpr_deposit_sorted."""
    out = []
    for a in range(geom.d):
        _, _, _, _, _, _, r0, shift, hx = geom.kmap[a]
        xn = np.mod(r0 + 0.5, 1.0) - 0.5
        k = np.mod((xn + shift) * (2 * np.pi), 2 * np.pi)
        out.append(int(np.rint(k / hx)) % int(geom.L[a]))
    return out


def _grid64(ctx: _Ctx, kept: dict, nout: Optional[int] = None) -> torch.Tensor:
    """(nout, cells) FP64 grid of the first nout channels (default all) from
    the exact fixed-point sums of an FP32 spread (flpr_spread_grid64_channels;
    `kept` from _spread_fft)."""
    cells = int(np.prod(kept["L"]))
    nout = kept["C"] if nout is None else int(nout)
    out = ctx.empty((nout, cells))
    ws = kept["ws"]
    ctx.check(ctx.lib.flpr_spread_grid64_channels(kept["d"], kept["n"], _lib.ivec(kept["L"]),
                                                  kept["msp"], kept["C"], nout, ws.data_ptr(),
                                                  ws.numel(), out.data_ptr(), ctx.stream),
              "flpr_spread_grid64_channels")
    return out


def _spectra64(ctx: _Ctx, st) -> torch.Tensor:
    """FP64 spectra of every channel (D2Z of the FP64 grid), formed once."""
    if getattr(st, "spec64", None) is None:
        geom, d = st.geom, st.geom.d
        cells = int(np.prod(geom.L))
        half = cells // int(geom.L[-1]) * (int(geom.L[-1]) // 2 + 1)
        C = st.grid64.shape[0]
        spec = ctx.empty((C, half, 2))
        ws = ctx.ws(ctx.lib.flpr_forward_fft_ws(ctx.handle, d, _lib.ivec(geom.L), C,
                                                _lib.FLPR_PREC_F64))
        ctx.check(ctx.lib.flpr_forward_fft(ctx.handle, d, _lib.ivec(geom.L), C,
                                           st.grid64.data_ptr(), spec.data_ptr(),
                                           _lib.FLPR_PREC_F64, ws.data_ptr(), ws.numel(),
                                           ctx.stream), "flpr_forward_fft")
        st.spec64 = spec
    return st.spec64


# Bandwidths whose kernel covers fewer data points than this (n times the
# kernel's +-h box over the data box) are evaluated with FP64 planes on the
# FP32 path: there the local moment matrices are nearly empty and FP32 planes
# carry relative errors far above 1e-5.
SPARSE_POINTS = 4.0


def _sparse_bandwidths(geom, n: int, bw: np.ndarray) -> np.ndarray:
    """Per bandwidth row: does its kernel cover fewer than SPARSE_POINTS points?"""
    span = np.maximum(np.asarray(geom.hi, float) - np.asarray(geom.lo, float), 1e-300)
    frac = np.minimum(1.0, 2.0 * np.asarray(bw, float) / span[None, :])
    return n * np.prod(frac, axis=1) < SPARSE_POINTS


# 2-D separable kernels take the two-pass convolution unless this is set
# (the full 2-D inverse per product, kept for comparison)
_CONV_FULL_2D = False


def _conv(ctx: _Ctx, geom: _Geom, spec, kern: _Kernel, prods, prec: int, add_eps: bool):
    """Planes for a product list [(chan, hidx, pow tuple)] -> (nprod, M)."""
    d = geom.d
    nprod = len(prods)
    real_dt = torch.float32 if prec == _lib.FLPR_PREC_F32 else torch.float64
    out = ctx.empty((nprod, geom.M), dtype=real_dt)
    chan = [p[0] for p in prods]
    if kern.separable and d == 2 and not _CONV_FULL_2D:
        hidx = [p[1] for p in prods]
        pw = [v for p in prods for v in p[2]]
        ws = ctx.ws(ctx.lib.flpr_conv2d_sep_ws(ctx.handle, _lib.ivec(geom.G), _lib.ivec(geom.L),
                                               nprod, prec))
        ctx.check(ctx.lib.flpr_conv2d_sep(ctx.handle, _lib.ivec(geom.G), _lib.ivec(geom.L),
                                          _lib.ivec(geom.qout[0]), kern.H, kern.npow,
                                          spec.data_ptr(), kern.data_ptr(), nprod,
                                          _lib.ivec(chan), _lib.ivec(hidx), _lib.ivec(pw),
                                          kern.scale, 1 if add_eps else 0, out.data_ptr(), prec,
                                          ws.data_ptr(), ws.numel(), ctx.stream),
                  "flpr_conv2d_sep")
        return out
    ws = ctx.ws(ctx.lib.flpr_conv_ws(ctx.handle, d, _lib.ivec(geom.L), nprod, prec))
    if kern.separable:
        hidx = [p[1] for p in prods]
        pw = [v for p in prods for v in p[2]]
        ctx.check(ctx.lib.flpr_conv(ctx.handle, d, _lib.ivec(geom.G), _lib.ivec(geom.L),
                                    _lib.ivec(geom.qout[0]), kern.H, kern.npow, spec.data_ptr(),
                                    kern.data_ptr(), nprod, _lib.ivec(chan), _lib.ivec(hidx),
                                    _lib.ivec(pw), kern.scale, 1 if add_eps else 0,
                                    out.data_ptr(), prec, ws.data_ptr(), ws.numel(), ctx.stream),
                  "flpr_conv")
    else:
        kidx = [kern.elems[tuple(p[2])] * kern.H + int(p[1]) for p in prods]
        ctx.check(ctx.lib.flpr_conv_full(ctx.handle, d, _lib.ivec(geom.G), _lib.ivec(geom.L),
                                         _lib.ivec(geom.qout[0]), len(kern.elems) * kern.H,
                                         spec.data_ptr(), kern.data_ptr(), nprod,
                                         _lib.ivec(chan), _lib.ivec(kidx), kern.scale,
                                         1 if add_eps else 0, out.data_ptr(), prec,
                                         ws.data_ptr(), ws.numel(), ctx.stream), "flpr_conv_full")
    return out


def _conv_s(ctx: _Ctx, geom: _Geom, spec, kern: _Kernel, hks, epw, prec: int,
            add_eps: bool) -> torch.Tensor:
    """The moment planes S of the ones channel for the bandwidth rows `hks`
    and every element power in `epw` -> (len(epw) * len(hks), M), element
    major.  Elements with the same power (order 2: 21 elements, 15 powers)
    are convolved once and their planes repeated."""
    uniq = []
    for e in epw:
        if tuple(e) not in uniq:
            uniq.append(tuple(e))
    H = len(hks)
    out = _conv(ctx, geom, spec, kern, [(0, hk, u) for u in uniq for hk in hks], prec, add_eps)
    if len(uniq) == len(epw):
        return out
    blocks = [out[uniq.index(tuple(e)) * H:(uniq.index(tuple(e)) + 1) * H] for e in epw]
    return torch.cat(blocks, dim=0)


def _precision(opts, dims: Optional[int] = None) -> int:
    p = opts.get("precision", None)
    if p is None:
        # The reference grids are complex64 below accuracy 5 (type_utils.py:158-168).
        # Local-quadratic (order 2) moment systems are ill-conditioned: FP32 S
        # planes lose ~1e-5 in m at the largest bandwidths and ~1e-2 where h
        # approaches the grid spacing.  In 2-D with the full sweep and DoF,
        # order-2 mean fits run the FP32 path with their moment planes in FP64
        # (formed from the exact FP64 grid of the fixed-point spread) and the
        # sparse bandwidths wholly in FP64 (_evaluate_device).  Variance fits
        # return exp(m) of a log response (|m| ~ 5-10), so their relative
        # error is the absolute error of m: FP32 value channels would give
        # ~4e-5; they, and order 2 elsewhere, keep their grids in FP64.
        order = int(opts.get("order", 0))
        if int(opts["accuracy"]) < 5 and (
                order < 2 or (dims == 2 and bool(opts.get("calc_dof", True))
                              and str(opts.get("bandwidth_search", "full")) != "learned"
                              and str(opts.get("y_type_out", "mean")) != "variance")):
            return _lib.FLPR_PREC_F32
        return _lib.FLPR_PREC_F64
    p = str(p).lower()
    if p in ("fp32", "float32", "single"):
        return _lib.FLPR_PREC_F32
    if p in ("fp64", "float64", "double"):
        return _lib.FLPR_PREC_F64
    raise ValueError(f"precision must be 'fp32' or 'fp64', got {p!r}")


def _check_supported(dims: int, opts) -> None:
    if dims > 3:
        raise NotImplementedError(
            f"fastlpr_b200 supports 1-3 predictor dimensions on the GPU; got dx={dims}")
    acc = int(opts["accuracy"])
    if acc < 0 or acc > 12:
        raise NotImplementedError(f"accuracy={acc} is not supported on the GPU (supported: 0-12)")
    _kernel_id(opts)


def _check_interp_methods(opts, dims: int, n: int) -> Dict[str, str]:
    """Interpolation methods of the fit: GCV and DoF default to linear in 1-D
    or with n >= 5000 and to the not-a-knot cubic spline otherwise
    (api.py:594-600, api.py:651-657); the final interpolant defaults to
    linear (api.py:488).  Only 'linear' and 'cubic' are implemented."""
    default = "linear" if (dims == 1 or n >= 5000) else "cubic"
    out = {"gcv": spline.check_method("gcv_interp_method", opts.get("gcv_interp_method", default)),
           "dof": spline.check_method("dof_interp_method", opts.get("dof_interp_method", default)),
           "output": spline.check_method("interp_method", opts.get("interp_method", "linear"))}
    G = _grid_shape(opts, n, dims)
    if "cubic" in out.values() and np.any(G < 4):
        raise ValueError(f"cubic interpolation needs at least 4 grid points per axis, got N={G}")
    return out


def _grid_shape(opts, n, dims) -> np.ndarray:
    N = opts.get("N", None)
    if N is None:
        dn = int(np.ceil(n ** (1.0 / dims)))
        N = dn if dims == 1 else [dn] * dims
    if np.isscalar(N):
        N = [int(N)] * dims
    G = np.array([int(v) for v in N])
    if len(G) != dims:
        raise ValueError(f"options['N'] must have {dims} entries")
    if np.any(G < 2):
        raise ValueError("grid size N must be at least 2 per axis")
    return G


def _raw_axes(geom: _Geom, opts) -> List[np.ndarray]:
    """core.py:64-99: linspace(min, max, G) of the raw data, or opts['xrange']."""
    xr = opts.get("xrange", None)
    if xr is None:
        lo, hi = geom.xmin, geom.xmax
    else:
        r = np.asarray(xr, dtype=float)
        if r.ndim != 2 or r.shape[1] != 2:
            raise ValueError("xrange must be of shape (dims, 2)")
        lo, hi = r[:, 0], r[:, 1]
    return [np.linspace(lo[a], hi[a], int(geom.G[a]), dtype=float) for a in range(geom.d)]


def _axes_arg(axes: Sequence[np.ndarray]) -> List[float]:
    out = []
    for a in axes:
        out += [float(a[0]), float(a[1] - a[0]) if len(a) > 1 else 1.0]
    return out


# ---------------------------------------------------------------------------
# cv_fastlpr
# ---------------------------------------------------------------------------
class _LprSetup:
    """Validated inputs and options of one cv_fastlpr call."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def _lpr_setup(x, y, h, options) -> _LprSetup:
    """Input checks and option defaults of cv_fastlpr (api.py:167-420)."""
    x_arr = _as_column_matrix(x)
    y_arr = np.asarray(y)
    if y_arr.ndim == 1:
        y_arr = y_arr[:, None]
    elif y_arr.ndim == 2:
        if y_arr.shape[0] == 1 and y_arr.shape[1] > 1:
            y_arr = y_arr.T
    else:
        raise ValueError(f"Response y must be 1D or 2D array. Got {y_arr.ndim}D array.")
    dy = y_arr.shape[1]
    if y_arr.shape[0] != x_arr.shape[0]:
        raise ValueError(
            f"Response y must have same number of samples as x. x has {x_arr.shape[0]} samples, "
            f"y has {y_arr.shape[0]} samples.")
    if x_arr.shape[0] == 0:
        raise ValueError("Input x must have at least one sample.")

    opts = set_defaults(options, order=0, regularization=1e-8, num_dof_sample=10,
                        kernel_type="gaussian", y_type_out="mean", calc_dof=True,
                        gcv_selection="first")
    n = x_arr.shape[0]
    if opts.get("accuracy") is None:
        opts["accuracy"] = max(6 - int(np.ceil(np.log10(n))), 4)
    order = int(opts["order"])
    if order not in (0, 1, 2):
        raise ValueError("Polynomial order must be 0, 1, or 2.")
    dims = x_arr.shape[1]
    if dims > 10:
        raise ValueError(f"dx={dims} exceeds maximum supported dimension (10). "
                         "High-dimensional regression suffers from the curse of dimensionality.")
    elif dims > 6:
        warnings.warn(f"dx={dims} is high-dimensional and may cause memory issues. "
                      "Consider dimensionality reduction techniques.", UserWarning)
    bandwidths = _prepare_bandwidths(h, dims, opts, lambda: _default_hrange(x_arr))
    _check_supported(dims, opts)
    if dims == 3 and order == 2:
        raise ValueError("Order 2 not supported for 3D (max order 1)")
    if n < 2:
        raise ValueError("Input x must have at least two samples.")
    y_type_out = str(opts.get("y_type_out", "mean"))
    variance = y_type_out == "variance"
    y_is_complex = bool(np.iscomplexobj(y_arr))
    if variance and y_is_complex:
        raise NotImplementedError("variance mode needs a real response")
    _check_interp_methods(opts, dims, n)
    prec = _precision(opts, dims)
    return _LprSetup(x_arr=x_arr, y_arr=y_arr, dy=dy, bandwidths=bandwidths, opts=opts,
                     order=order, prec=prec, variance=variance, y_is_complex=y_is_complex,
                     n=n, d=dims)


def cv_fastlpr(x, y, h=None, options: Optional[dict] = None) -> RegressionOutput:
    """Local polynomial regression with GCV bandwidth selection (drop-in for the
    reference ``cv_fastlpr``, api.py:167-832).

    Options are the reference's (order, regularization, num_dof_sample,
    kernel_type, y_type_out, calc_dof, gcv_selection, accuracy, N, xrange, dh,
    flag_power2, dstd, random_matrix, dof_seed, interp methods) plus
    ``precision`` ('fp32' | 'fp64'; default follows the reference's dtype
    rule: FP32 grids below accuracy 5), ``device`` and ``bandwidth_search``:
    'full' (default, the reference's sweep of every bandwidth) or 'learned'
    (the trained proposal network picks five neighbouring bandwidths of the
    list; while their GCV minimum sits on an edge of that window the window
    moves that way, at most three times, and otherwise the full sweep runs;
    needs a list of isotropic, increasing bandwidths, a real single response,
    the Gaussian kernel and d <= 2, else the full sweep runs).  ``metadata['bandwidth_search']``
    records what happened.
    """
    su = _lpr_setup(x, y, h, options)
    ctx = _Ctx(_device(su.opts))
    search = str(su.opts.get("bandwidth_search", "full"))
    if search not in ("full", "learned"):
        raise ValueError(f"bandwidth_search must be 'full' or 'learned', got {search!r}")
    with torch.cuda.device(ctx.device):
        model = None
        if search == "learned":
            from . import learned as _learned
            model = _learned.default_model(ctx.device)
        return _fit_lpr(ctx, su.x_arr, su.y_arr, su.dy, su.bandwidths, su.opts, su.order,
                        su.prec, su.variance, su.y_is_complex, timings=su.opts.get("_timings"),
                        learned=model)


def cv_fastlpr_device(x: torch.Tensor, y: torch.Tensor, h=None,
                      options: Optional[dict] = None) -> RegressionOutput:
    """cv_fastlpr for data already resident on the GPU.

    x: (n, d) float64 CUDA tensor, y: (n,) or (n, dy) float64 CUDA tensor
    (real response).  Same options and result as :func:`cv_fastlpr`; the
    host-side NaN/Inf scan of the inputs is skipped.
    """
    if not (isinstance(x, torch.Tensor) and x.is_cuda and isinstance(y, torch.Tensor) and y.is_cuda):
        raise TypeError("cv_fastlpr_device expects CUDA tensors")
    if x.dim() == 1:
        x = x[:, None]
    if y.dim() == 1:
        y = y[:, None]
    x = x.to(torch.float64).contiguous()
    y = y.to(torch.float64)
    n, dims = x.shape
    if y.shape[0] != n:
        raise ValueError("Response y must have same number of samples as x.")
    opts = set_defaults(options, order=0, regularization=1e-8, num_dof_sample=10,
                        kernel_type="gaussian", y_type_out="mean", calc_dof=True,
                        gcv_selection="first")
    if opts.get("accuracy") is None:
        opts["accuracy"] = max(6 - int(np.ceil(np.log10(n))), 4)
    order = int(opts["order"])
    if order not in (0, 1, 2):
        raise ValueError("Polynomial order must be 0, 1, or 2.")
    if h is None:
        raise ValueError("cv_fastlpr_device needs explicit bandwidths")
    bandwidths = _prepare_bandwidths(h, dims, opts, None)
    _check_supported(dims, opts)
    if str(opts.get("y_type_out", "mean")) == "variance":
        raise NotImplementedError("variance mode: use cv_fastlpr")
    prec = _precision(opts, dims)
    ctx = _Ctx(x.device)
    search = str(opts.get("bandwidth_search", "full"))
    if search not in ("full", "learned"):
        raise ValueError(f"bandwidth_search must be 'full' or 'learned', got {search!r}")
    with torch.cuda.device(ctx.device):
        model = None
        if search == "learned":
            from . import learned as _learned
            model = _learned.default_model(ctx.device)
        ycols = [y[:, c].contiguous() for c in range(y.shape[1])]
        return _fit_lpr(ctx, None, None, y.shape[1], bandwidths, opts, order, prec, False, False,
                        dev_inputs=(x, ycols), timings=opts.get("_timings"), learned=model)


class _LprState:
    """Bandwidth-independent part of one LPR fit: the data on the device, the
    grid geometry, the probes, the spectra of every channel and (dual form)
    the adjoint deposits."""


def _prepare_lpr(ctx, x_arr, y_arr, dy, opts, order, prec, variance, y_is_complex,
                 dev_inputs, ev, hook=None, stats=None, probes=None,
                 bandwidths: Optional[np.ndarray] = None) -> _LprState:
    """Bandwidth-independent stage.  `hook(dx, ycols, stats, n, d, d_stats=None)`
    runs once the point statistics exist, before the spread is enqueued (the
    learned search enqueues its data summary there, ahead of the spread); on the
    path whose knot maps are formed on the device it gets the device
    statistics (d_stats: minima then maxima) instead of the host ones.  With `stats` (the
    point statistics of these device inputs, already checked) nothing here
    waits for the device, so the stage can be captured in a CUDA graph
    (`probes`: the (tensor, R) of _probes for these points, formed earlier).
    `bandwidths`: the list the fit will evaluate; on the FP32 path, when
    some of them cover few points (_sparse_bandwidths), the exact FP64 grid
    of the spread is kept for their FP64 planes."""
    lib = ctx.lib
    st = _LprState()
    kept = {}
    if dev_inputs is not None:
        dx, ycols = dev_inputs
        n, d = dx.shape
    else:
        n, d = x_arr.shape
        dx = ctx.upload(x_arr)
        # response channels (real, or real/imag interleaved per column), (n,) each
        ycols = []
        for c in range(dy):
            col = y_arr[:, c]
            if y_is_complex:
                ycols.append(ctx.upload(np.ascontiguousarray(col.real, dtype=float)))
                ycols.append(ctx.upload(np.ascontiguousarray(col.imag, dtype=float)))
            else:
                ycols.append(ctx.upload(np.ascontiguousarray(col, dtype=float)))
    y_raw_dev = None
    flags_h = None
    if dev_inputs is None and stats is None:
        # NaN/Inf checks of the inputs (api.py:310-323) run on the device; the
        # flags come back with the point statistics' synchronisation
        flags_h = _to_host(_finite_flags([dx, torch.stack(ycols)]))
    ev.mark("upload")
    if variance:
        y_raw_dev = ycols[0]
        ylog = ctx.empty(n)
        ctx.check(lib.flpr_log_shift(n, y_raw_dev.data_ptr(), 1.0 / n, ylog.data_ptr(),
                                     ctx.stream), "flpr_log_shift")
        ycols = [ylog]
    ny = len(ycols)
    G = _grid_shape(opts, n, d)
    accuracy = int(opts["accuracy"])
    flag_power2 = bool(opts.get("flag_power2", True))
    calc_dof = bool(opts.get("calc_dof", True))
    if calc_dof:
        if probes is None:
            probes = _probes(ctx, n, int(opts.get("num_dof_sample", 10)),
                             opts.get("dof_seed", 42), opts.get("random_matrix", None))
        ptens, R = probes
        pcols = [ptens[r] for r in range(R)]
    else:
        R = 0
        pcols = []
    # The user's accuracy applies to the response channels only (their
    # transform in nufft_regression_with_precomputed_kdf, api.py:640); the
    # design planes (compute_design_matrix, api.py:571) and the probes
    # (estimate_dof_nufft_vectorized, regression.py:756) use the default.
    acc_default = max(6 - int(np.ceil(np.log10(n))), 4)
    spec = None
    if stats is None and accuracy == acc_default and accuracy <= 6:
        # one spread at the default accuracy: its knot maps are formed on the
        # device from the statistics, so the spread and the transform are
        # enqueued before the statistics reach the host (the host geometry
        # below repeats the same arithmetic)
        st_dev = _point_stats_dev(ctx, dx, n, d)
        st_host = _to_host(st_dev)
        st_ready = torch.cuda.Event()
        st_ready.record()
        L, qin, _ = _grid_params(G, flag_power2)
        ks, r0, hx = _knot_consts(G, L, qin)
        kmap_dev = ctx.empty(9 * d)
        ctx.check(lib.flpr_knot_map(d, n, st_dev.data_ptr(), _lib.dvec(ks), _lib.dvec(r0),
                                    _lib.dvec(hx), kmap_dev.data_ptr(), ctx.stream),
                  "flpr_knot_map")
        if hook is not None:
            hook(dx, ycols, None, n, d, d_stats=st_dev[:2 * d])
        pre = SimpleNamespace(n=n, d=d, L=L, accuracy=accuracy, kmap=None)
        spec = _spread_fft(ctx, pre, dx, ycols + pcols, prec, ev, kmap_dev=kmap_dev, keep=kept)
        st_ready.synchronize()
        stats = st_host.numpy().reshape(4, d)
    elif stats is None:
        stats = _point_stats(ctx, dx, n, d)
    if flags_h is not None:
        _raise_nonfinite(flags_h.numpy(), [("Input x", 0), ("Response y", 1)], "cv_fastlpr")
    geom = _make_geom(stats, n, d, G, accuracy, flag_power2)
    ev.mark("setup")
    if spec is None:
        if hook is not None:
            hook(dx, ycols, stats, n, d)
        if geom.accuracy == acc_default:
            spec = _spread_fft(ctx, geom, dx, ycols + pcols, prec, ev, keep=kept)
        else:
            spec_s = _spread_fft(ctx, geom, dx, pcols, prec, ev, accuracy=acc_default, ones=True)
            spec_y = _spread_fft(ctx, geom, dx, ycols, prec, ev, accuracy=geom.accuracy,
                                 ones=False)
            spec = torch.cat([spec_s[:1], spec_y, spec_s[1:]], dim=0)
            del spec_s, spec_y
    axes_raw = _raw_axes(geom, opts)
    methods = _check_interp_methods(opts, d, n)
    st.grid64 = None
    st.spec64 = None
    st.__dict__.update(dict(
        n=n, d=d, dx=dx, ycols=ycols, pcols=pcols, R=R, ny=ny, y_raw_dev=y_raw_dev,
        stats=stats, geom=geom, spec=spec, calc_dof=calc_dof, order=order, prec=prec,
        dy=dy, variance=variance, y_is_complex=y_is_complex, opts=opts,
        axes_raw=axes_raw, ax_arg=_lib.dvec(_axes_arg(axes_raw)), G_arg=_lib.ivec(geom.G),
        methods=methods, spl=None, kid=_kernel_id(opts),
        dual=(calc_dof and ny <= 4 and not opts.get("_direct_reduce", False)
              and methods["gcv"] == "linear" and methods["dof"] == "linear"), Q=None))
    if kept and kept["prec"] == _lib.FLPR_PREC_F32 and bandwidths is not None:
        sparse_any = bool(np.any(_sparse_bandwidths(geom, n, bandwidths)))
        if order == 2 or sparse_any:
            # the exact FP64 grid for FP64 planes; the ones channel alone
            # when only the order-2 moment planes need it (_evaluate_device)
            Lq = (_lib.ivec(geom.G), _lib.ivec(geom.L), _lib.ivec(geom.qout[0]))
            ones_only = (order == 2 and not sparse_any and d == 2 and st.dual
                         and st.kid in (0, 1) and not opts.get("_no_fused", False)
                         and lib.flpr_lpr2d_fused_supported(*Lq, 1, 2, ny + R) == 1)
            st.grid64 = _grid64(ctx, kept, 1 if ones_only else None)
    if "cubic" in methods.values():
        st.spl = spline.tables(axes_raw, ctx.device)
    if st.dual:
        # dual form: grid-domain dot products with the adjoint deposits
        M = geom.M
        Cv = ny + R
        npair = (2 ** d) * (2 ** d + 1) // 2
        st.Q = ctx.empty((M, Cv))
        st.Bst = ctx.empty((M, npair))
        st.sq = ctx.empty(Cv)
        if kept and d <= 2 and kept["C"] == 1 + Cv:
            # from the spread's tile-sorted records: exact and order-free
            ws2 = ctx.ws(lib.flpr_deposit_sorted_ws(d, n, _lib.ivec(kept["L"]), kept["msp"],
                                                    kept["C"]))
            ctx.check(lib.flpr_deposit_sorted(d, n, dx.data_ptr(), _lib.ivec(kept["L"]),
                                              kept["msp"], kept["C"], 1,
                                              _lib.pvec([c.data_ptr() for c in ycols + pcols]),
                                              kept["ws"].data_ptr(),
                                              kept["ws"].numel(), st.ax_arg, st.G_arg,
                                              _lib.ivec(_node0_cells(geom)), st.Q.data_ptr(),
                                              st.Bst.data_ptr(), st.sq.data_ptr(),
                                              ws2.data_ptr(), ws2.numel(), ctx.stream),
                      "flpr_deposit_sorted")
            del ws2
        else:
            ctx.check(lib.flpr_deposit(d, n, dx.data_ptr(), st.ax_arg, st.G_arg, Cv,
                                       _lib.pvec([c.data_ptr() for c in ycols + pcols]),
                                       st.Q.data_ptr(), st.Bst.data_ptr(), st.sq.data_ptr(),
                                       ctx.stream), "flpr_deposit")
        ev.mark("deposit")
    kept.clear()
    return st


def _evaluate_lpr(ctx, st: _LprState, bandwidths: np.ndarray, ev) -> dict:
    """Kernel spectra, convolutions, solves and GCV for one bandwidth list."""
    filt = _filter_bandwidths(ctx, st.geom, bandwidths, 2 * st.order + 1, st.kid)
    r = _evaluate_device(ctx, st, filt, ev)
    return _evaluate_host(st, r, r["packed"].cpu().numpy() if r["packed"] is not None else None)


def _evaluate_device(ctx, st: _LprState, filt, ev) -> dict:
    """Device part of the evaluation: convolutions, solves and the GCV/DoF
    reductions, packed into one device vector (``packed``).  `filt` is the
    result of _filter_bandwidths.  Nothing here waits for the device.

    On the FP32 path, bandwidths whose kernel covers few points
    (_sparse_bandwidths; the FP64 grid was kept for them) get FP64 planes:
    the leading ones of an increasing list as a separate group sharing the
    regularisation of the whole list (_evaluate_split), otherwise the whole
    list in FP64."""
    kern0, bw0, keep0, _ = filt
    if (st.prec == _lib.FLPR_PREC_F32 and getattr(st, "grid64", None) is not None
            and not getattr(kern0, "device_window", False)):
        mask = _sparse_bandwidths(st.geom, st.n, bw0[keep0])
        k64 = int(mask.sum())
        leading = k64 < len(mask) and bool(np.all(mask[:k64]))
        if st.order == 2:
            # moment planes in FP64, value channels on the fused FP32 path
            Lq = (_lib.ivec(st.geom.G), _lib.ivec(st.geom.L), _lib.ivec(st.geom.qout[0]))
            if ((k64 == 0 or leading) and k64 < len(mask) and st.d == 2 and st.dual
                    and kern0.separable and not st.opts.get("_no_fused", False)
                    and ctx.lib.flpr_lpr2d_fused_supported(*Lq, len(mask) - k64, 2,
                                                           st.ny + st.R) == 1):
                return _evaluate_split(ctx, st, filt, k64, ev, s64_all=True)
            # otherwise FP64 throughout
            k64, leading = len(mask), False
        if k64:
            if st.grid64.shape[0] < 1 + st.ny + st.R:
                raise _lib.FastLPRError("the FP64 grid holds only the ones channel but the "
                                        "evaluation needs every channel in FP64")
            if leading and st.dual and kern0.separable:
                return _evaluate_split(ctx, st, filt, k64, ev)
            st64 = copy.copy(st)
            st64.spec = _spectra64(ctx, st)
            st64.prec = _lib.FLPR_PREC_F64
            st64.grid64 = None
            return dict(_evaluate_device(ctx, st64, filt, ev), fp64_bandwidths=len(mask))
    lib = ctx.lib
    d, n, ny, R, order, prec = st.d, st.n, st.ny, st.R, st.order, st.prec
    geom, spec, opts, calc_dof = st.geom, st.spec, st.opts, st.calc_dof
    ycols, pcols = st.ycols, st.pcols
    npow = 2 * order + 1
    kern, bw, keep, _ = filt
    H = len(keep)
    epw = _element_powers(d, order)
    ns = len(epw)
    nt = 1 if order == 0 else len(_design_powers(d, order))
    h_t = list(keep) if calc_dof else [int(keep[0])]
    Ht = len(h_t)
    Cv = ny + R
    M = geom.M
    Lq = (_lib.ivec(geom.G), _lib.ivec(geom.L), _lib.ivec(geom.qout[0]))
    use_fused = st.dual and kern.separable and _fused_ok(ctx, st, prec, H)
    if not use_fused:
        S = _conv_s(ctx, geom, spec, kern, [int(hk) for hk in keep], epw, prec, order == 0)
        ev.mark("conv_S")
        T = _conv(ctx, geom, spec, kern,
                  [(1 + c, int(hk), epw[i]) for i in range(nt) for c in range(Cv) for hk in h_t],
                  prec, False)
        ev.mark("conv_T")
    bw_k = bw[keep]
    scalar = ctx.empty(1)
    reg = float(opts["regularization"])
    # lambda (order >= 1) / max(s) (order 0) is taken over every kept bandwidth;
    # without DoF only the first bandwidth's T is needed.
    if st.dual:
        m = ctx.empty((H, M, ny))
        dots = ctx.empty((Cv, H))
        if use_fused:
            S = ctx.empty((ns, H, M),
                          dtype=torch.float32 if prec == _lib.FLPR_PREC_F32 else torch.float64)
            ws = ctx.ws(lib.flpr_lpr2d_fused_ex_ws(prec, *Lq, H, order, Cv))
            ctx.check(lib.flpr_lpr2d_fused_ex(prec, _FUSED_BOTH, *Lq, H, npow, order, Cv, ny,
                                              spec.data_ptr(), kern.data_ptr(), kern.scale,
                                              st.Q.data_ptr(), reg, S.data_ptr(), None,
                                              m.data_ptr(), dots.data_ptr(), scalar.data_ptr(),
                                              None, ws.data_ptr(), ws.numel(), ctx.stream),
                      "flpr_lpr2d_fused_ex")
            del ws
            ev.mark("conv_solve")
        else:
            ctx.check(lib.flpr_solve_reduce(order, nt, H, H, M, Cv, S.data_ptr(), T.data_ptr(),
                                            reg, ny, m.data_ptr(), st.Q.data_ptr(),
                                            dots.data_ptr(), scalar.data_ptr(), prec,
                                            ctx.stream), "flpr_solve_reduce")
            ev.mark("solve")
        quad = ctx.empty((H, ny))
        _stencil_quad(ctx, st, H, ny, m, quad)
        ev.mark("interp_reduce")
        # one device -> host read for the three reductions
        packed = torch.cat([st.sq.reshape(-1), dots.reshape(-1), quad.reshape(-1)])
        mstride = ny
    else:
        packed = None
        m = ctx.empty((Ht, M, Cv))
        ctx.check(lib.flpr_solve(order, nt, H, Ht, M, Cv, S.data_ptr(), T.data_ptr(), reg,
                                 m.data_ptr(), scalar.data_ptr(), prec, ctx.stream), "flpr_solve")
        ev.mark("solve")
        mstride = Cv
        if calc_dof:
            yptr = _lib.pvec([c.data_ptr() for c in ycols])
            pptr = _lib.pvec([c.data_ptr() for c in pcols])
            red = {}
            for method in sorted(set((st.methods["gcv"], st.methods["dof"]))):
                rss = ctx.empty((H, ny))
                pdot = ctx.empty((max(R, 1), H))
                pp = ctx.empty(max(R, 1))
                if method == "linear":
                    ctx.check(lib.flpr_interp_reduce(d, n, st.dx.data_ptr(), st.ax_arg, st.G_arg,
                                                     H, ny, R, m.data_ptr(), yptr, pptr,
                                                     rss.data_ptr(), pdot.data_ptr(),
                                                     pp.data_ptr(), None, 0, ctx.stream),
                              "flpr_interp_reduce")
                else:
                    # spline coefficients of every fitted grid (H, M, Cv), then
                    # the same reductions through the cubic spline
                    coef = m.clone()
                    ctx.check(lib.flpr_spline_prefilter(d, st.G_arg, Ht, Cv, st.spl.lu.data_ptr(),
                                                        coef.data_ptr(), ctx.stream),
                              "flpr_spline_prefilter")
                    ctx.check(lib.flpr_spline_reduce(d, n, st.dx.data_ptr(),
                                                     st.spl.axes.data_ptr(), st.G_arg, H, ny, R,
                                                     coef.data_ptr(), yptr, pptr, rss.data_ptr(),
                                                     pdot.data_ptr(), pp.data_ptr(), ctx.stream),
                              "flpr_spline_reduce")
                red[method] = (rss, pdot, pp)
            ev.mark("interp_reduce")
            packed = torch.cat([red[st.methods["gcv"]][0].reshape(-1),
                                red[st.methods["dof"]][1].reshape(-1),
                                red[st.methods["dof"]][2].reshape(-1)])
    return dict(keep=keep, bw_k=bw_k, H=H, m=m, S=S, ns=ns, mstride=mstride, packed=packed,
                dual=st.dual)


def _stencil_quad(ctx, st, H: int, ny: int, m: torch.Tensor, quad: torch.Tensor) -> None:
    """sum B m m of the dual form, reduced in a fixed order."""
    lib = ctx.lib
    ws = ctx.ws(lib.flpr_stencil_quad_fixed_ws(st.d, st.G_arg, H, ny))
    ctx.check(lib.flpr_stencil_quad_fixed(st.d, st.G_arg, H, ny, m.data_ptr(), st.Bst.data_ptr(),
                                          quad.data_ptr(), ws.data_ptr(), ws.numel(), ctx.stream),
              "flpr_stencil_quad_fixed")


def _kernel_rows(kern: _Kernel, rows: np.ndarray, geom) -> _Kernel:
    """The per-axis factors of a consecutive subset of a separable kernel's
    bandwidths, sliced on the device (no upload: usable inside a capture)."""
    r0, r1 = int(rows[0]), int(rows[-1]) + 1
    parts, off = [], 0
    for La in geom.L:
        seg = int(kern.H) * kern.npow * int(La)
        parts.append(kern.data[off:off + seg].view(kern.H, kern.npow * int(La), 2)[r0:r1]
                     .reshape(-1, 2))
        off += seg
    if not np.array_equal(np.asarray(rows), np.arange(r0, r1)):
        raise ValueError("kernel rows must be consecutive")
    return _Kernel(kern.kid, torch.cat(parts, dim=0).contiguous(), r1 - r0, kern.npow, kern.scale)


_FUSED_BOTH, _FUSED_S, _FUSED_T = 0, 1, 2


def _fused_ok(ctx, st, prec: int, H: int) -> bool:
    """Whether the fused 2-D passes serve this fit in `prec`."""
    if st.d != 2 or st.opts.get("_no_fused", False) or H < 1:
        return False
    Lq = (_lib.ivec(st.geom.G), _lib.ivec(st.geom.L), _lib.ivec(st.geom.qout[0]))
    return ctx.lib.flpr_lpr2d_fused_ex_supported(prec, *Lq, H, st.order, st.ny + st.R) == 1


def _fused_s_planes(ctx, st, spec, kern: "_Kernel", prec: int) -> torch.Tensor:
    """The S planes (ns, H, M) of the kernel's bandwidths from the ones
    channel of `spec` by the fused S pass in `prec`."""
    geom, order = st.geom, st.order
    ns = len(_element_powers(st.d, order))
    Cv = st.ny + st.R
    Lq = (_lib.ivec(geom.G), _lib.ivec(geom.L), _lib.ivec(geom.qout[0]))
    S = ctx.empty((ns, kern.H, geom.M),
                  dtype=torch.float64 if prec == _lib.FLPR_PREC_F64 else torch.float32)
    ws = ctx.ws(ctx.lib.flpr_lpr2d_fused_ex_ws(prec, *Lq, kern.H, order, Cv))
    ctx.check(ctx.lib.flpr_lpr2d_fused_ex(prec, _FUSED_S, *Lq, kern.H, kern.npow, order, Cv, st.ny,
                                          spec.data_ptr(), kern.data_ptr(), kern.scale, None,
                                          float(st.opts["regularization"]), S.data_ptr(), None,
                                          None, None, None, None, ws.data_ptr(), ws.numel(),
                                          ctx.stream), "flpr_lpr2d_fused_ex")
    return S


def _evaluate_split(ctx, st: _LprState, filt, k64: int, ev, s64_all: bool = False) -> dict:
    """_evaluate_device with the first k64 bandwidths in FP64 (planes from
    the FP64 spectra) and the rest on the FP32 path; lambda (or max s) is
    the larger of the two groups' (the reference's, over all bandwidths).
    s64_all: the FP32 group's moment planes S are FP64 too (from the FP64
    spectra of the ones channel; flpr_lpr2d_fused_t), only its value
    channels run in FP32; k64 may then be 0."""
    lib = ctx.lib
    kern, bw, keep, _ = filt
    d, ny, R, order = st.d, st.ny, st.R, st.order
    geom = st.geom
    bw_k = bw[keep]
    H = len(keep)
    H32 = H - k64
    npow = 2 * order + 1
    k32k = _kernel_rows(kern, keep[k64:], geom)
    epw = _element_powers(d, order)
    ns = len(epw)
    nt = 1 if order == 0 else len(_design_powers(d, order))
    Cv = ny + R
    M = geom.M
    F32, F64 = _lib.FLPR_PREC_F32, _lib.FLPR_PREC_F64
    spec64 = _spectra64(ctx, st)
    scal64 = None
    # the FP64 group on the fused FP64 passes (S planes first: its lambda
    # floors the other group's), else on the cuFFT planes
    fused64 = _fused_ok(ctx, st, F64, max(k64, H32))
    if k64:
        k64k = _kernel_rows(kern, keep[:k64], geom)
        if fused64:
            S64 = _fused_s_planes(ctx, st, spec64, k64k, F64)
        else:
            S64 = _conv_s(ctx, geom, spec64, k64k, list(range(k64)), epw, F64, order == 0)
            T64 = _conv(ctx, geom, spec64, k64k,
                        [(1 + c, hk, epw[i]) for i in range(nt) for c in range(Cv)
                         for hk in range(k64)], F64, False)
        scal64 = ctx.empty(1)
        ctx.check(lib.flpr_scalar_of(order, nt, k64, M, S64.data_ptr(), F64, None,
                                     scal64.data_ptr(), ctx.stream), "flpr_scalar_of")
    reg = float(st.opts["regularization"])
    m = ctx.empty((H, M, ny))
    m32 = m.data_ptr() + k64 * M * ny * 8
    dots32 = ctx.empty((Cv, H32))
    scalar = ctx.empty(1)
    Lq = (_lib.ivec(geom.G), _lib.ivec(geom.L), _lib.ivec(geom.qout[0]))
    use_fused = (d == 2 and not st.opts.get("_no_fused", False)
                 and lib.flpr_lpr2d_fused_supported(*Lq, H32, order, Cv) == 1)
    floor = scal64.data_ptr() if scal64 is not None else None
    if s64_all:
        if fused64:
            S32 = _fused_s_planes(ctx, st, spec64, k32k, F64)
        else:
            S32 = _conv_s(ctx, geom, spec64, k32k, list(range(H32)), epw, F64, order == 0)
        ctx.check(lib.flpr_scalar_of(order, nt, H32, M, S32.data_ptr(), F64, floor,
                                     scalar.data_ptr(), ctx.stream), "flpr_scalar_of")
        ws = ctx.ws(lib.flpr_lpr2d_fused_ws(*Lq, H32, order, Cv))
        ctx.check(lib.flpr_lpr2d_fused_t(*Lq, H32, npow, order, Cv, ny, st.spec.data_ptr(),
                                         k32k.data_ptr(), k32k.scale, st.Q.data_ptr(), reg,
                                         S32.data_ptr(), scalar.data_ptr(), m32,
                                         dots32.data_ptr(), ws.data_ptr(), ws.numel(),
                                         ctx.stream), "flpr_lpr2d_fused_t")
        del ws
    elif use_fused:
        S32 = ctx.empty((ns, H32, M), dtype=torch.float32)
        ws = ctx.ws(lib.flpr_lpr2d_fused_ws(*Lq, H32, order, Cv))
        ctx.check(lib.flpr_lpr2d_fused_floor(*Lq, H32, npow, order, Cv, ny, st.spec.data_ptr(),
                                             k32k.data_ptr(), k32k.scale, st.Q.data_ptr(), reg,
                                             S32.data_ptr(), m32, dots32.data_ptr(),
                                             scalar.data_ptr(), floor, ws.data_ptr(),
                                             ws.numel(), ctx.stream), "flpr_lpr2d_fused_floor")
        del ws
    else:
        S32 = _conv_s(ctx, geom, st.spec, k32k, list(range(H32)), epw, F32, order == 0)
        T32 = _conv(ctx, geom, st.spec, k32k,
                    [(1 + c, hk, epw[i]) for i in range(nt) for c in range(Cv) for hk in range(H32)],
                    F32, False)
        ctx.check(lib.flpr_scalar_of(order, nt, H32, M, S32.data_ptr(), F32, floor,
                                     scalar.data_ptr(), ctx.stream), "flpr_scalar_of")
        ctx.check(lib.flpr_solve_reduce_given(order, nt, H32, H32, M, Cv, S32.data_ptr(),
                                              T32.data_ptr(), reg, ny, m32, st.Q.data_ptr(),
                                              dots32.data_ptr(), scalar.data_ptr(), F32,
                                              ctx.stream), "flpr_solve_reduce_given")
    parts_dots, parts_s0 = [], []
    if k64:
        dots64 = ctx.empty((Cv, k64))
        if fused64:
            ws = ctx.ws(lib.flpr_lpr2d_fused_ex_ws(F64, *Lq, k64, order, Cv))
            ctx.check(lib.flpr_lpr2d_fused_ex(F64, _FUSED_T, *Lq, k64, npow, order, Cv, ny,
                                              spec64.data_ptr(), k64k.data_ptr(), k64k.scale,
                                              st.Q.data_ptr(), reg, None, S64.data_ptr(),
                                              m.data_ptr(), dots64.data_ptr(), scalar.data_ptr(),
                                              None, ws.data_ptr(), ws.numel(), ctx.stream),
                      "flpr_lpr2d_fused_ex")
            del ws
        else:
            ctx.check(lib.flpr_solve_reduce_given(order, nt, k64, k64, M, Cv, S64.data_ptr(),
                                                  T64.data_ptr(), reg, ny, m.data_ptr(),
                                                  st.Q.data_ptr(), dots64.data_ptr(),
                                                  scalar.data_ptr(), F64, ctx.stream),
                      "flpr_solve_reduce_given")
        parts_dots.append(dots64)
        parts_s0.append(S64.view(ns, k64, M)[0])
    ev.mark("conv_solve")
    dots = torch.cat(parts_dots + [dots32], dim=1)
    quad = ctx.empty((H, ny))
    _stencil_quad(ctx, st, H, ny, m, quad)
    ev.mark("interp_reduce")
    packed = torch.cat([st.sq.reshape(-1), dots.reshape(-1), quad.reshape(-1)])
    S0 = torch.cat(parts_s0 + [S32.view(ns, H32, M)[0].to(torch.float64)], dim=0)
    return dict(keep=keep, bw_k=bw_k, H=H, m=m, S=S0.view(1, H, M), ns=1, mstride=ny,
                packed=packed, dual=True, fp64_bandwidths=k64, s_planes_fp64=bool(s64_all))


def _evaluate_host(st: _LprState, r: dict, packed: Optional[np.ndarray]) -> dict:
    """GCV, DoF and the 1-SE choice from the downloaded reductions."""
    n, ny, R, H = st.n, st.ny, st.R, r["H"]
    Cv = ny + R
    if st.calc_dof:
        if r["dual"]:
            sq_h = packed[:Cv]
            dots_h = packed[Cv:Cv + Cv * H].reshape(Cv, H)
            quad_h = packed[Cv + Cv * H:].reshape(H, ny)
            rss_h = sq_h[None, :ny] - 2.0 * dots_h[:ny].T + quad_h
            pdot_h = dots_h[ny:]
            pp_h = sq_h[ny:]
        else:
            Rm = max(R, 1)
            rss_h = packed[:H * ny].reshape(H, ny)
            pdot_h = packed[H * ny:H * ny + Rm * H].reshape(Rm, H)[:R]
            pp_h = packed[H * ny + Rm * H:][:R]
        gcv = _gcv_from_sums(n, rss_h, pdot_h, pp_h, st.dy, st.y_is_complex, st.opts)
        dstd = float(st.opts.get("dstd", 0.0))
        sel = _one_se_rule(gcv["gcv_m"], gcv["gcv_sd"], r["bw_k"], prefer_smaller=True,
                           dstd=dstd)
    else:
        gcv = None
        sel = 0
    return dict(r, gcv=gcv, sel=sel)


def _finalize_lpr(ctx, st: _LprState, r: dict, ev, search) -> RegressionOutput:
    """Fitted values at the selected bandwidth and the result structure."""
    pend = _finalize_enqueue(ctx, st, r, ev)
    torch.cuda.current_stream(ctx.device).synchronize()
    return _finalize_build(ctx, st, r, pend, ev, search)


def _finalize_enqueue(ctx, st: _LprState, r: dict, ev, device_select: bool = False,
                      bufs: Optional[dict] = None, hsum_dev: Optional[torch.Tensor] = None) -> dict:
    """Device part of the output stage: fitted values at the selected
    bandwidth, residuals, grid and s0 copied into pinned host memory
    (asynchronously; valid after the stream synchronises).

    device_select: GCV, DoF and the 1-SE choice come from flpr_gcv_select
    on the packed reductions and the chosen grid is gathered on the device
    (flpr_select_grid), so nothing here waits for the host; `r` then needs
    no host evaluation.  bufs: preallocated pinned buffers (see _output_bufs)
    for the outputs they name; with bufs given, the other outputs are
    returned as device tensors for the caller to download.  hsum_dev:
    per-bandwidth sums of h on the device."""
    lib = ctx.lib
    d, n, ny = st.d, st.n, st.ny
    geom = st.geom
    m, S = r["m"], r["S"]
    H, ns, M = r["H"], r["ns"], geom.M
    gcv_dev = sel_dev = None
    if device_select:
        sel_dev = ctx.empty(1, dtype=torch.int32)
        if st.calc_dof:
            if hsum_dev is None:
                hs = torch.from_numpy(np.ascontiguousarray(np.sum(r["bw_k"], axis=1))).pin_memory()
                hsum_dev = hs.to(ctx.device, non_blocking=True)
            gcv_dev = ctx.empty(4 * H)
            agg = {"first": 0, "average": 1, "sum": 2}.get(str(st.opts.get("gcv_selection",
                                                                            "first")))
            if agg is None:
                raise ValueError(f"Unknown aggregation method: {st.opts.get('gcv_selection')}. "
                                 "Use 'first', 'average', or 'sum'.")
            ctx.check(lib.flpr_gcv_select(H, ny, st.R, 1 if r["dual"] else 0,
                                          1 if st.y_is_complex else 0, agg, float(n),
                                          float(st.opts.get("dstd", 0.0)), r["packed"].data_ptr(),
                                          hsum_dev.data_ptr(), gcv_dev.data_ptr(),
                                          sel_dev.data_ptr(), ctx.stream), "flpr_gcv_select")
        else:
            sel_dev.zero_()
        gv_dev = ctx.empty((ny, M))
        s0_dev = ctx.empty(M)
        s_prec = _lib.FLPR_PREC_F32 if S.dtype == torch.float32 else _lib.FLPR_PREC_F64
        ctx.check(lib.flpr_select_grid(M, ny, r["mstride"], m.shape[0], m.data_ptr(),
                                       S.data_ptr(), s_prec, sel_dev.data_ptr(),
                                       gv_dev.data_ptr(), s0_dev.data_ptr(), ctx.stream),
                  "flpr_select_grid")
    else:
        sel = r["sel"]
        mv = m[sel if st.calc_dof else 0]                # (M, mstride)
        gv_dev = mv[:, :ny].t().contiguous()             # (ny, M)
        s0_dev = S.view(ns, H, M)[0, sel]
    yhat_dev = ctx.empty((ny, n))
    if st.methods["output"] == "cubic":
        coef = gv_dev.clone()
        ctx.check(lib.flpr_spline_prefilter(d, st.G_arg, ny, 1, st.spl.lu.data_ptr(),
                                            coef.data_ptr(), ctx.stream), "flpr_spline_prefilter")
        ctx.check(lib.flpr_spline_eval(d, n, st.dx.data_ptr(), st.spl.axes.data_ptr(), st.G_arg,
                                       ny, coef.data_ptr(), yhat_dev.data_ptr(), ctx.stream),
                  "flpr_spline_eval")
    else:
        ctx.check(lib.flpr_interp_eval(d, n, st.dx.data_ptr(), st.ax_arg, st.G_arg, ny,
                                       gv_dev.data_ptr(), yhat_dev.data_ptr(), ctx.stream),
                  "flpr_interp_eval")
    dn = None
    if st.variance:
        acc = ctx.empty(1)
        ctx.check(lib.flpr_exp_weighted_sum(n, st.y_raw_dev.data_ptr(), yhat_dev.data_ptr(),
                                            acc.data_ptr(), ctx.stream), "flpr_exp_weighted_sum")
        # d = 1 / mean(y exp(-yhat)) (api.py:777-786), kept on the device
        dn = 1.0 / ((1.0 / n) * acc)
        yhat_dev = torch.exp(yhat_dev) / dn
        gv_dev = torch.exp(gv_dev) / dn
    ev.mark("final_interp")
    # residuals on the device; every result is copied into pinned host memory
    # with one synchronisation (the caching host allocator recycles the pages)
    if st.variance:
        res_dev = st.y_raw_dev[None, :] - yhat_dev
    else:
        res_dev = torch.stack(st.ycols[:ny], dim=0) - yhat_dev
    # fitted values, residuals and grid values in the layouts of the result
    # (formed here so the host only takes views of the downloaded arrays)
    yhat_dev = _result_layout(yhat_dev, st.dy, st.y_is_complex)
    res_dev = _result_layout(res_dev, st.dy, st.y_is_complex)
    gv_dev = _result_layout(gv_dev, st.dy, st.y_is_complex)
    parts = {"yh": yhat_dev, "rh": res_dev, "gvh": gv_dev, "s0h": s0_dev, "dn": dn,
             "gcv": gcv_dev, "sel": sel_dev}
    out = {}
    for k, t in parts.items():
        if t is None:
            out[k] = None
        elif bufs is not None and bufs.get(k) is not None:
            bufs[k].copy_(t.reshape(bufs[k].shape), non_blocking=True)
            out[k] = bufs[k]
        elif bufs is not None:
            out[k] = t
        else:
            out[k] = _to_host(t)
    return out


def _result_layout(t: torch.Tensor, dy: int, y_is_complex: bool) -> torch.Tensor:
    """(channels, k) device rows -> (k,) for one response column, (k, dy)
    otherwise; complex responses (real/imaginary row pairs) as complex128."""
    if y_is_complex:
        t = torch.view_as_complex(t.reshape(dy, 2, -1).permute(2, 0, 1).contiguous())
    elif dy > 1:
        t = t.t().contiguous()
    else:
        return t[0]
    return t[:, 0] if dy == 1 else t


def _output_bufs(st: _LprState, H: int) -> dict:
    """Pinned host buffers for the small outputs of
    _finalize_enqueue(device_select=True): the bandwidth choice, the GCV
    arrays and the variance normaliser."""
    def pin(shape, dtype=torch.float64):
        return torch.empty(shape, dtype=dtype, pin_memory=True)

    return {"dn": pin(1) if st.variance else None,
            "gcv": pin(4 * H) if st.calc_dof else None, "sel": pin(1, torch.int32)}


def _finalize_build(ctx, st: _LprState, r: dict, pend: dict, ev, search,
                    copy: bool = False) -> RegressionOutput:
    """Result structure from the downloaded outputs of _finalize_enqueue
    (copy: detach the arrays from reused pinned buffers)."""
    d, dy = st.d, st.dy
    geom, opts = st.geom, st.opts
    bw_k = r["bw_k"]
    if pend.get("sel") is not None:
        sel = int(pend["sel"].numpy()[0])
        if st.calc_dof:
            if sel < 0:
                raise ValueError(
                    "All GCV scores are NaN or Inf. Regression failed for all bandwidths. "
                    "Try: (1) Use larger bandwidth h, (2) Increase grid points, "
                    "(3) Check for data quality issues")
            g4 = pend["gcv"].numpy().reshape(4, r["H"]).copy()
            gcv = {"gcv_m": g4[0], "gcv_sd": g4[1], "dof": g4[2], "dof_stderr": g4[3]}
        else:
            gcv = None
    else:
        sel, gcv = r["sel"], r["gcv"]
    yh, rh, gvh = pend["yh"].numpy(), pend["rh"].numpy(), pend["gvh"].numpy()
    if copy:
        yh, rh, gvh = yh.copy(), rh.copy(), gvh.copy()
    s0h = pend["s0h"]
    d_norm = float(pend["dn"].numpy()[0]) if pend["dn"] is not None else None
    gshape = tuple(int(g) for g in geom.G)
    # already (n,) / (n, dy), complex where the response is (_result_layout)
    yhat, residuals = yh, rh
    grid_values = gvh.reshape(gshape if dy == 1 else gshape + (dy,))
    s0 = s0h.numpy().reshape(gshape)
    if copy:
        s0 = s0.copy()
    ev.mark("download")
    ev.finish()
    interp = GridInterpolant(st.axes_raw, grid_values, ctx.device, method=st.methods["output"])
    selected = bw_k[sel]
    if st.calc_dof:
        idmin = int(np.argmin(gcv["gcv_m"]))
        gcv_result = {
            "bandwidths": bw_k,
            "gcv_m": gcv["gcv_m"],
            "gcv_sd": gcv["gcv_sd"],
            "idmin": idmin,
            "id1se": int(sel),
            "h1se": selected,
            "hmin": bw_k[idmin],
            "dof": gcv["dof"],
            "dof_stderr": gcv["dof_stderr"],
        }
        dof = gcv["dof"][sel]
        dof_se = gcv["dof_stderr"][sel]
    else:
        gcv_result = {
            "bandwidths": bw_k, "gcv_m": np.array([np.nan]), "gcv_sd": np.array([np.nan]),
            "idmin": 0, "id1se": 0, "h1se": selected, "hmin": selected,
            "dof": np.array([np.nan]), "dof_stderr": np.array([np.nan]),
        }
        dof = dof_se = np.nan
    metadata = {
        "options": opts,
        "order": st.order,
        "bandwidths_tested": bw_k,
        "fitted_at_samples": yhat,
        "residuals": residuals,
        "mean": geom.mean,
        "std": geom.std,
        "dof": dof,
        "dof_stderr": dof_se,
        "precision": "fp32" if st.prec == _lib.FLPR_PREC_F32 else "fp64",
        # FP32 path: bandwidths whose kernel covers few points, evaluated in FP64
        "fp64_bandwidths": int(r.get("fp64_bandwidths", 0)),
        # FP32 path of order 2: moment planes S in FP64, value channels in FP32
        "moment_planes": "fp64" if (st.prec == _lib.FLPR_PREC_F64
                                    or r.get("s_planes_fp64", False)) else "fp32",
        "bandwidth_search": search if search is not None else {"mode": "full"},
    }
    return RegressionOutput(yhat=yhat, grid=tuple(st.axes_raw), h=selected, gcv_yhat=gcv_result,
                            fpp_yhat=interp, metadata=metadata, dof=dof, dof_stderr=dof_se,
                            d=d_norm, s0=s0)


# windows a learned search may walk before it falls back to the full sweep
_MAX_WALKS = 3


def _start_summary(ctx, pending: dict, dx, ycols, stats, n, d, d_stats=None, model=None,
                   order: int = 0, log_h=None) -> None:
    """The proposal chain, enqueued on the caller's stream ahead of the
    spread: binned moment sums of the data, their feature vector, the
    network and the window start in the bandwidth list
    (learned.DeviceProposal), copied to pinned host memory.  Nothing here
    waits for the device.  (On a second stream beside the spread the fit was
    1-1.5% slower: the binned sums' shared-memory atomics compete with the
    spread's kernels for the same SMs.)"""
    from . import learned as _learned
    if len(ycols) != 1 or d > 2 or model is None or log_h is None:
        return
    if d_stats is None:
        d_stats = ctx.upload(np.ascontiguousarray(stats[:2].ravel()))
    prop = _learned.DeviceProposal(model, [(d, order, n)], [log_h], ctx.device)
    _lib.check(ctx.lib.flpr_bin_moments(d, n, dx.data_ptr(), ycols[0].data_ptr(),
                                        d_stats.data_ptr(), prop.bins.data_ptr(), ctx.stream),
               "flpr_bin_moments")
    prop.enqueue(ctx.stream)
    lo_h, t_h = _to_host(prop.lo), _to_host(prop.t)
    done = torch.cuda.Event()
    done.record()
    pending.update(prop=prop, lo=lo_h, t=t_h, done=done, keep=(d_stats,))


def _window_filter(ctx, st: _LprState, filt_all, lo_dev: torch.Tensor, W: int):
    """Kernel factors of the W consecutive bandwidths starting at the index
    in lo_dev (on the device) of a filter over the whole list, gathered on
    the device (flpr_copy_rows), and their bandwidth sums.  The returned
    filter's bandwidth rows are placeholders until the host knows the
    window."""
    kern, bw, keep, _ = filt_all
    H, npow = kern.H, kern.npow
    data = ctx.empty((int(sum(W * npow * int(La) for La in st.geom.L)), 2))
    src, dst = kern.data_ptr(), data.data_ptr()
    for La in st.geom.L:
        row = npow * int(La) * 16
        ctx.check(ctx.lib.flpr_copy_rows(src, dst, row, W, lo_dev.data_ptr(), ctx.stream),
                  "flpr_copy_rows")
        src += H * row
        dst += W * row
    hs_all = st.__dict__.get("_hsum_all")
    if hs_all is None or hs_all.shape[0] != H:
        hs = torch.from_numpy(np.ascontiguousarray(np.sum(bw[keep], axis=1))).pin_memory()
        hs_all = hs.to(ctx.device, non_blocking=True)
    hsum = ctx.empty(W)
    ctx.check(ctx.lib.flpr_copy_rows(hs_all.data_ptr(), hsum.data_ptr(), 8, W, lo_dev.data_ptr(),
                                     ctx.stream), "flpr_copy_rows")
    kw = _Kernel(kern.kid, data, W, npow, kern.scale)
    kw.device_window = True     # bandwidths chosen on the device: no host-side split
    return (kw, bw[keep][:W], np.arange(W), np.zeros(W, dtype=bool)), hsum, hs_all


def _learned_search(ctx, st: _LprState, bandwidths: np.ndarray, model, ev, pending: dict):
    """Proposal + five-bandwidth window, walked toward an edge minimum (the
    next window shares the edge bandwidth) at most _MAX_WALKS times; returns
    (evaluation, search record, pending outputs or None) or None when the
    full sweep must run.  The first window is chosen and evaluated without a
    host round trip: the proposal chain was enqueued ahead of the spread
    (_start_summary), the window's kernel factors are gathered on the device
    at the start index it wrote, and GCV, the 1-SE choice and the output
    stage are enqueued behind them; one synchronisation brings back the
    window, its scores and the outputs (used as they are when the window is
    accepted)."""
    from . import learned as _learned
    if not (st.calc_dof and st.ny == 1 and not st.y_is_complex and st.d <= 2
            and st.kid == 0) or not pending.get("prop"):
        return None
    nlist = int(bandwidths.shape[0])
    npow = 2 * st.order + 1
    filt_all = _filter_bandwidths(ctx, st.geom, bandwidths, npow, st.kid)
    if len(filt_all[2]) != nlist:
        return None                         # a bandwidth of the list is filtered out
    R = _learned.REFINE
    torch.cuda.current_stream(ctx.device).wait_event(pending["done"])
    filt_w, hsum, _ = _window_filter(ctx, st, filt_all, pending["prop"].lo, R)
    r = _evaluate_device(ctx, st, filt_w, ev)
    pend = _finalize_enqueue(ctx, st, r, ev, device_select=True, hsum_dev=hsum)
    torch.cuda.current_stream(ctx.device).synchronize()
    ev.mark("proposal")
    return _learned_finish(ctx, st, bandwidths, r, pend, int(pending["lo"].numpy()[0]),
                           float(pending["t"].numpy()[0]), ev)


def _learned_finish(ctx, st: _LprState, bandwidths: np.ndarray, r: dict, pend: dict, lo: int,
                    t: float, ev):
    """Acceptance of a first window evaluated on the device (start index lo,
    proposal t; r / pend its evaluation and output stage, complete), then the
    walks toward an edge minimum: (evaluation, search record, pending
    outputs or None) or None when the full sweep must run."""
    from . import learned as _learned
    R = _learned.REFINE
    nlist = int(bandwidths.shape[0])
    window = np.arange(lo, lo + R)
    r["bw_k"] = bandwidths[window]
    record = {"mode": "learned", "proposal_index": t, "windows": [[int(i) for i in window]],
              "nlist": nlist, "accepted": False}
    gcv_m = pend["gcv"].numpy()[:R]
    for walk in range(_MAX_WALKS + 1):
        pos = int(np.argmin(gcv_m))
        if _learned.accept_window(window, pos, nlist):
            record["accepted"] = True
            record["evaluated"] = len({i for w in record["windows"] for i in w})
            return r, record, (pend if walk == 0 else None)
        if walk == _MAX_WALKS:
            break
        step = R - 1
        lo = int(window[0]) + (step if pos == len(window) - 1 else -step)
        lo = int(np.clip(lo, 0, nlist - R))
        nxt = np.arange(lo, lo + R)
        if np.array_equal(nxt, window):
            return None
        window = nxt
        record["windows"].append([int(i) for i in window])
        filt = _filter_bandwidths(ctx, st.geom, bandwidths[window], 2 * st.order + 1, st.kid)
        r = _evaluate_device(ctx, st, filt, ev)
        r = _evaluate_host(st, r, r["packed"].cpu().numpy())
        gcv_m = r["gcv"]["gcv_m"]
    return None


def _full_sweep(ctx, st: _LprState, bandwidths: np.ndarray, ev, search,
                filt=None) -> RegressionOutput:
    """Every bandwidth of the list: GCV, the 1-SE choice and the output stage
    are enqueued on the device behind the reductions; one synchronisation."""
    if filt is None:
        filt = _filter_bandwidths(ctx, st.geom, bandwidths, 2 * st.order + 1, st.kid)
    r = _evaluate_device(ctx, st, filt, ev)
    pend = _finalize_enqueue(ctx, st, r, ev, device_select=True)
    torch.cuda.current_stream(ctx.device).synchronize()
    return _finalize_build(ctx, st, r, pend, ev, search)


def _fit_lpr(ctx, x_arr, y_arr, dy, bandwidths, opts, order, prec, variance, y_is_complex,
             dev_inputs=None, timings=None, learned=None):
    """One LPR fit.  With a proposal network (`learned`) a walked window of
    five bandwidths replaces the sweep when its GCV minimum is trusted; the
    full sweep over `bandwidths` runs otherwise (sharing the spectra)."""
    ev = _PhaseEvents(timings)
    ev.mark("start")
    pending = {}
    hook = None
    if learned is not None:
        from . import learned as _learned
        lh = _learned.isotropic_log_h(bandwidths)

        def hook(dx, ycols, stats, n, d, d_stats=None):
            _start_summary(ctx, pending, dx, ycols, stats, n, d, d_stats=d_stats, model=learned,
                           order=order, log_h=lh)
    st = _prepare_lpr(ctx, x_arr, y_arr, dy, opts, order, prec, variance, y_is_complex,
                      dev_inputs, ev, hook=hook, bandwidths=bandwidths)
    found = (_learned_search(ctx, st, bandwidths, learned, ev, pending)
             if learned is not None else None)
    if found is not None:
        r, search, pend = found
        if pend is not None:
            return _finalize_build(ctx, st, r, pend, ev, search)
        return _finalize_lpr(ctx, st, r, ev, search)
    search = None if learned is None else {"mode": "learned", "accepted": False,
                                           "fallback": "full sweep"}
    return _full_sweep(ctx, st, bandwidths, ev, search)


def _gcv_from_sums(n, rss, pdot, pp, dy, y_is_complex, opts):
    """DoF (regression.py:1276-1354) and GCV (regression.py:280-471) from the
    device reductions."""
    H = rss.shape[0]
    R = pdot.shape[0]
    if y_is_complex:
        rss_col = rss[:, 0::2] + rss[:, 1::2]
    else:
        rss_col = rss
    tr = n * (pdot / pp[:, None])
    tr = np.where(np.isnan(tr), n, tr)
    tr = np.clip(tr, 0.0, n)
    dof = np.mean(tr, axis=0)
    if R > 1:
        dof_se = np.std(tr, axis=0, ddof=1) / np.sqrt(R)
        pd = 1 - tr / n
        if y_is_complex:
            pd = 2 * pd - 1
        pdc = np.clip(pd, 0.0, 1.0)
        pen = 1.0 / np.maximum(pdc, 0.01) ** 2
        pen_std = np.std(pen, axis=0, ddof=1)
        pen_mean = np.mean(pen, axis=0)
        if y_is_complex:
            dof = n * (1 - np.mean(pdc, axis=0))
    else:
        dof_se = np.zeros(H)
        pen_std = np.zeros(H)
        pen_mean = None
    agg = str(opts.get("gcv_selection", "first"))
    gcv_m = np.empty(H)
    gcv_sd = np.empty(H)
    for ih in range(H):
        mse = rss_col[ih] / n
        if pen_mean is not None:
            pen_v = float(pen_mean[ih])
        else:
            pdv = max(float(np.clip(1.0 - dof[ih] / n, 0.0, 1.0)), 0.01)
            pen_v = 1.0 / pdv ** 2
        g = mse * pen_v
        if agg == "first":
            sc, ms = float(g[0]), float(mse[0])
        elif agg == "average":
            sc, ms = float(np.mean(g)), float(np.mean(mse))
        elif agg == "sum":
            sc, ms = float(np.sum(g)), float(np.sum(mse))
        else:
            raise ValueError(f"Unknown aggregation method: {agg}. Use 'first', 'average', or 'sum'.")
        gcv_m[ih] = sc
        gcv_sd[ih] = ms * pen_std[ih] if pen_std[ih] > 0 else 0.0
    return {"gcv_m": gcv_m, "gcv_sd": gcv_sd, "dof": dof, "dof_stderr": dof_se,
            "trace": tr, "rss": rss_col}


# ---------------------------------------------------------------------------
# cv_fastkde
# ---------------------------------------------------------------------------
def cv_fastkde(x, h=None, options: Optional[dict] = None) -> KDEOutput:
    """Kernel density estimation with LCV bandwidth selection (drop-in for the
    reference ``cv_fastkde``, api.py:835-1184)."""
    x_arr = _as_column_matrix(x)
    n, dims = x_arr.shape
    if n < 2:
        raise ValueError(f"Input x must have at least 2 observations. Got {n} observations.")

    opts = set_defaults(options, order=0, calc_dof=False, y_type_out="mean")
    opts = set_defaults(opts, kernel_type="gaussian", verbose=False, dh=20)
    if opts.get("accuracy") is None:
        opts["accuracy"] = max(6 - int(np.ceil(np.log10(n))), 4)
    if opts.get("N") is None:
        an = int(np.ceil(n ** (1.0 / dims)))
        opts["N"] = [an] * dims if dims > 1 else an
    bandwidths = _prepare_bandwidths(h, dims, opts, lambda: _default_hrange(x_arr))
    _check_supported(dims, opts)
    Nopt = opts["N"]
    gs = Nopt if isinstance(Nopt, int) else (Nopt[0] if dims == 1 else Nopt)
    G = np.atleast_1d(np.asarray(gs, dtype=int))
    if G.size == 1:
        G = np.repeat(G, dims)
    prec = _precision(opts)
    ctx = _Ctx(_device(opts))
    with torch.cuda.device(ctx.device):
        return _fit_kde(ctx, x_arr, bandwidths, opts, G, prec)


def _fit_kde(ctx, x_arr, bandwidths, opts, G, prec):
    lib = ctx.lib
    n, d = x_arr.shape
    dx = ctx.upload(x_arr)
    flags_h = _to_host(_finite_flags([dx]))
    stats = _point_stats(ctx, dx, n, d)
    _raise_nonfinite(flags_h.numpy(), [("Input x", 0)], "cv_fastkde")
    geom = _make_geom(stats, n, d, G, int(opts["accuracy"]), bool(opts.get("flag_power2", True)))
    kern, bw, keep, ihbad = _filter_bandwidths(ctx, geom, bandwidths, 1, _kernel_id(opts))
    if len(keep) != bandwidths.shape[0] or bw.shape[0] != bandwidths.shape[0]:
        # the reference indexes its density columns by the unfiltered list here
        raise ValueError("a bandwidth is too small for the KDE grid")
    H = len(keep)
    spec = _spread_fft(ctx, geom, dx, [], prec)
    S = _conv(ctx, geom, spec, kern, [(0, int(k), (0,) * d) for k in keep], prec, True)
    S64 = S if S.dtype == torch.float64 else S.to(torch.float64)
    # raw grid axes by inverting centring and z-scoring (api.py:1038-1057)
    axes_raw = []
    for a in range(d):
        axs = np.linspace(geom.lo[a], geom.hi[a], int(G[a]))
        xs_min_u = (geom.xmin[a] - geom.mean[a]) / geom.std[a]
        xs_max_u = (geom.xmax[a] - geom.mean[a]) / geom.std[a]
        axes_raw.append((axs + (xs_max_u + xs_min_u) / 2) * geom.std[a] + geom.mean[a])
    dxg = float(np.prod([ax[1] - ax[0] for ax in axes_raw]))
    k0 = [(1.0 / SQRT_2PI) / float(np.prod(bandwidths[i])) for i in range(H)]
    M = geom.M
    f = ctx.empty((H, M))
    lcv = ctx.empty((H, 2))
    ws = ctx.ws(lib.flpr_kde_ws(n, H, M))
    ctx.check(lib.flpr_kde_lcv(d, n, dx.data_ptr(), _lib.dvec(_axes_arg(axes_raw)),
                               _lib.ivec(geom.G), H, S64.data_ptr(), dxg, _lib.dvec(k0),
                               f.data_ptr(), lcv.data_ptr(), ws.data_ptr(), ws.numel(),
                               ctx.stream), "flpr_kde_lcv")
    # both results into pinned memory with one synchronisation (a pageable
    # copy of the (H, M) densities runs at a fraction of the link speed)
    lc_h, f_h = _to_host(lcv), _to_host(f)
    torch.cuda.current_stream(ctx.device).synchronize()
    lc = lc_h.numpy()
    lcv_m = lc[:, 0].copy()
    var_l = lc[:, 1] / n
    lcv_sd = np.sqrt(var_l) * np.sqrt(n)
    sel = _one_se_rule(lcv_m, lcv_sd, bandwidths, prefer_smaller=False)
    gshape = tuple(int(g) for g in G)
    fall = f_h.numpy().reshape((H,) + gshape)
    fhat_all = np.moveaxis(fall, 0, -1)
    fhat = fall[sel]
    interp = GridInterpolant(axes_raw, fhat, ctx.device,
                             method=opts.get("output_interp_method", "linear"))
    unique_axes = [np.unique(bandwidths[:, a]) for a in range(d)]
    gsh = tuple(len(u) for u in unique_axes)
    matrix = lcv_m.reshape(gsh) if int(np.prod(gsh)) == len(lcv_m) else None
    idmax = int(np.argmax(lcv_m))
    lcv_result = {
        "hlist": bandwidths,
        "lcv_m": lcv_m,
        "lcv_sd": lcv_sd,
        "idmax": idmax,
        "id1se": int(sel),
        "hmax": bandwidths[idmax],
        "h1se": bandwidths[sel],
        "unique_axes": unique_axes,
        "matrix": matrix,
    }
    metadata = {"options": opts, "bandwidths_tested": bandwidths, "fhat_all": fhat_all,
                "precision": "fp32" if prec == _lib.FLPR_PREC_F32 else "fp64"}
    return KDEOutput(fhat=fhat, grid=tuple(axes_raw), h=bandwidths[sel], lcv=lcv_result,
                     fpp=interp, metadata=metadata)
