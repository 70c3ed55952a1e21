"""numpy/scipy restatement of the reference fastLPR NUFFT path (FP64).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the CPU
baseline of ``bench.py``.  Every function cites the reference code it
restates; paths are relative to ``fastLPR_py/src/fastlpr/``.

The restatement follows the reference step by step, including its
structure (one full-size inverse FFT per (design element, bandwidth,
channel) product), so that timing it gives a faithful CPU baseline.  It
runs the whole chain in float64/complex128, which is the reference with
``nufftn_type1.get_complex_dtype`` returning complex128.
"""
from __future__ import annotations

import math
import warnings
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import scipy.fft as sfft

from .spline import cubic_interp

SQRT_2PI = math.sqrt(2.0 * math.pi)

_NATIVE = None


def _native():
    """ctypes handle of oracle/liboracle.so (C restatement of the hot loops),
    or None when it has not been built."""
    global _NATIVE
    if _NATIVE is None:
        import ctypes
        import os
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "liboracle.so")
        if not os.path.exists(path):
            _NATIVE = False
        else:
            lib = ctypes.CDLL(path)
            P = ctypes.c_void_p
            lib.oracle_spread.argtypes = [ctypes.c_int, ctypes.c_int64, P, ctypes.c_int, P, P,
                                          ctypes.c_int, P, P]
            lib.oracle_interp.argtypes = [ctypes.c_int, ctypes.c_int64, P, P, P, ctypes.c_int64,
                                          P, P]
            _NATIVE = lib
    return _NATIVE or None


# --------------------------------------------------------------------------
# Bandwidth grid -- bandwidth.py:22-137
# --------------------------------------------------------------------------
def get_hlist(n, range, spacing=None) -> np.ndarray:  # noqa: A002 (reference name)
    """Bandwidth candidates, Cartesian product in Fortran order (bandwidth.py:105-137)."""
    r = np.asarray(range, dtype=float)
    if r.ndim == 1:
        r = r.reshape(1, 2)
    dims = r.shape[0]
    n_list = [int(n)] * dims if np.isscalar(n) else [int(v) for v in n]
    if len(n_list) != dims:
        raise ValueError("n must match the number of rows in range.")
    if spacing is None:
        spacing = lambda lo, hi, num: np.logspace(np.log10(lo), np.log10(hi), num)  # noqa: E731
    grids = [spacing(lo, hi, num) if num > 1 else np.array([lo], dtype=float)
             for (lo, hi), num in zip(r, n_list)]
    mesh = np.meshgrid(*grids, indexing="ij")
    return np.column_stack([a.ravel("F") for a in mesh])


# --------------------------------------------------------------------------
# Grid / padding parameters -- convolution.py:389-409, kernel.py:97-156
# --------------------------------------------------------------------------
def grid_params(G: Sequence[int], flag_power2: bool = True):
    """Padded length L, knot window qin and crop window qout per axis."""
    G = np.atleast_1d(np.asarray(G, dtype=int))
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


def spread_params(L: Sequence[int], accuracy: int):
    """compute_grid_params for the knot grid (kernel.py:136-156): Msp, tau, ratio.
    accuracy 0 is nearest-bin binning (nufftn_type1.py:442-516): one tap of
    weight 1, i.e. Msp = 0 with an infinite tau."""
    L = np.atleast_1d(np.asarray(L, dtype=int))
    if accuracy <= 6:
        ratio = 1
    elif accuracy <= 11:
        ratio = 2
    else:
        ratio = 3
    msp = accuracy
    tau = (np.pi * msp) / (L * L * ratio * (ratio - 0.5))
    if accuracy == 0:
        tau = np.full(np.shape(L), np.inf)
    return msp, tau, ratio


# --------------------------------------------------------------------------
# Knot mapping -- convolution.py:176-213, convolution.py:68, nufftn_type1.py:140-176
# --------------------------------------------------------------------------
def knot_coordinates(x_scaled: np.ndarray, L, G, qin) -> np.ndarray:
    """Map centred data to NUFFT knots xmod in [0, 2*pi) per axis."""
    x = np.atleast_2d(np.asarray(x_scaled, dtype=float))
    n, dims = x.shape
    L = np.atleast_1d(L)
    G = np.atleast_1d(G)
    x_min = x.min(axis=0)
    x_max = x.max(axis=0)
    x_scale = x_max - x_min
    x_scale[x_scale == 0] = 1.0
    x_norm = np.empty_like(x)
    for d in range(dims):
        idx_range = np.linspace(-0.5, 0.5 - 1 / L[d], L[d])
        if G[d] != L[d]:
            ks = idx_range[qin[1, d]] - idx_range[qin[0, d]]
            x_norm[:, d] = (x[:, d] - x_min[d]) / x_scale[d] * ks + idx_range[qin[0, d]]
        else:
            ks = idx_range[-1] - idx_range[0]
            x_norm[:, d] = (x[:, d] - x_min[d]) / x_scale[d] * ks - 0.5
    x_norm += 0.5
    np.mod(x_norm, 1.0, out=x_norm)
    knots = x_norm - 0.5                      # nufft_type1_wrapper (convolution.py:68)
    knots = knots * (L / L)                   # scale_knots: * Fs / N with Fs = N
    kmin = (knots.min(axis=0) + knots.max(axis=0)) * 0.5 - 0.5
    shift = -0.5 - kmin
    knots = knots + shift
    knots = knots * (2 * np.pi)
    np.mod(knots, 2 * np.pi, out=knots)
    return knots


# --------------------------------------------------------------------------
# Gaussian gridding -- spreading_fused.py:48-129 (real channels)
# --------------------------------------------------------------------------
def spread_grid(xmod: np.ndarray, chans: np.ndarray, L, msp: int, tau) -> np.ndarray:
    """Accumulate every channel onto the periodic L^d grid.

    Returns (C, *L) float64.  Channel values must be real; complex responses
    are passed as separate real and imaginary channels.
    """
    xmod = np.atleast_2d(xmod)
    n, dims = xmod.shape
    chans = np.asarray(chans, dtype=float).reshape(n, -1)
    C = chans.shape[1]
    L = np.atleast_1d(L).astype(np.int64)
    tau = np.atleast_1d(tau).astype(float)
    lib = _native()
    if lib is not None and dims <= 3 and 2 * msp + 1 <= 32:
        xm = np.ascontiguousarray(xmod, dtype=float)
        ch = np.ascontiguousarray(chans)
        Lc = np.ascontiguousarray(L)
        tc = np.ascontiguousarray(tau)
        out = np.zeros((C, int(np.prod(L))))
        lib.oracle_spread(dims, n, xm.ctypes.data, C, ch.ctypes.data, Lc.ctypes.data, msp,
                          tc.ctypes.data, out.ctypes.data)
        return out.reshape((C,) + tuple(L))
    hx = 2 * np.pi / L
    m = np.round(xmod / hx).astype(np.int64)
    strides = np.ones(dims, dtype=np.int64)
    for d in range(dims - 2, -1, -1):
        strides[d] = strides[d + 1] * L[d + 1]
    total = int(np.prod(L))
    out = np.zeros((C, total), dtype=float)
    taps = np.arange(-msp, msp + 1)
    # per-axis tap indices and exponents, then every tap combination
    idx_ax, ex_ax = [], []
    for d in range(dims):
        mj = m[:, d][:, None] + taps[None, :]
        idx_ax.append(np.mod(mj, L[d]) * strides[d])
        diff = xmod[:, d][:, None] - hx[d] * mj
        ex_ax.append(diff * diff / (4 * tau[d]))
    for combo in np.ndindex(*([len(taps)] * dims)):
        idx = np.zeros(n, dtype=np.int64)
        ex = np.zeros(n)
        for d, j in enumerate(combo):
            idx += idx_ax[d][:, j]
            ex = ex + ex_ax[d][:, j]
        w = np.exp(-ex)
        for c in range(C):
            out[c] += np.bincount(idx, weights=chans[:, c] * w, minlength=total)
    return out.reshape((C,) + tuple(L))


def nufft_spectra_oversampled(grid: np.ndarray, n_points: int, L, ratio: int, tau,
                              workers: int = 1) -> np.ndarray:
    """Oversampled path (accuracy >= 7), nufftn_type1.py:693-770 then the
    ifftshift of convolution.py:235-236: FFT of the ratio*L grid, fftshift,
    the central L frequencies, / (M ratio^d), times 1/Kn with
    Kn = sqrt(prod tau / pi^d) exp(-sum tau_d f_d^2) over the centred
    frequencies f of nufftfreqs(L), back to standard order."""
    dims = grid.ndim - 1
    L = np.atleast_1d(L).astype(int)
    tau = np.atleast_1d(tau).astype(float)
    spec = grid.astype(np.complex128)
    for ax in range(dims, 0, -1):
        spec = sfft.fft(spec, axis=ax, workers=workers)
    spec = np.fft.fftshift(spec, axes=tuple(range(1, dims + 1)))
    Mr = np.array(spec.shape[1:])
    start = np.ceil((Mr - L) / 2).astype(int)
    spec = spec[(slice(None),) + tuple(slice(start[a], start[a] + L[a]) for a in range(dims))]
    spec = spec / (n_points * ratio ** dims)
    freqs = [np.arange(int(np.fix(-La / 2)), La - int(np.fix(La / 2))) for La in L]
    ex = np.zeros(tuple(L))
    for a in range(dims):
        shape = [1] * dims
        shape[a] = L[a]
        ex = ex + tau[a] * (freqs[a].astype(float) ** 2).reshape(shape)
    kn = np.sqrt(np.prod(tau) / np.pi ** dims) * np.exp(-ex)
    kn = np.maximum(kn, np.finfo(float).tiny)
    spec = spec * (1.0 / kn)[None]
    return np.fft.ifftshift(spec, axes=tuple(range(1, dims + 1)))


def channel_spectra(xmod: np.ndarray, chans: np.ndarray, L, accuracy: int, n_points: int,
                    workers: int = 1) -> np.ndarray:
    """(C, *L) spectra of the channels at one accuracy (spreading + FFT)."""
    msp, tau, ratio = spread_params(L, accuracy)
    grid = spread_grid(xmod, chans, np.asarray(L) * ratio, msp, tau)
    if ratio > 1:
        return hermitian_part(nufft_spectra_oversampled(grid, n_points, L, ratio, tau, workers),
                              range(1, grid.ndim))
    return nufft_spectra(grid, n_points, workers)


def nufft_spectra(grid: np.ndarray, n_points: int, workers: int = 1) -> np.ndarray:
    """FFT of every channel over all axes, divided by the point count.

    nufftn_type1.py:701-711 (fft per axis, fftshift, / M) followed by the
    ifftshift of convolution.py:235-236; the shift pair cancels.
    """
    dims = grid.ndim - 1
    spec = grid.astype(np.complex128)
    for ax in range(dims, 0, -1):
        spec = sfft.fft(spec, axis=ax, workers=workers)
    return spec / n_points


# --------------------------------------------------------------------------
# Kernel-moment spectra -- convolution.py:318-794, design_matrix_optimized.py:30-298
# --------------------------------------------------------------------------
def design_powers(dims: int, order: int) -> List[Tuple[int, ...]]:
    """Polynomial term exponents (design_matrix_optimized.py:30-76)."""
    if order == 0:
        return [(0,) * dims]
    powers = []
    if dims == 1:
        for p in range(order + 1):
            powers.append((p,))
    elif dims == 2:
        for tot in range(order + 1):
            for px in range(tot, -1, -1):
                powers.append((px, tot - px))
    elif dims == 3:
        for tot in range(order + 1):
            for px in range(tot, -1, -1):
                for py in range(tot - px, -1, -1):
                    powers.append((px, py, tot - px - py))
    else:
        raise ValueError("dims > 3 not supported by the restatement")
    return powers


def design_pairs(nt: int) -> List[Tuple[int, int]]:
    """Lower-triangular pairs in column-major order (design_matrix_optimized.py:79-107)."""
    return [(i, j) for j in range(nt) for i in range(j, nt)]


def element_powers(dims: int, order: int) -> List[Tuple[int, ...]]:
    """Exponent of u for every packed S element: p_i + p_j."""
    pw = design_powers(dims, order)
    if order == 0:
        return [pw[0]]
    return [tuple(a + b for a, b in zip(pw[i], pw[j])) for i, j in design_pairs(len(pw))]


def kernel_grid_axes(x_scaled: np.ndarray, G) -> List[np.ndarray]:
    """Kernel evaluation grid: linspace(min, max, G) of the centred data (convolution.py:412-428)."""
    x = np.atleast_2d(x_scaled)
    return [np.linspace(x[:, d].min(), x[:, d].max(), int(G[d])) for d in range(x.shape[1])]


def radial_kernel(kernel_type: str, ssq: np.ndarray) -> np.ndarray:
    """K as a function of ||u||^2 (kernel.py:159-431), before the 1/det(h)."""
    kt = kernel_type.lower()
    eps = np.finfo(float).eps
    if kt in ("gauss", "gaussian", "normal"):
        return np.exp(-0.5 * ssq) * (1.0 / SQRT_2PI)
    if kt in ("gaussian_ft", "normal_ft"):
        return np.exp(-0.5 * ssq)
    if kt in ("epan", "epanechnikov"):
        return np.maximum(0.75 * (1.0 - ssq), eps)
    if kt == "tricube":
        r = np.sqrt(ssq)
        return np.maximum(eps, (70.0 / 81.0) * (1 - r ** 3) ** 3 * (r <= 1))
    if kt in ("quartic", "biweight"):
        return np.maximum(eps, (15.0 / 16.0) * (1 - ssq) ** 2 * (ssq <= 1))
    if kt == "triweight":
        return np.maximum(eps, (35.0 / 32.0) * (1 - ssq) ** 3 * (ssq <= 1))
    if kt in ("uniform", "rectangular"):
        return 0.5 * (np.sqrt(ssq) <= 1).astype(float)
    raise ValueError(f"Unknown kernel type: {kernel_type}")


def kernel_spectra(x_scaled, h, G, order: int, flag_power2: bool = True, workers: int = 1,
                   kernel_type: str = "gaussian"):
    """FFT of K(u) * u^a on the padded grid for every packed element and bandwidth.

    Returns (spectra list[ns] of (*L, H) complex128, params dict with L, qin,
    qout, h (filtered), ihbad).  Follows compute_kernel_fourier
    (convolution.py:318-652) with the kernels of kernel.py:159-431.
    """
    x = np.atleast_2d(np.asarray(x_scaled, dtype=float))
    h = np.atleast_2d(np.asarray(h, dtype=float))
    n, dims = x.shape
    G = np.atleast_1d(np.asarray(G, dtype=int))
    if G.size == 1:
        G = np.repeat(G, dims)
    L, qin, qout = grid_params(G, flag_power2)
    axes = kernel_grid_axes(x, G)
    mesh = np.meshgrid(*axes, indexing="ij")

    def _elements(hh):
        H = hh.shape[0]
        u = [mesh[d][..., None] / hh[None, :, d] for d in range(dims)]
        ssq = np.zeros(tuple(G) + (H,))
        for d in range(dims):
            ssq = ssq + u[d] ** 2
        kd = radial_kernel(kernel_type, ssq) / np.prod(hh, axis=1)
        elems = []
        for pw in element_powers(dims, order):
            e = kd
            for d in range(dims):
                if pw[d]:
                    e = e * u[d] ** pw[d]
            elems.append(e)
        return elems

    elems = _elements(h)
    sums0 = np.abs(np.sum(elems[0], axis=tuple(range(dims))))
    ihbad = sums0 < np.finfo(float).eps * 10
    if np.any(ihbad) and not np.all(ihbad):
        warnings.warn(f"{int(np.sum(ihbad))} bandwidth(s) are too small for this grid and will be removed",
                      stacklevel=2)
        elems = [e[..., ~ihbad] for e in elems]
        h = h[~ihbad]
    elif np.all(ihbad):
        hs = (4.0 / (dims + 2) / n) ** (1.0 / (dims + 4))
        warnings.warn(f"All bandwidths too small. Using Silverman's rule: h = {hs:.4f}", stacklevel=2)
        h = np.full((1, dims), hs)
        elems = _elements(h)
        ihbad = np.array([False])
    spectra = []
    for e in elems:
        pad = []
        for d in range(dims):
            before = (L[d] - G[d]) // 2 + 1
            pad.append((before, L[d] - G[d] - before))
        pad.append((0, 0))
        kp = np.pad(e, pad).astype(np.complex128)
        for d in range(dims):
            kp = sfft.fft(kp, axis=d, workers=workers)
        spectra.append(kp)
    return spectra, dict(L=L, qin=qin, qout=qout, h=h, ihbad=ihbad, G=G)


def hermitian_part(spec: np.ndarray, axes: Sequence[int]) -> np.ndarray:
    """(X[f] + conj(X[-f])) / 2 over the frequency `axes`.  The reference
    keeps the real part of the inverse transform of K X (K Hermitian);
    that real part is the inverse transform of K times this part of X, which
    makes the half-spectrum convolution below exact for spectra that are not
    Hermitian (the cropped oversampled spectra of accuracy >= 7)."""
    conj_neg = np.conj(spec)
    for ax in axes:
        conj_neg = np.roll(np.flip(conj_neg, axis=ax), 1, axis=ax)
    return 0.5 * (spec + conj_neg)


def convolve(spec_c: np.ndarray, kdf: np.ndarray, qout, G, real: bool = True, workers: int = 1):
    """nufft_convolve (convolution.py:907-951): product, inverse FFT per axis, crop.

    spec_c: (*L, C), kdf: (*L, H) -> (*G, H, C).  The reference forms the
    full product, inverts every axis and keeps the real part.  For Hermitian
    spectra (transforms of real grids; see hermitian_part) that real part is
    obtained from the half spectrum along the last axis: the leading axes are
    inverted on the kept columns and cropped, the last axis by a real inverse
    transform of length L.  Same values up to rounding, a third of the work.
    """
    dims = kdf.ndim - 1
    if not real:
        prod = kdf[..., :, None] * spec_c[..., None, :]
        for ax in range(dims):
            prod = sfft.ifft(prod, axis=ax, workers=workers, overwrite_x=True)
        sl = tuple(slice(qout[0, d], qout[0, d] + G[d]) for d in range(dims))
        return prod[sl]
    Ll = kdf.shape[dims - 1]
    half = (slice(None),) * (dims - 1) + (slice(0, Ll // 2 + 1),)
    prod = kdf[half][..., :, None] * spec_c[half][..., None, :]
    for ax in range(dims - 1):
        prod = sfft.ifft(prod, axis=ax, workers=workers, overwrite_x=True)
        crop = (slice(None),) * ax + (slice(qout[0, ax], qout[0, ax] + G[ax]),)
        prod = prod[crop]
    out = sfft.irfft(prod, n=Ll, axis=dims - 1, workers=workers)
    crop = (slice(None),) * (dims - 1) + (slice(qout[0, dims - 1], qout[0, dims - 1] + G[dims - 1]),)
    return out[crop]


# --------------------------------------------------------------------------
# Solve -- regression.py:162-277, lwp_formulas.py:12-14
# --------------------------------------------------------------------------
def solve_system(S: List[np.ndarray], T: List[np.ndarray], order: int, regularization: float,
                 lam: Optional[float] = None):
    """m = e1' (S + lambda I)^-1 T at every grid point.

    S: list[ns] of (*G, H); T: list[nt] of (*G, H, C).  Order 0 uses
    m = t / max(s, max(s) * reg) (regression.py:207-230).  For order >= 1,
    lambda = 1e-6 * max over all grid points and bandwidths of |diag S|
    (regression.py:243-267) unless ``lam`` is given.
    """
    if order == 0:
        s = S[0]
        thr = np.max(s) * regularization
        return T[0] / np.maximum(s, thr)[..., None], None
    nt = len(T)
    if lam is None:
        max_diag = 0.0
        for k in range(nt):
            di = k * nt - k * (k - 1) // 2
            max_diag = max(max_diag, float(np.max(np.abs(S[di]))))
        lam = 1e-6 * max_diag
    A = {}
    for k, (i, j) in enumerate(design_pairs(nt)):
        A[i, j] = A[j, i] = S[k] + (lam if i == j else 0.0)
    if nt > 4:
        # 2-D order 2: the reference's closed form reads a data file its
        # package does not ship (lwp_formulas.py:436-444); solve directly
        M = np.empty(S[0].shape + (nt, nt))
        for (i, j), v in A.items():
            M[..., i, j] = v
        beta = np.linalg.solve(M, np.stack(T, axis=-2))   # T: (*G, H, nt, C)
        return beta[..., 0, :], lam
    # Cramer's rule, the form of the reference's closed-form estimators
    # (lwp_formulas.py:133-380): the first row of (S + lambda I)^-1 is the
    # first column of cofactors over the determinant (S is symmetric)
    cof = [_cofactor0(A, nt, j) for j in range(nt)]
    det = sum(A[0, j] * cof[j] for j in range(nt))
    num = cof[0][..., None] * T[0]
    for j in range(1, nt):
        num += cof[j][..., None] * T[j]
    num /= det[..., None]
    return num, lam


def _det(A, rows, cols):
    """Determinant of the sub-matrix of the element arrays A[i, j]."""
    if len(rows) == 1:
        return A[rows[0], cols[0]]
    out = 0.0
    for k, c in enumerate(cols):
        sub = _det(A, rows[1:], cols[:k] + cols[k + 1:])
        out = out + (A[rows[0], c] * sub if k % 2 == 0 else -(A[rows[0], c] * sub))
    return out


def _cofactor0(A, nt, j):
    """Cofactor (0, j) of the nt x nt element arrays A."""
    rows = list(range(1, nt))
    cols = [c for c in range(nt) if c != j]
    m = _det(A, rows, cols)
    return m if j % 2 == 0 else -m


# --------------------------------------------------------------------------
# Linear interpolation on a uniform grid -- interp_optimized.py:60-78, 83-130
# --------------------------------------------------------------------------
def linear_interp(axes: Sequence[np.ndarray], values: np.ndarray, pts: np.ndarray) -> np.ndarray:
    """Clamped multilinear interpolation; values (*G, ...) -> (n, ...)."""
    pts = np.atleast_2d(pts)
    dims = len(axes)
    lib = _native()
    if lib is not None and not np.iscomplexobj(values) and dims <= 3 and \
            all(len(a) > 1 for a in axes):
        G = np.array([len(a) for a in axes], dtype=np.int64)
        extra = values.shape[dims:]
        K = int(np.prod(extra)) if extra else 1
        vals = np.ascontiguousarray(values, dtype=float).reshape(int(np.prod(G)), K)
        ax = np.array([[a[0], a[1] - a[0]] for a in axes], dtype=float).ravel()
        p = np.ascontiguousarray(pts, dtype=float)
        out = np.empty((p.shape[0], K))
        lib.oracle_interp(dims, p.shape[0], p.ctypes.data, G.ctypes.data, ax.ctypes.data, K,
                          vals.ctypes.data, out.ctypes.data)
        return out.reshape((p.shape[0],) + extra)
    idx, frac = [], []
    for d in range(dims):
        ax = axes[d]
        x0 = ax[0]
        dx = ax[1] - ax[0] if len(ax) > 1 else 1.0
        nx = len(ax)
        t = (pts[:, d] - x0) / dx
        i = np.floor(t).astype(np.int64)
        f = t - i
        lo = t < 0
        hi = t >= nx - 1
        i = np.where(lo, 0, np.where(hi, nx - 2, i))
        f = np.where(lo, 0.0, np.where(hi, 1.0, f))
        idx.append(i)
        frac.append(f)
    extra = values.shape[dims:]
    out = np.zeros((pts.shape[0],) + extra, dtype=np.result_type(values.dtype, np.float64))
    for corner in np.ndindex(*([2] * dims)):
        w = np.ones(pts.shape[0])
        ii = []
        for d, c in enumerate(corner):
            w = w * (frac[d] if c else (1.0 - frac[d]))
            ii.append(idx[d] + c)
        v = values[tuple(ii)]
        out += w.reshape((-1,) + (1,) * len(extra)) * v
    return out


def _interp(axes, values, pts, method):
    """GCV/DoF interpolation (api.py:594-600, api.py:651-657): linear, or the
    exact not-a-knot cubic spline that scipy's 'cubic' method builds."""
    if method == "linear":
        return linear_interp(axes, values, pts)
    if method == "cubic":
        return cubic_interp(axes, values, pts)
    raise ValueError(f"interpolation method {method!r} is not restated")


# --------------------------------------------------------------------------
# Selection -- api.py:73-164
# --------------------------------------------------------------------------
def one_se_rule(scores, errs, bandwidths, prefer_smaller: bool, dstd: float = 1.0) -> int:
    valid = np.isfinite(scores)
    if not np.any(valid):
        raise ValueError("All GCV scores are NaN or Inf. Regression failed for all bandwidths.")
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


def hutchinson_probes(n: int, num: int = 10, seed: int = 42) -> np.ndarray:
    """p = MT19937(seed).standard_normal((n, num)) (regression.py:1182-1194)."""
    return np.random.Generator(np.random.MT19937(seed)).standard_normal((n, num))


# --------------------------------------------------------------------------
# Shared preparation -- api.py:284-421, model.py:32-126, core.py:64-99
# --------------------------------------------------------------------------
def _as_column_matrix(x):
    """helpers.py:31-71: complex predictors become [real, imag] columns."""
    arr = np.asarray(x)
    if arr.ndim == 1:
        arr = arr[:, None]
    if np.iscomplexobj(arr):
        cc = np.any(arr.imag != 0, axis=0)
        arr = np.column_stack([arr.real, arr.imag[:, cc]]) if np.any(cc) else arr.real
    return arr.astype(float)


def _standardize(x):
    mean = x.mean(axis=0)
    std = x.std(axis=0, ddof=1)
    std[std == 0] = 1.0
    xs = (x - mean) / std
    center = (xs.max(axis=0) + xs.min(axis=0)) / 2
    return xs - center, mean, std, center


def _grid_shape(opts, n, dims):
    N = opts.get("N", None)
    if N is None:
        dn = int(np.ceil(n ** (1.0 / dims)))
        N = dn if dims == 1 else [dn] * dims
    if np.isscalar(N):
        N = [int(N)] * dims
    return np.array([int(v) for v in N])


def _raw_axes(x, G, opts):
    xr = opts.get("xrange", None)
    if xr is None:
        lo, hi = x.min(axis=0), x.max(axis=0)
    else:
        r = np.asarray(xr, dtype=float)
        lo, hi = r[:, 0], r[:, 1]
    return [np.linspace(lo[d], hi[d], int(G[d])) for d in range(x.shape[1])]


def _prepare_bandwidths(h, dims, opts, x):
    if h is None:
        scale = np.std(x, axis=0, ddof=1)
        scale[scale == 0] = 1.0
        rng = np.column_stack((0.1 * scale, scale))
        dh = opts.get("dh", None)
        if dh is None:
            dh = 20 if dims == 1 else [20] * dims
        bw = get_hlist(dh, rng)
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
                raise ValueError("Bandwidth array must have the same dimensionality as the input data.")
            bw = a.reshape(-1, dims)
    if not np.all(np.isfinite(bw)):
        raise ValueError("Bandwidth values must be finite (no NaN or Inf).")
    if np.any(bw <= 0):
        raise ValueError("Bandwidth values must be strictly positive.")
    return bw


# --------------------------------------------------------------------------
# cv_fastlpr -- api.py:167-832
# --------------------------------------------------------------------------
def cv_fastlpr(x, y, h=None, options: Optional[Dict] = None, workers: int = 1,
               h_chunk: int = 8, timings: Optional[Dict[str, float]] = None) -> Dict[str, object]:
    """Full GCV sweep; returns a dict with every output field and intermediates.

    ``timings`` (optional) accumulates wall seconds per phase: 'prep',
    'spread', 'fft', 'final' do not depend on the number of bandwidths;
    'kernel', 'conv', 'solve', 'interp' grow linearly with it.
    """
    import time as _time
    _t = [_time.perf_counter()]

    def _mark(name):
        now = _time.perf_counter()
        if timings is not None:
            timings[name] = timings.get(name, 0.0) + now - _t[0]
        _t[0] = now

    x = _as_column_matrix(x)
    y = np.asarray(y)
    if y.ndim == 1:
        y = y[:, None]
    elif y.ndim == 2 and y.shape[0] == 1 and y.shape[1] > 1:
        y = y.T
    n, dims = x.shape
    opts = dict(options or {})
    for k, v in dict(order=0, regularization=1e-8, num_dof_sample=10, kernel_type="gaussian",
                     y_type_out="mean", calc_dof=True, gcv_selection="first").items():
        opts.setdefault(k, v)
    if opts.get("accuracy") is None:
        opts["accuracy"] = max(6 - int(np.ceil(np.log10(n))), 4)
    acc = int(opts["accuracy"])
    order = int(opts["order"])
    reg = float(opts["regularization"])
    bw = _prepare_bandwidths(h, dims, opts, x)
    variance = str(opts["y_type_out"]) == "variance"
    y_raw = y.ravel().copy() if variance else None
    if variance:
        y = np.log(y + 1.0 / len(y))
    xs, mean, std, _ = _standardize(x)
    G = _grid_shape(opts, n, dims)
    axes_raw = _raw_axes(x, G, opts)
    flag_power2 = bool(opts.get("flag_power2", True))
    _mark("prep")
    kdf, prm = kernel_spectra(xs, bw, G, order, flag_power2, workers,
                              kernel_type=str(opts.get("kernel_type", "gaussian")))
    _mark("kernel")
    bw = prm["h"]
    H = bw.shape[0]
    L, qin, qout = prm["L"], prm["qin"], prm["qout"]
    xmod = knot_coordinates(xs, L, G, qin)

    y_complex = np.iscomplexobj(y)
    dy = y.shape[1]
    ycols = []
    for c in range(dy):
        ycols.append(y[:, c].real)
        if y_complex:
            ycols.append(y[:, c].imag)
    ycols = np.column_stack(ycols)
    calc_dof = bool(opts.get("calc_dof", True))
    if calc_dof:
        rm = opts.get("random_matrix", None)
        if rm is not None:
            p = np.asarray(rm, dtype=float)
            if p.shape[0] != n:
                raise ValueError("random_matrix has wrong shape")
        else:
            p = hutchinson_probes(n, int(opts.get("num_dof_sample", 10)), opts.get("dof_seed", 42))
        R = p.shape[1]
    else:
        p = np.zeros((n, 0))
        R = 0
    _mark("prep")
    # The user's accuracy applies to the response channels only (their
    # transform in nufft_regression_with_precomputed_kdf, api.py:640); the
    # design planes (compute_design_matrix, api.py:571) and the probes
    # (estimate_dof_nufft_vectorized, regression.py:756) use the default one.
    acc_default = max(6 - int(np.ceil(np.log10(n))), 4)
    grid = None
    if acc == acc_default:
        msp, tau, ratio = spread_params(L, acc)
        grid = spread_grid(xmod, np.column_stack([np.ones(n), ycols, p]),
                           np.asarray(L) * ratio, msp, tau)
        spec = (hermitian_part(nufft_spectra_oversampled(grid, n, L, ratio, tau, workers),
                               range(1, dims + 1)) if ratio > 1
                else nufft_spectra(grid, n, workers))
    else:
        s_ones_p = channel_spectra(xmod, np.column_stack([np.ones(n), p]), L, acc_default, n,
                                   workers)
        s_y = channel_spectra(xmod, ycols, L, acc, n, workers)
        spec = np.concatenate([s_ones_p[:1], s_y, s_ones_p[1:]], axis=0)
    _mark("spread")
    spec = np.moveaxis(spec, 0, -1)  # (*L, C)
    _mark("fft")

    nt = 1 if order == 0 else len(design_powers(dims, order))
    ns = len(kdf)
    Gt = tuple(G)
    S = [np.empty(Gt + (H,)) for _ in range(ns)]
    Tall = [np.empty(Gt + (H, spec.shape[-1] - 1)) for _ in range(nt)]
    for h0 in range(0, H, h_chunk):
        sl = slice(h0, min(H, h0 + h_chunk))
        for k in range(ns):
            S[k][..., sl] = convolve(spec[..., :1], kdf[k][..., sl], qout, G, True, workers)[..., 0]
        for i in range(nt):
            Tall[i][..., sl, :] = convolve(spec[..., 1:], kdf[i][..., sl], qout, G, True, workers)
    if order == 0:
        S[0] = S[0] + np.finfo(float).eps   # regression.py:116
    _mark("conv")
    m, lam = solve_system(S, Tall, order, reg)   # (*G, H, Cy + R)
    _mark("solve")
    ncy = ycols.shape[1]
    m_y_re = m[..., :ncy]
    if y_complex:
        m_y = m_y_re[..., 0::2] + 1j * m_y_re[..., 1::2]
    else:
        m_y = m_y_re
    m_p = m[..., ncy:]

    interp_default = "linear" if (dims == 1 or n >= 5000) else "cubic"
    out: Dict[str, object] = dict(S=S, T=Tall, m=m, lam=lam, spec=spec, grid=grid, xmod=xmod,
                                  L=L, qin=qin, qout=qout, G=G, bandwidths=bw, axes_raw=axes_raw,
                                  mean=mean, std=std, x_scaled=xs, opts=opts, probes=p)
    if not calc_dof:
        gv = m_y[..., 0, :] if H > 1 else m_y[..., 0, :]
        gv = gv[..., 0] if dy == 1 else gv
        yhat = _interp(axes_raw, gv, x, opts.get("interp_method", "linear"))
        sel = 0
        dof = dof_se = np.nan
        gcv_m = gcv_sd = np.array([np.nan])
        idmin = 0
        dof_all = dof_se_all = np.array([np.nan])
    else:
        dof_method = opts.get("dof_interp_method", interp_default)
        phat = _interp(axes_raw, m_p, x, dof_method).real  # (n, H, R)
        pp = np.sum(p * p, axis=0)
        pph = np.einsum("nr,nhr->rh", p, phat)
        tr = n * (pph / pp[:, None])
        tr = np.where(np.isnan(tr), n, tr)
        tr = np.clip(tr, 0.0, n)
        dof_all = np.mean(tr, axis=0)
        if R > 1:
            dof_se_all = np.std(tr, axis=0, ddof=1) / np.sqrt(R)
            pd = 1 - tr / n
            if y_complex:
                pd = 2 * pd - 1
            pdc = np.clip(pd, 0.0, 1.0)
            pen = 1.0 / np.maximum(pdc, 0.01) ** 2
            pen_std = np.std(pen, axis=0, ddof=1)
            pen_mean = np.mean(pen, axis=0)
            if y_complex:
                dof_all = n * (1 - np.mean(pdc, axis=0))
        else:
            dof_se_all = np.zeros(H)
            pen_std = np.zeros(H)
            pen_mean = None
        gcv_method = opts.get("gcv_interp_method", interp_default)
        yhat_all = _interp(axes_raw, m_y, x, gcv_method)   # (n, H, dy)
        agg = str(opts.get("gcv_selection", "first"))
        gcv_m = np.empty(H)
        gcv_sd = np.empty(H)
        rss_all = np.empty((H, dy))
        for ih in range(H):
            res = np.abs(y - yhat_all[:, ih, :]) ** 2
            rss = np.sum(res, axis=0)
            mse = rss / n
            rss_all[ih] = rss
            if pen_mean is not None:
                pen = float(pen_mean[ih])
            else:
                pdv = max(float(np.clip(1.0 - dof_all[ih] / n, 0.0, 1.0)), 0.01)
                pen = 1.0 / pdv ** 2
            g = mse * pen
            if agg == "first":
                sc, ms = float(g[0]), float(mse[0])
            elif agg == "average":
                sc, ms = float(np.mean(g)), float(np.mean(mse))
            elif agg == "sum":
                sc, ms = float(np.sum(g)), float(np.sum(mse))
            else:
                raise ValueError(f"Unknown aggregation method: {agg}")
            gcv_m[ih] = sc
            gcv_sd[ih] = ms * pen_std[ih] if pen_std[ih] > 0 else 0.0
        dstd = float(opts.get("dstd", 0.0))
        sel = one_se_rule(gcv_m, gcv_sd, bw, prefer_smaller=True, dstd=dstd)
        idmin = int(np.argmin(gcv_m))
        dof, dof_se = dof_all[sel], dof_se_all[sel]
        _mark("interp")
        gv = m_y[..., sel, :]
        gv = gv[..., 0] if dy == 1 else gv
        yhat = linear_interp(axes_raw, gv, x)
        out.update(rss=rss_all, pdot=pph, pp=pp, trace=tr, yhat_all=yhat_all)
    if dy == 1 and not calc_dof:
        pass
    s0 = S[0][..., sel]
    d_norm = None
    if variance:
        d_norm = 1.0 / ((1.0 / len(y_raw)) * np.sum(y_raw * np.exp(-yhat)))
        yhat = np.exp(yhat) / d_norm
        gv = np.exp(gv) / d_norm
    _mark("final")
    out.update(yhat=yhat, grid_values=gv, h_sel=bw[sel], id1se=int(sel), idmin=int(idmin),
               gcv_m=gcv_m, gcv_sd=gcv_sd, dof_all=dof_all, dof_stderr_all=dof_se_all,
               dof=dof, dof_stderr=dof_se, s0=s0, d=d_norm)
    return out


# --------------------------------------------------------------------------
# cv_fastkde -- api.py:835-1184
# --------------------------------------------------------------------------
def cv_fastkde(x, h=None, options: Optional[Dict] = None, workers: int = 1,
               h_chunk: int = 8) -> Dict[str, object]:
    x = _as_column_matrix(x)
    n, dims = x.shape
    if n < 2:
        raise ValueError(f"Input x must have at least 2 observations. Got {n} observations.")
    opts = dict(options or {})
    for k, v in dict(order=0, calc_dof=False, y_type_out="mean", kernel_type="gaussian",
                     verbose=False, dh=20).items():
        opts.setdefault(k, v)
    if opts.get("accuracy") is None:
        opts["accuracy"] = max(6 - int(np.ceil(np.log10(n))), 4)
    acc = int(opts["accuracy"])
    if opts.get("N") is None:
        an = int(np.ceil(n ** (1.0 / dims)))
        opts["N"] = [an] * dims if dims > 1 else an
    xs, mean, std, center = _standardize(x)
    bw = _prepare_bandwidths(h, dims, opts, x)
    G = np.atleast_1d(np.asarray(opts["N"] if isinstance(opts["N"], int) else
                                 (opts["N"][0] if dims == 1 else opts["N"]), dtype=int))
    if G.size == 1:
        G = np.repeat(G, dims)
    flag_power2 = bool(opts.get("flag_power2", True))
    kdf, prm = kernel_spectra(xs, bw, G, 0, flag_power2, workers,
                              kernel_type=str(opts.get("kernel_type", "gaussian")))
    bw = prm["h"]
    H = bw.shape[0]
    L, qin, qout = prm["L"], prm["qin"], prm["qout"]
    msp, tau, ratio = spread_params(L, acc)
    xmod = knot_coordinates(xs, L, G, qin)
    grid = spread_grid(xmod, np.ones((n, 1)), np.asarray(L) * ratio, msp, tau)
    if ratio > 1:
        spec = np.moveaxis(hermitian_part(nufft_spectra_oversampled(grid, n, L, ratio, tau,
                                                                    workers),
                                          range(1, dims + 1)), 0, -1)
    else:
        spec = np.moveaxis(nufft_spectra(grid, n, workers), 0, -1)
    s = np.empty(tuple(G) + (H,))
    for h0 in range(0, H, h_chunk):
        sl = slice(h0, min(H, h0 + h_chunk))
        s[..., sl] = convolve(spec, kdf[0][..., sl], qout, G, True, workers)[..., 0]
    s = s + np.finfo(float).eps
    ax_s = [np.linspace(xs.min(axis=0)[d], xs.max(axis=0)[d], G[d]) for d in range(dims)]
    xs_unc_min = ((x - mean) / std).min(axis=0)
    xs_unc_max = ((x - mean) / std).max(axis=0)
    ax_raw = [(ax_s[d] + (xs_unc_max[d] + xs_unc_min[d]) / 2) * std[d] + mean[d] for d in range(dims)]
    dxg = np.prod([a[1] - a[0] for a in ax_raw])
    dens = []
    for ih in range(H):
        sc = s[..., ih]
        tot = np.sum(sc) * dxg
        f = sc / tot if tot > 0 else sc
        dens.append(np.maximum(f, 0.0))
    lcv_m = np.empty(H)
    lcv_sd = np.empty(H)
    for ih in range(H):
        fa = linear_interp(ax_raw, dens[ih], x)
        k0 = (1.0 / SQRT_2PI) / np.prod(bw[ih])
        floo = np.maximum((n / (n - 1)) * (fa - k0 / n), 1e-10)
        lg = np.log(floo)
        lcv_m[ih] = float(np.sum(lg))
        lcv_sd[ih] = float(np.std(lg) * np.sqrt(n))
    sel = one_se_rule(lcv_m, lcv_sd, bw, prefer_smaller=False)
    return dict(fhat=dens[sel], fhat_all=np.stack(dens, axis=-1), h_sel=bw[sel], lcv_m=lcv_m,
                lcv_sd=lcv_sd, idmax=int(np.argmax(lcv_m)), id1se=int(sel), axes_raw=ax_raw,
                bandwidths=bw, S=s, spec=spec, grid=grid, L=L, qin=qin, qout=qout, G=G,
                mean=mean, std=std, x_scaled=xs)


# --------------------------------------------------------------------------
# Shared-data batch helpers -- batch.py:139-760
# --------------------------------------------------------------------------
def rgi_interp(axes: Sequence[np.ndarray], values: np.ndarray, pts: np.ndarray,
               method: str) -> np.ndarray:
    """scipy's RegularGridInterpolator(method, fill_value=None): 'linear'
    continues the edge cells beyond the grid (cell index clamped to
    [0, n - 2], fraction unclamped), 'cubic' is the not-a-knot spline with
    its end pieces extended."""
    pts = np.atleast_2d(pts)
    if method == "cubic":
        return cubic_interp(axes, values, pts)
    if method != "linear":
        raise ValueError(f"interpolation method {method!r} is not restated")
    dims = len(axes)
    idx, frac = [], []
    for d in range(dims):
        ax = np.asarray(axes[d], dtype=float)
        i = np.clip(np.searchsorted(ax, pts[:, d], side="right") - 1, 0, len(ax) - 2)
        idx.append(i)
        frac.append((pts[:, d] - ax[i]) / (ax[i + 1] - ax[i]))
    extra = values.shape[dims:]
    out = np.zeros((pts.shape[0],) + extra, dtype=np.result_type(values.dtype, np.float64))
    for corner in np.ndindex(*([2] * dims)):
        w = np.ones(pts.shape[0])
        ii = []
        for d, c in enumerate(corner):
            w = w * (frac[d] if c else (1.0 - frac[d]))
            ii.append(idx[d] + c)
        out += w.reshape((-1,) + (1,) * len(extra)) * values[tuple(ii)]
    return out


def batch_method(dims: int, opts: Dict, key: str) -> str:
    """batch.py:646-651 / 718-720: the option, else linear in 1-D, cubic otherwise."""
    return str(opts.get(key, "linear" if dims == 1 else "cubic"))


def batch_evaluate_at_points(x, y, h, options, eval_points, bandwidth_indices=None,
                             workers: int = 1) -> np.ndarray:
    """batch.py:595-669: the fitted grids of the chosen bandwidths evaluated
    at new points with RegularGridInterpolator (fill_value=None)."""
    o = cv_fastlpr(x, y, h, dict(options, calc_dof=False), workers=workers)
    m = o["m"]                                   # (*G, H, C)
    dims = len(o["G"])
    ny = (1 if np.asarray(y).ndim == 1 else np.asarray(y).shape[1])
    idx = list(range(m.shape[dims])) if bandwidth_indices is None else list(bandwidth_indices)
    vals = m[..., idx, :ny]
    vals = vals[..., 0] if ny == 1 else vals
    return rgi_interp(o["axes_raw"], vals, eval_points,
                      batch_method(dims, o["opts"], "interp_method"))


def compute_gcv_scores_batch(axes_raw, x_raw, y_raw, m_all, dof_all, dof_stderr_all,
                             penalty_std_all, opts) -> Tuple[np.ndarray, np.ndarray]:
    """batch.py:672-760 with compute_gcv (regression.py:280-471)."""
    dims = len(axes_raw)
    yhat = rgi_interp(axes_raw, np.asarray(m_all), x_raw,
                      batch_method(dims, opts, "gcv_interp_method"))
    y = np.asarray(y_raw)
    if y.ndim == 1:
        y = y[:, None]
    N = y.shape[0]
    agg = str(opts.get("gcv_selection", "first"))
    H = len(np.atleast_1d(dof_all))
    scores, errs = np.empty(H), np.empty(H)
    for k in range(H):
        yh = yhat[:, k] if yhat.ndim == 2 else yhat[:, k, :]
        yh = yh[:, None] if yh.ndim == 1 else yh
        mse = np.sum(np.abs(y - yh) ** 2, axis=0) / N
        pdof = float(np.clip(1.0 - float(np.atleast_1d(dof_all)[k]) / N, 0.0, 1.0))
        g = mse / max(pdof, 0.01) ** 2
        if agg == "first":
            s, ms = g[0], mse[0]
        elif agg == "average":
            s, ms = np.mean(g), np.mean(mse)
        else:
            s, ms = np.sum(g), np.sum(mse)
        ps = float(np.atleast_1d(penalty_std_all)[k])
        scores[k] = s
        errs[k] = ms * ps if ps > 0 else 0.0
    return scores, errs
