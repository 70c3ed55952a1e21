"""Test infrastructure: CPU restatement of the learned bandwidth proposal.

Nothing here is called by the product: the tests use it as the checker of
the CUDA MLP kernels (``flpr_mlp_fwd`` / ``flpr_mlp_bwd`` / ``flpr_mlp_step``)
and of the binned moment sums (``flpr_bin_moments``).  The reference has no
learned component, so these restate the definitions the C ABI documents:

* dense ReLU network h_{l+1} = relu(h_l W_l^T + b_l), no ReLU on the last
  layer, W_l stored (out, in); products take BF16-rounded operands and
  accumulate in (at least) FP32, exactly where the kernels round;
* Adam with bias correction and an L2 term added to the gradient;
* per-cell count, sum y and sum y^2 on a 4096-cell grid over [min, max]
  (4096 bins in 1-D, 64 x 64 in 2-D).
"""
from __future__ import annotations

import numpy as np

CELLS = 4096


def bins_per_axis(d: int) -> int:
    return 4096 if d == 1 else 64


def to_bf16(a) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), returned
    as float32."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    bias = 0x7FFF + ((u >> 16) & 1)
    r = ((u + bias) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(f.shape)


def unpack(params: np.ndarray, dims):
    """Split a packed parameter vector into [(W_l, b_l)]."""
    out, o = [], 0
    for l in range(len(dims) - 1):
        n_in, n_out = dims[l], dims[l + 1]
        W = params[o:o + n_out * n_in].reshape(n_out, n_in)
        o += n_out * n_in
        b = params[o:o + n_out]
        o += n_out
        out.append((W, b))
    return out


def forward(params32: np.ndarray, dims, x: np.ndarray):
    """Forward pass with the kernels' roundings.  Returns (out fp32 (B, dims[-1]),
    list of BF16-rounded layer inputs h_0..h_{L-1})."""
    layers = unpack(np.asarray(params32, np.float32), dims)
    h = to_bf16(x)
    hs = [h]
    for l, (W, b) in enumerate(layers):
        z = h.astype(np.float64) @ to_bf16(W).astype(np.float64).T + b.astype(np.float64)
        if l == len(layers) - 1:
            return z.astype(np.float32), hs
        h = to_bf16(np.maximum(z, 0.0).astype(np.float32))
        hs.append(h)
    raise AssertionError("unreachable")


def backward(params32: np.ndarray, dims, hs, dout: np.ndarray) -> np.ndarray:
    """Gradient of sum(dout * out) for every parameter (packed like the
    parameters), with BF16 rounding of the propagated gradients as in
    flpr_mlp_bwd."""
    layers = unpack(np.asarray(params32, np.float32), dims)
    grads = [None] * len(layers)
    dz32 = np.asarray(dout, np.float32).astype(np.float64)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        dz16 = to_bf16(dz32.astype(np.float32)).astype(np.float64)
        dW = dz16.T @ hs[l].astype(np.float64)
        db = dz32.sum(axis=0)
        grads[l] = (dW, db)
        if l == 0:
            break
        dh = dz16 @ to_bf16(W).astype(np.float64)
        dz32 = np.where(hs[l] > 0, dh, 0.0).astype(np.float32).astype(np.float64)
    return np.concatenate([np.concatenate([g[0].ravel(), g[1]]) for g in grads]).astype(np.float32)


def forward_exact(params: np.ndarray, dims, x: np.ndarray) -> np.ndarray:
    """Float64 forward pass without any rounding (for finite differences)."""
    h = np.asarray(x, np.float64)
    layers = unpack(np.asarray(params, np.float64), dims)
    for l, (W, b) in enumerate(layers):
        h = h @ W.T + b
        if l < len(layers) - 1:
            h = np.maximum(h, 0.0)
    return h


def backward_exact(params: np.ndarray, dims, x: np.ndarray, dout: np.ndarray) -> np.ndarray:
    """Float64 gradient of sum(dout * out) without rounding."""
    layers = unpack(np.asarray(params, np.float64), dims)
    hs = [np.asarray(x, np.float64)]
    for l, (W, b) in enumerate(layers[:-1]):
        hs.append(np.maximum(hs[-1] @ W.T + b, 0.0))
    grads = [None] * len(layers)
    dz = np.asarray(dout, np.float64)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        grads[l] = (dz.T @ hs[l], dz.sum(axis=0))
        if l == 0:
            break
        dz = np.where(hs[l] > 0, dz @ W, 0.0)
    return np.concatenate([np.concatenate([g[0].ravel(), g[1]]) for g in grads])


def adam(p, g, m, v, lr, b1, b2, eps, wd, step):
    """One Adam step (float32), as flpr_mlp_step."""
    p, g, m, v = (np.asarray(a, np.float32).copy() for a in (p, g, m, v))
    g = g + np.float32(wd) * p
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    c1 = np.float32(1 - b1 ** step)
    c2 = np.float32(1 - b2 ** step)
    p = p - np.float32(lr) * (m / c1) / (np.sqrt(v / c2) + np.float32(eps))
    return p, m, v


def bin_moments(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """(3, 4096): count, sum y, sum y^2 per cell over [min, max] (flpr_bin_moments)."""
    x = np.asarray(x, np.float64)
    if x.ndim == 1:
        x = x[:, None]
    n, d = x.shape
    bins = bins_per_axis(d)
    cell = np.zeros(n, dtype=np.int64)
    for a in range(d):
        lo, hi = x[:, a].min(), x[:, a].max()
        scale = bins / (hi - lo) if hi > lo else 0.0
        b = np.clip(np.floor((x[:, a] - lo) * scale).astype(np.int64), 0, bins - 1)
        cell = cell * bins + b
    cells = CELLS
    y = np.asarray(y, np.float64)
    return np.stack([np.bincount(cell, minlength=cells).astype(np.float64),
                     np.bincount(cell, weights=y, minlength=cells),
                     np.bincount(cell, weights=y * y, minlength=cells)])
