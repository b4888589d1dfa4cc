"""CPU restatement of the warm-start network (test infrastructure only).

The learned warm start has no counterpart in the reference; this module is
the FP64 numpy statement of what the GPU network computes, used by the tests
to check the tensor-core convolutions, their gradients and the whole
network's forward and backward passes.  Layouts follow the GPU: activations
NHWC, weights [Cout][taps][Cin] with tap t = 3 * (dy + 1) + (dx + 1).
"""
from __future__ import annotations

import numpy as np


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round float values to bfloat16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def tap_offsets(taps: int):
    if taps == 1:
        return [(0, 0)]
    return [(t // 3 - 1, t % 3 - 1) for t in range(9)]


def shift(x: np.ndarray, dy: int, dx: int) -> np.ndarray:
    """out[n, y, x] = x[n, y + dy, x + dx] with zeros outside the image."""
    N, H, W, C = x.shape
    out = np.zeros_like(x)
    ys = slice(max(0, -dy), min(H, H - dy))
    xs = slice(max(0, -dx), min(W, W - dx))
    yd = slice(max(0, dy), min(H, H + dy))
    xd = slice(max(0, dx), min(W, W + dx))
    out[:, ys, xs] = x[:, yd, xd]
    return out


def conv(x, w, bias=None, add=None, relu=False, mask=None):
    """out[p][co] = act(sum_t sum_ci x[p + off(t)][ci] w[co][t][ci] + bias + add)."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    cout, taps, cin = w.shape
    out = np.zeros(x.shape[:3] + (cout,))
    for t, (dy, dx) in enumerate(tap_offsets(taps)):
        out += shift(x, dy, dx) @ w[:, t, :].T
    if bias is not None:
        out += np.asarray(bias, np.float64)
    if add is not None:
        out += np.asarray(add, np.float64)
    if relu:
        out = np.maximum(out, 0.0)
    if mask is not None:
        out = np.where(np.asarray(mask) > 0, out, 0.0)
    return out


def conv_wgrad(g, x, taps):
    """dw[co][t][ci] = sum_p g[p][co] x[p + off(t)][ci]."""
    g = np.asarray(g, np.float64)
    x = np.asarray(x, np.float64)
    cout, cin = g.shape[-1], x.shape[-1]
    dw = np.zeros((cout, taps, cin))
    gf = g.reshape(-1, cout)
    for t, (dy, dx) in enumerate(tap_offsets(taps)):
        dw[:, t, :] = gf.T @ shift(x, dy, dx).reshape(-1, cin)
    return dw


def conv_dgrad_weights(w):
    """Weights of the data gradient: w'[ci][t][co] = w[co][taps - 1 - t][ci]
    (the transposed convolution is a convolution with the flipped kernel)."""
    w = np.asarray(w)
    return np.ascontiguousarray(w[:, ::-1, :].transpose(2, 1, 0))
