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


# ----------------------------------------------------------------------------
# The whole network (same layer list, parameter order and bf16 storage points
# as the GPU model: activations and gradients are held in bf16 between
# layers, weights are used in bf16, the 1x1 output layer in FP32).
# ----------------------------------------------------------------------------
BASE = 32
PATCH_CHANNELS = 64


def layer_shapes(views: int, base: int = BASE):
    """(cin, cout, taps) of the 14 convolution layers in parameter order."""
    shapes = [(PATCH_CHANNELS, base, 1), (base, base, 9)]
    for l in range(1, 4):
        shapes += [(base << (l - 1), base << l, 9), (base << l, base << l, 9)]
    for l in (2, 1, 0):
        shapes += [(base << (l + 1), base << l, 9), (base << l, base << l, 9)]
    return shapes


def unpack(params: np.ndarray, views: int, base: int = BASE):
    layers, off = [], 0
    for cin, cout, taps in layer_shapes(views, base):
        w = params[off:off + cout * taps * cin].reshape(cout, taps, cin)
        off += cout * taps * cin
        b = params[off:off + cout]
        off += cout
        layers.append((w, b))
    out_w = params[off:off + base]
    out_b = params[off + base]
    assert off + base + 1 == params.size
    return layers, out_w, out_b


def _pool(x):
    N, H, W, C = x.shape
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2])


def _up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def _sum2(x):
    return x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2]


def input_patches(views: np.ndarray, q=bf16_round):
    """views: V x N x H x W samples -> (patches N x H x W x 64 in bf16, scale N)."""
    V, N, H, W = views.shape
    v = views.astype(np.float64)
    scale = (1.0 + v.mean(axis=(0, 2, 3))).astype(np.float32).astype(np.float64)
    norm = v / scale[None, :, None, None]
    chans = np.concatenate([norm, norm.mean(axis=0, keepdims=True)], axis=0).transpose(1, 2, 3, 0)
    col = np.zeros((N, H, W, PATCH_CHANNELS))
    for t, (dy, dx) in enumerate(tap_offsets(9)):
        col[..., t * (V + 1):(t + 1) * (V + 1)] = shift(chans, dy, dx)
    return q(col), scale


def _identity(a):
    return np.asarray(a, np.float64)


def network_forward(params: np.ndarray, views: np.ndarray, base: int = BASE, quantise: bool = True):
    """Estimate (N x H x W, sample units) and the intermediate tensors.
    quantise=False drops the bf16 rounding (exact FP64 network)."""
    q = bf16_round if quantise else _identity
    V = views.shape[0]
    layers, out_w, out_b = unpack(np.asarray(params, np.float64), V, base)
    wq = [(np.asarray(q(w), np.float64), b) for w, b in layers]
    col, scale = input_patches(views, q)
    c = {"col": col, "scale": scale}

    def layer(i, x, add=None):
        w, b = wq[i]
        return q(conv(x, w, b, add, relu=True))

    c["Ea0"] = layer(0, col)
    c["Eb0"] = layer(1, c["Ea0"])
    for l in range(1, 4):
        c[f"P{l - 1}"] = q(_pool(c[f"Eb{l - 1}"]))
        c[f"Ea{l}"] = layer(2 * l, c[f"P{l - 1}"])
        c[f"Eb{l}"] = layer(2 * l + 1, c[f"Ea{l}"])
    src = c["Eb3"]
    for l in (2, 1, 0):
        c[f"U{l}"] = _up(src)
        c[f"Da{l}"] = layer(8 + 2 * (2 - l), c[f"U{l}"], c[f"Eb{l}"])
        c[f"Db{l}"] = layer(9 + 2 * (2 - l), c[f"Da{l}"])
        src = c[f"Db{l}"]
    y = c["Db0"] @ out_w + out_b
    c["y"] = y
    return y * scale[:, None, None], c


def network_grads(params: np.ndarray, views: np.ndarray, target: np.ndarray, base: int = BASE,
                  quantise: bool = True):
    """Mean L1 loss (normalised units) and the gradient of every parameter,
    in the GPU's parameter order."""
    q = bf16_round if quantise else _identity
    V = views.shape[0]
    params = np.asarray(params, np.float64)
    layers, out_w, out_b = unpack(params, V, base)
    wq = [np.asarray(q(w), np.float64) for w, _ in layers]
    _, c = network_forward(params, views, base, quantise)
    scale = c["scale"]
    t = np.asarray(target, np.float64) / scale[:, None, None]
    d = c["y"] - t
    count = d.size
    loss = np.abs(d).sum() / count
    gy = np.sign(d) / count
    grads = [None] * len(layers)

    def back(i, g, x, mask):
        """weight and bias gradient of layer i from its output gradient g
        (already masked) and input x; returns the input gradient."""
        w = wq[i]
        grads[i] = (conv_wgrad(g, x, w.shape[1]), g.sum(axis=(0, 1, 2)))
        if mask is None and i == 0:
            return None
        gi = conv(g, conv_dgrad_weights(w))
        if mask is not None:
            gi = np.where(mask > 0, gi, 0.0)
        return q(gi)

    g_out_w = np.einsum("nhw,nhwc->c", gy, c["Db0"])
    g_out_b = gy.sum()
    g = q(np.where(c["Db0"] > 0, gy[..., None] * out_w, 0.0))
    g_skip = {}
    for l in (0, 1, 2):
        gDa = back(9 + 2 * (2 - l), g, c[f"Da{l}"], c[f"Da{l}"])
        gU = back(8 + 2 * (2 - l), gDa, c[f"U{l}"], None)
        g_skip[l] = gDa
        src = c["Eb3"] if l == 2 else c[f"Db{l + 1}"]
        g = q(np.where(src > 0, _sum2(gU), 0.0))
    for l in (3, 2, 1, 0):
        if l < 3:
            g = q(np.where(c[f"Eb{l}"] > 0, 0.25 * _up(gP) + g_skip[l], 0.0))
        gEa = back(2 * l + 1, g, c[f"Ea{l}"], c[f"Ea{l}"])
        x_in = c["col"] if l == 0 else c[f"P{l - 1}"]
        gP = back(2 * l, gEa, x_in, None) if l > 0 else None
        if l == 0:
            back(0, gEa, x_in, None)
        g = None
    flat = []
    for (dw, db) in grads:
        flat += [dw.reshape(-1), db.reshape(-1)]
    flat += [g_out_w, np.array([g_out_b])]
    return loss, np.concatenate(flat)
