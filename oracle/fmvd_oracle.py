"""FP64 CPU oracle for the multi-view reconstruction path (TEST INFRASTRUCTURE).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs may
import it.  It restates, in float64 numpy, what the reference library computes
(bene51/gpu_deconvolution); every function cites the reference lines it follows.

Parity pinning: the reference ships no golden vectors or tests.  This oracle is
pinned against the reference's own CUDA build (``oracle/_ref``), run on a B200,
through the fixtures committed under ``tests/golden/`` (generated by
``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import numpy as np

PSF_INDEPENDENT = 0
PSF_EFFICIENT_BAYESIAN = 1
PSF_OPTIMIZATION_1 = 2
PSF_OPTIMIZATION_2 = 3


# --------------------------------------------------------------------------
# FFT sizing and clamp-to-border padding
# --------------------------------------------------------------------------
def align_up(a: int, b: int) -> int:
    """``iAlignUp`` (fmvd_deconvolve.cpp:22-26)."""
    return a - a % b + b if a % b else a


def snap_transform_size(n: int) -> int:
    """``snapTransformSize`` (fmvd_deconvolve.cpp:28-51): align to 16; keep a
    power of two; else the next power of two if <= 1024; else align to 512."""
    n = align_up(n, 16)
    hibit = n.bit_length() - 1
    if (1 << hibit) == n:
        return n
    hipot = 1 << (hibit + 1)
    if hipot <= 1024:
        return hipot
    return align_up(n, 512)


def clamp_map(n_fft: int, n_data: int, border: int) -> np.ndarray:
    """Source index for every padded index along one axis.

    The padding kernels (fmvd_deconvolve_cuda.cu:96-112, 222-238 and
    fmvd_deconvolve_cuda.impl.cu:39-55) copy index ``i < n_data`` as is,
    repeat the last sample for ``n_data <= i < n_data + border`` and use
    sample 0 beyond that.
    """
    i = np.arange(n_fft)
    return np.where(i < n_data, i, np.where(i < n_data + border, n_data - 1, 0))


def pad_clamp(img: np.ndarray, fftH: int, fftW: int, borderY: int, borderX: int) -> np.ndarray:
    dataH, dataW = img.shape
    my = clamp_map(fftH, dataH, borderY)
    mx = clamp_map(fftW, dataW, borderX)
    return img[my[:, None], mx[None, :]]


def pad_kernel(k: np.ndarray, fftH: int, fftW: int) -> np.ndarray:
    """``padKernel`` (fmvd_deconvolve.cu:13-68): zero-pad to fftH x fftW with
    the kernel centre (kH/2, kW/2) moved to (0, 0), wrapping around."""
    kH, kW = k.shape
    out = np.zeros((fftH, fftW), dtype=np.float64)
    ys = (np.arange(kH) - kH // 2) % fftH
    xs = (np.arange(kW) - kW // 2) % fftW
    out[ys[:, None], xs[None, :]] = k
    return out


def circ_conv(img: np.ndarray, kernel_spectrum: np.ndarray) -> np.ndarray:
    """Circular convolution on the padded domain, the cuFFT R2C -> multiply ->
    C2R sequence (fmvd_deconvolve.impl.cpp:264-271) in float64."""
    return np.fft.irfft2(np.fft.rfft2(img) * kernel_spectrum, s=img.shape)


# --------------------------------------------------------------------------
# Kernel preparation (plan time)
# --------------------------------------------------------------------------
def normalize(k: np.ndarray) -> np.ndarray:
    """``normalize`` (fmvd_deconvolve.cpp:53-68): double sum, float divide."""
    s = np.float32(np.sum(k.astype(np.float64)))
    return (k.astype(np.float32) / s).astype(np.float32)


def invert_kernel(k: np.ndarray) -> np.ndarray:
    """``computeInvertedKernel`` (fmvd_deconvolve.cpp:70-79): point mirror."""
    return k[::-1, ::-1].copy()


def convolve_single_plane(data: np.ndarray, kernel: np.ndarray) -> np.ndarray:
    """``convolve_single_plane`` (fmvd_deconvolve.cpp:90-137): clamp-to-border
    padded circular convolution of a small image, cropped back to its size."""
    dataH, dataW = data.shape
    kH, kW = kernel.shape
    fftH = snap_transform_size(dataH + kH - 1)
    fftW = snap_transform_size(dataW + kW - 1)
    padded = pad_clamp(data.astype(np.float64), fftH, fftW, kH // 2, kW // 2)
    spec = np.fft.rfft2(pad_kernel(kernel.astype(np.float64), fftH, fftW))
    return circ_conv(padded, spec)[:dataH, :dataW]


def compute_kernel2(kernels: list[np.ndarray], psf_type: int) -> list[np.ndarray]:
    """``computeKernel2`` (fmvd_deconvolve.cpp:139-204).  ``kernels`` are the
    caller's UNNORMALISED kernels; every result is normalised to sum 1."""
    n = len(kernels)
    out = []
    for v in range(n):
        kv = kernels[v].astype(np.float64)
        if psf_type == PSF_INDEPENDENT:
            k2 = invert_kernel(kv)
        elif psf_type == PSF_EFFICIENT_BAYESIAN:
            k2 = invert_kernel(kv)
            for w in range(n):
                if w == v:
                    continue
                t1 = convolve_single_plane(invert_kernel(kv), kernels[w])
                t1 = convolve_single_plane(t1, invert_kernel(kernels[w].astype(np.float64)))
                k2 = k2 * t1
        elif psf_type == PSF_OPTIMIZATION_1:
            k2 = invert_kernel(kv)
            for w in range(n):
                if w == v:
                    continue
                k2 = k2 * convolve_single_plane(invert_kernel(kv), kernels[w])
        elif psf_type == PSF_OPTIMIZATION_2:
            k2 = invert_kernel(kv ** n)
        else:
            raise ValueError(f"unknown psf type {psf_type}")
        out.append(k2 / np.sum(k2))
    return out


def prepare_weights(weights: list[np.ndarray], fftH: int, fftW: int, kH: int, kW: int) -> np.ndarray:
    """``prepareWeights`` (fmvd_deconvolve.impl.cpp:86-124) with ``padWeights``
    (fmvd_deconvolve_cuda.cu:71-157; borders kH/2 rows, kW/2 columns) and
    ``normalizeWeights`` (fmvd_deconvolve_cuda.cu:160-199; divide only where
    the view sum is > 0)."""
    padded = np.stack([pad_clamp(w.astype(np.float64), fftH, fftW, kH // 2, kW // 2) for w in weights])
    s = padded.sum(axis=0)
    return np.where(s > 0, padded / np.where(s > 0, s, 1.0), padded)


class Plan:
    """The state ``fmvd_initialize_cuda_*`` builds (fmvd_deconvolve.impl.cpp:130-203)."""

    def __init__(self, dataH, dataW, weights, kernels, psf_type, bits=16):
        self.dataH, self.dataW = dataH, dataW
        self.nViews = len(kernels)
        self.kH, self.kW = kernels[0].shape
        self.fftH = snap_transform_size(dataH + self.kH - 1)
        self.fftW = snap_transform_size(dataW + self.kW - 1)
        self.bits = bits
        k2 = compute_kernel2(kernels, psf_type)          # from the unnormalised kernels
        k1 = [np.asarray(k, np.float64) / np.sum(k) for k in kernels]
        self.K = [np.fft.rfft2(pad_kernel(k, self.fftH, self.fftW)) for k in k1]
        self.Khat = [np.fft.rfft2(pad_kernel(k, self.fftH, self.fftW)) for k in k2]
        self.W = prepare_weights(weights, self.fftH, self.fftW, self.kH, self.kW)

    def pad_data(self, view_plane: np.ndarray) -> np.ndarray:
        """Padded data of one view plane.  The launcher's parameters are named
        (kernelW, kernelH) but receive (kernelH, kernelW)
        (fmvd_deconvolve_cuda.impl.cu:76-77 vs fmvd_deconvolve.impl.cpp:36-37),
        so the row border is kW/2 and the column border kH/2."""
        return pad_clamp(view_plane.astype(np.float64), self.fftH, self.fftW, self.kW // 2, self.kH // 2)

    def initial_estimate(self) -> np.ndarray:
        """memset 0, then ``+= 10`` once per view (fmvd_deconvolve_cuda.impl.cu:62)."""
        return np.full((self.fftH, self.fftW), 10.0 * self.nViews)

    def iterate(self, e: np.ndarray, padded_views: list[np.ndarray], iterations: int) -> np.ndarray:
        """The RL loop (fmvd_deconvolve.impl.cpp:262-274): views are applied in
        order, each update written before the next view blurs the estimate."""
        for _ in range(iterations):
            for v in range(self.nViews):
                b = circ_conv(e, self.K[v])
                t = np.where(b > 1, padded_views[v] / np.where(b > 1, b, 1.0), b)   # divide_kernel quirk
                r = circ_conv(t, self.Khat[v])
                e = e + self.W[v] * (e * r - e)                                   # multiply32_kernel
        return e

    def deconvolve_plane(self, views: list[np.ndarray], iterations: int) -> np.ndarray:
        """Float estimate (fftH x fftW) after ``iterations`` for one z-plane."""
        pv = [self.pad_data(p) for p in views]
        return self.iterate(self.initial_estimate(), pv, iterations)

    def unpad(self, est: np.ndarray) -> np.ndarray:
        return unpad(est, self.dataH, self.dataW, self.bits)


def unpad(est: np.ndarray, dataH: int, dataW: int, bits: int = 16) -> np.ndarray:
    """``unpadData_kernel`` (fmvd_deconvolve_cuda.impl.cu:107-128): crop,
    clip at 2^bits - 1, truncate toward zero.  Negative values saturate to 0
    (float to unsigned conversion on the GPU saturates)."""
    mx = (1 << bits) - 1
    v = np.minimum(est[:dataH, :dataW], mx)
    v = np.trunc(np.maximum(v, 0.0))
    return v.astype(np.uint16 if bits == 16 else np.uint8)


def deconvolve_volume(views: np.ndarray, weights, kernels, psf_type: int, iterations: int, bits: int = 16,
                      return_float: bool = False):
    """Plane-wise deconvolution of ``views`` (V x D x H x W): what
    ``fmvd_deconvolve_planes_cuda_*`` returns through its sink, one plane per z."""
    V, D, H, W = views.shape
    plan = Plan(H, W, list(weights), list(kernels), psf_type, bits)
    outs, ests = [], []
    for z in range(D):
        est = plan.deconvolve_plane([views[v, z] for v in range(V)], iterations)
        outs.append(plan.unpad(est))
        if return_float:
            ests.append(est)
    out = np.stack(outs)
    if return_float:
        return out, np.stack(ests)
    return out


# --------------------------------------------------------------------------
# Affine resampling (transform) and the transformed weight mask
# --------------------------------------------------------------------------
def affine_coords(m: np.ndarray, x, y, z):
    """``rx = m0*x + m1*y + m2*z + m3`` etc. (fmvd_transform.impl.cu:41-43),
    evaluated in float32 as the device does."""
    m = np.asarray(m, np.float32)
    x = np.asarray(x, np.float32)
    y = np.asarray(y, np.float32)
    z = np.asarray(z, np.float32)
    rx = ((m[0] * x + m[1] * y) + m[2] * z) + m[3]
    ry = ((m[4] * x + m[5] * y) + m[6] * z) + m[7]
    rz = ((m[8] * x + m[9] * y) + m[10] * z) + m[11]
    return rx.astype(np.float32), ry.astype(np.float32), rz.astype(np.float32)


def texture_weight(coord: np.ndarray, frac_mode: str = "round"):
    """Texel index and 1/256-quantised weight of CUDA linear texture filtering
    for an unnormalised coordinate ``coord`` (texel centres at i + 0.5).

    The texture unit computes xB = coord - 0.5, i = floor(xB) and
    alpha = frac(xB) held in 9-bit fixed point with 8 fractional bits.
    """
    xb = coord.astype(np.float64) - 0.5
    i = np.floor(xb)
    a = xb - i
    if frac_mode == "round":
        aq = np.floor(a * 256.0 + 0.5) / 256.0        # nearest, halves up
    else:
        aq = np.floor(a * 256.0) / 256.0
    return i.astype(np.int64), aq


def transform_volume(src: np.ndarray, inv: np.ndarray, td: int, th: int, tw: int, bits: int = 16,
                     frac_mode: str = "round", out_float: bool = False):
    """``transform_cuda_*`` plane kernel (fmvd_transform.impl.cu:24-56,120-128):
    target voxel -> source coordinate by the 3x4 inverse, trilinear texture
    fetch at coord + 0.5 with border value 0, normalised by 2^bits - 1, then
    stored as (SAMPLE)(v * 2^bits + 0.5).  The weights are quantised to 1/256
    with round-half-up, as a one-axis probe of the B200 texture unit shows;
    the unit's rounding of other coordinates can differ by one 1/256 step,
    which is the tolerance parity is checked at."""
    d, h, w = src.shape
    maxv = float((1 << bits) - 1)
    zz, yy, xx = np.meshgrid(np.arange(td), np.arange(th), np.arange(tw), indexing="ij")
    rx, ry, rz = affine_coords(inv, xx, yy, zz)
    cx = (rx.astype(np.float64) + 0.5).astype(np.float32)
    cy = (ry.astype(np.float64) + 0.5).astype(np.float32)
    cz = (rz.astype(np.float64) + 0.5).astype(np.float32)
    ix, ax = texture_weight(cx, frac_mode)
    iy, ay = texture_weight(cy, frac_mode)
    iz, az = texture_weight(cz, frac_mode)
    srcf = src.astype(np.float64) / maxv

    def fetch(k, j, i):
        ok = (i >= 0) & (i < w) & (j >= 0) & (j < h) & (k >= 0) & (k < d)
        vals = srcf[np.clip(k, 0, d - 1), np.clip(j, 0, h - 1), np.clip(i, 0, w - 1)]
        return np.where(ok, vals, 0.0)

    v = np.zeros(rx.shape, np.float64)
    for dz in (0, 1):
        wz = az if dz else 1.0 - az
        for dy in (0, 1):
            wy = ay if dy else 1.0 - ay
            for dx in (0, 1):
                wx = ax if dx else 1.0 - ax
                v += wz * wy * wx * fetch(iz + dz, iy + dy, ix + dx)
    if out_float:
        return v
    # (SAMPLE)(v * 2^bits + 0.5): the device converts through a 32-bit
    # unsigned integer, so 2^bits wraps to 0 (measured on the B200 with the
    # texture restatement: a fetch of 1.0 gives 0)
    q = np.floor(v * float(1 << bits) + 0.5).astype(np.int64) % (1 << bits)
    return q.astype(np.uint16 if bits == 16 else np.uint8)


def transform_weight_sensitivity(src: np.ndarray, inv: np.ndarray, td: int, th: int, tw: int, bits: int = 16):
    """Per-voxel bound, in sample units, on how much the resampled value can
    move when each axis weight moves by one step of the texture unit's 1/256
    weight granularity: (1/256) * sum over axes of the largest texel
    difference along that axis within the voxel's 2x2x2 cell.  Used as the
    parity tolerance against the hardware texture path."""
    d, h, w = src.shape
    zz, yy, xx = np.meshgrid(np.arange(td), np.arange(th), np.arange(tw), indexing="ij")
    rx, ry, rz = affine_coords(inv, xx, yy, zz)
    ix = np.floor(rx.astype(np.float64)).astype(np.int64)
    iy = np.floor(ry.astype(np.float64)).astype(np.int64)
    iz = np.floor(rz.astype(np.float64)).astype(np.int64)
    s = src.astype(np.float64)

    def t(k, j, i):
        ok = (i >= 0) & (i < w) & (j >= 0) & (j < h) & (k >= 0) & (k < d)
        return np.where(ok, s[np.clip(k, 0, d - 1), np.clip(j, 0, h - 1), np.clip(i, 0, w - 1)], 0.0)

    c = {(a, b, e): t(iz + a, iy + b, ix + e) for a in (0, 1) for b in (0, 1) for e in (0, 1)}
    gx = np.max([np.abs(c[(a, b, 1)] - c[(a, b, 0)]) for a in (0, 1) for b in (0, 1)], axis=0)
    gy = np.max([np.abs(c[(a, 1, e)] - c[(a, 0, e)]) for a in (0, 1) for e in (0, 1)], axis=0)
    gz = np.max([np.abs(c[(1, b, e)] - c[(0, b, e)]) for b in (0, 1) for e in (0, 1)], axis=0)
    return (gx + gy + gz) / 256.0


def transformed_mask(inv: np.ndarray, z: int, w: int, h: int, d: int, zspacing: float,
                     tw: int, th: int, border: float) -> np.ndarray:
    """``create_transformed_mask_kernel`` (fmvd_transform.cu:19-67): 0 outside
    the source box, else the product of cosine ramps
    0.5 * (1 - cos(pi * dist / border)) over the axes closer than ``border``
    to an edge (the z distance scaled by ``zspacing``)."""
    yy, xx = np.meshgrid(np.arange(th), np.arange(tw), indexing="ij")
    rx, ry, rz = affine_coords(inv, xx, yy, np.full_like(xx, z))
    rx, ry, rz = rx.astype(np.float64), ry.astype(np.float64), rz.astype(np.float64)
    inside = (rx >= 0) & (rx < w) & (ry >= 0) & (ry < h) & (rz >= 0) & (rz < d)
    dx = np.where(rx < (w // 2), rx, w - rx)
    dy = np.where(ry < (h // 2), ry, h - ry)
    dz = np.where(rz < (d // 2), rz, d - rz) * zspacing
    v = np.ones_like(rx)
    for dist in (dx, dy, dz):
        ramp = 0.5 * (1.0 - np.cos(dist / border * np.pi))
        v = np.where(dist < border, v * ramp, v)
    return np.where(inside, v, 0.0)


# --------------------------------------------------------------------------
# Plane streaming call pattern (fmvd_deconvolve.impl.cpp:205-300)
# --------------------------------------------------------------------------
def plane_stats(a: np.ndarray, b: np.ndarray | None = None, rows: int | None = None,
                cols: int | None = None) -> np.ndarray:
    """FP64 per-plane sums of the convergence check (no reference
    counterpart): sum a, sum a^2, sum (a-b)^2, sum |a-b| over the top-left
    rows x cols of each plane."""
    a = np.asarray(a, np.float64)
    D, H, W = a.shape
    rows = H if rows is None else rows
    cols = W if cols is None else cols
    aa = a[:, :rows, :cols]
    out = np.zeros((D, 4))
    out[:, 0] = aa.sum(axis=(1, 2))
    out[:, 1] = (aa * aa).sum(axis=(1, 2))
    if b is not None:
        d = aa - np.asarray(b, np.float64)[:, :rows, :cols]
        out[:, 2] = (d * d).sum(axis=(1, 2))
        out[:, 3] = np.abs(d).sum(axis=(1, 2))
    return out


def streaming_call_counts(n_planes: int, n_streams: int) -> tuple[int, int]:
    """Number of datasource and datasink calls the reference driver makes for
    a source holding ``n_planes`` planes: it primes ``n_streams`` slots without
    looking at the return value, so fewer planes than slots still yields
    ``n_streams`` sink calls (the extra ones carry unfilled slots)."""
    returned = max(n_planes, n_streams)
    return returned + 1, returned
