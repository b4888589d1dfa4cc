"""Seeded synthetic multi-view data shaped like the benchmark workloads.

No public dataset is used: ground truth is a field of Gaussian beads (and
optionally smooth ellipsoidal shells) on a constant background; each view is a
per-plane 2-D convolution with an anisotropic, rotated Gaussian PSF, with
Poisson noise, quantised to unsigned 16 (or 8) bit.
"""
from __future__ import annotations

import numpy as np


def gaussian_psf(size_y: int, size_x: int, sigma_x: float, sigma_y: float, angle_deg: float) -> np.ndarray:
    """Normalised anisotropic 2-D Gaussian, major axis rotated by ``angle_deg``."""
    yy, xx = np.meshgrid(np.arange(size_y) - size_y // 2, np.arange(size_x) - size_x // 2, indexing="ij")
    a = np.deg2rad(angle_deg)
    u = np.cos(a) * xx + np.sin(a) * yy
    v = -np.sin(a) * xx + np.cos(a) * yy
    k = np.exp(-0.5 * ((u / sigma_x) ** 2 + (v / sigma_y) ** 2))
    return (k / k.sum()).astype(np.float32)


def bead_volume(shape, n_beads: int, rng: np.random.Generator, sigma: float = 1.0,
                amp=(500.0, 2000.0), background: float = 100.0, shells: int = 0,
                shell_value: float = 300.0) -> np.ndarray:
    """Float32 volume (D, H, W): ``n_beads`` Gaussian beads of width ``sigma``
    and amplitude U[amp] on ``background``, plus ``shells`` ellipsoidal shells."""
    D, H, W = shape
    vol = np.full(shape, background, np.float32)
    r = int(np.ceil(3 * sigma))
    g = np.arange(-r, r + 1)
    gz, gy, gx = np.meshgrid(g, g, g, indexing="ij")
    zs = rng.integers(0, D, n_beads)
    ys = rng.integers(0, H, n_beads)
    xs = rng.integers(0, W, n_beads)
    amps = rng.uniform(amp[0], amp[1], n_beads).astype(np.float32)
    blob = np.exp(-0.5 * (gz ** 2 + gy ** 2 + gx ** 2) / sigma ** 2).astype(np.float32)
    for z, y, x, a in zip(zs, ys, xs, amps):
        z0, z1 = max(z - r, 0), min(z + r + 1, D)
        y0, y1 = max(y - r, 0), min(y + r + 1, H)
        x0, x1 = max(x - r, 0), min(x + r + 1, W)
        vol[z0:z1, y0:y1, x0:x1] += a * blob[z0 - z + r:z1 - z + r, y0 - y + r:y1 - y + r, x0 - x + r:x1 - x + r]
    if shells:
        zz = np.arange(D, dtype=np.float32)[:, None, None]
        yy = np.arange(H, dtype=np.float32)[None, :, None]
        xx = np.arange(W, dtype=np.float32)[None, None, :]
        for _ in range(shells):
            c = rng.uniform(0.3, 0.7, 3) * np.array([D, H, W])
            radii = rng.uniform(0.15, 0.3, 3) * np.array([D, H, W])
            rho = np.sqrt(((zz - c[0]) / radii[0]) ** 2 + ((yy - c[1]) / radii[1]) ** 2 + ((xx - c[2]) / radii[2]) ** 2)
            vol += shell_value * np.exp(-0.5 * ((rho - 1.0) / 0.05) ** 2).astype(np.float32)
    return vol


def blur_planes(vol: np.ndarray, psf: np.ndarray) -> np.ndarray:
    """Per-plane 2-D 'same' convolution (zero boundary) via FFT."""
    D, H, W = vol.shape
    kH, kW = psf.shape
    fh, fw = H + kH - 1, W + kW - 1
    ks = np.fft.rfft2(psf, s=(fh, fw))
    out = np.empty_like(vol)
    for z in range(D):
        full = np.fft.irfft2(np.fft.rfft2(vol[z], s=(fh, fw)) * ks, s=(fh, fw))
        out[z] = full[kH // 2:kH // 2 + H, kW // 2:kW // 2 + W]
    return out


def quantise(vol: np.ndarray, rng: np.random.Generator, bits: int = 16, noise: bool = True) -> np.ndarray:
    v = rng.poisson(np.maximum(vol, 0)).astype(np.float64) if noise else vol
    mx = (1 << bits) - 1
    return np.clip(np.rint(v), 0, mx).astype(np.uint16 if bits == 16 else np.uint8)


def plain_rl_views(shape=(64, 256, 256), n_views: int = 2, n_beads: int = 200, ksize: int = 17,
                   sigma=(1.5, 4.0), angles=None, seed: int = 0, bits: int = 16):
    """Views, PSFs and equal weights in the shape of the small plain-RL
    workload: two views of a 256 x 256 x 64 bead field, 17 x 17 PSFs of
    sigma 1.5 x 4.0 px rotated 0 and 90 degrees."""
    rng = np.random.default_rng(seed)
    gt = bead_volume(shape, n_beads, rng)
    if angles is None:
        angles = [180.0 * v / n_views for v in range(n_views)]
    psfs = [gaussian_psf(ksize, ksize, sigma[0], sigma[1], a) for a in angles]
    views = np.stack([quantise(blur_planes(gt, p), rng, bits) for p in psfs])
    weights = np.ones((n_views,) + shape[1:], np.float32)
    return views, psfs, weights, gt


def rotation_y_inverse(angle_deg: float, frame_shape, src_shape, zscale: float, shift) -> np.ndarray:
    """3x4 row-major target->source matrix: rotate the common frame about the
    y axis through its centre by ``angle_deg``, then map z onto the source's
    coarser z sampling (``zscale`` target planes per source plane) and shift."""
    D, H, W = frame_shape
    d, h, w = src_shape
    a = np.deg2rad(angle_deg)
    c = np.array([W / 2.0, H / 2.0, D / 2.0])
    cs = np.array([w / 2.0, h / 2.0, d * zscale / 2.0])
    R = np.array([[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]])
    S = np.diag([1.0, 1.0, 1.0 / zscale])
    M = S @ R
    t = S @ (cs - R @ c) + np.asarray(shift, np.float64) * np.array([1.0, 1.0, 1.0 / zscale])
    return np.concatenate([M, t[:, None]], axis=1).astype(np.float32).reshape(-1)


# ----------------------------------------------------------------------------
# Many uneven volumes (the batched workload): specifications on the host,
# views generated on the GPU with torch (the same model as above: beads on a
# background, per-plane blur, Poisson noise at a given peak).
# ----------------------------------------------------------------------------
BATCH_PLANE_SIZES = (128, 192, 256, 384, 512, 768, 1024)


def batched_specs(seed: int = 0, count: int = 32, sizes=BATCH_PLANE_SIZES, depth=(16, 256), views=(2, 6),
                  ksize=(9, 41), iterations: int = 25) -> list[dict]:
    """Per-volume parameters: square planes from ``sizes``, depth U[depth],
    views U[views], odd kernel size U[ksize], sigma_x U[0.8, 2], sigma_y
    U[2, 6], a random in-plane angle per view, Poisson peak U[200, 5000]."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(rng.choice(sizes))
        k = int(rng.integers(ksize[0] // 2, ksize[1] // 2 + 1)) * 2 + 1
        V = int(rng.integers(views[0], views[1] + 1))
        specs.append({
            "index": i, "H": n, "W": n, "D": int(rng.integers(depth[0], depth[1] + 1)), "V": V, "k": k,
            "sigma": [[float(rng.uniform(0.8, 2.0)), float(rng.uniform(2.0, 6.0))] for _ in range(V)],
            "angle": [float(rng.uniform(0.0, 180.0)) for _ in range(V)],
            "peak": float(rng.uniform(200.0, 5000.0)), "iterations": iterations, "seed": int(rng.integers(1 << 30)),
        })
    return specs


def spec_psfs(spec: dict) -> list[np.ndarray]:
    k = spec["k"]
    return [gaussian_psf(k, k, s[0], s[1], a) for s, a in zip(spec["sigma"], spec["angle"])]


def bead_volume_torch(D, H, W, seed, device="cuda", density=5e-5, amp=(500.0, 2000.0), background=100.0,
                      sigma=1.0):
    """Ground truth on the GPU: Gaussian beads (width ``sigma`` voxels,
    amplitude U[amp]) at ``density`` beads per voxel on ``background``."""
    import torch
    g = torch.Generator(device=device).manual_seed(int(seed))
    gt = torch.zeros((D, H, W), dtype=torch.float32, device=device)
    n = max(1, int(density * D * H * W))
    idx = torch.randint(0, D * H * W, (n,), device=device, generator=g)
    a = torch.empty(n, device=device).uniform_(amp[0], amp[1], generator=g)
    gt.view(-1).index_add_(0, idx, a)
    r = int(np.ceil(3 * sigma))
    t = torch.arange(-r, r + 1, device=device, dtype=torch.float32)
    b = torch.exp(-0.5 * (t / sigma) ** 2)
    k = 2 * r + 1
    x = gt[None, None]
    x = torch.nn.functional.conv3d(x, b.view(1, 1, k, 1, 1), padding=(r, 0, 0))
    x = torch.nn.functional.conv3d(x, b.view(1, 1, 1, k, 1), padding=(0, r, 0))
    x = torch.nn.functional.conv3d(x, b.view(1, 1, 1, 1, k), padding=(0, 0, r))
    return x[0, 0] + background, g


def add_shells_torch(gt, n_shells: int, seed: int, value: float = 300.0, planes_per_chunk: int = 16):
    """Adds ``n_shells`` smooth ellipsoidal shells of peak ``value`` to the
    D x H x W CUDA volume ``gt`` in place (the shells of ``bead_volume``,
    evaluated a few planes at a time)."""
    import torch
    D, H, W = gt.shape
    rng = np.random.default_rng(seed)
    dev = gt.device
    yy = torch.arange(H, device=dev, dtype=torch.float32)[None, :, None]
    xx = torch.arange(W, device=dev, dtype=torch.float32)[None, None, :]
    for _ in range(n_shells):
        c = rng.uniform(0.3, 0.7, 3) * np.array([D, H, W])
        radii = rng.uniform(0.15, 0.3, 3) * np.array([D, H, W])
        for z0 in range(0, D, planes_per_chunk):
            z1 = min(z0 + planes_per_chunk, D)
            zz = torch.arange(z0, z1, device=dev, dtype=torch.float32)[:, None, None]
            rho = torch.sqrt(((zz - c[0]) / radii[0]) ** 2 + ((yy - c[1]) / radii[1]) ** 2 +
                             ((xx - c[2]) / radii[2]) ** 2)
            gt[z0:z1] += value * torch.exp(-0.5 * ((rho - 1.0) / 0.05) ** 2)
    return gt


def blur_noise_torch(gt, psfs, g, bits: int = 16):
    """V x D x H x W views of ``gt``: per-plane 'same' convolution with each
    PSF, Poisson noise, quantised (int16 holding uint16 bits, or uint8)."""
    import torch
    D, H, W = gt.shape
    V = len(psfs)
    device = gt.device
    out = torch.empty((V, D, H, W), dtype=torch.int16 if bits == 16 else torch.uint8, device=device)
    mx = (1 << bits) - 1
    for v, psf in enumerate(psfs):
        kH, kW = psf.shape
        fh, fw = H + kH - 1, W + kW - 1
        ks = torch.fft.rfft2(torch.from_numpy(np.ascontiguousarray(psf)).to(device), s=(fh, fw))
        for z0 in range(0, D, 32):
            z1 = min(z0 + 32, D)
            full = torch.fft.irfft2(torch.fft.rfft2(gt[z0:z1], s=(fh, fw)) * ks, s=(fh, fw))
            blurred = full[:, kH // 2:kH // 2 + H, kW // 2:kW // 2 + W].clamp_min(0)
            noisy = torch.poisson(blurred, generator=g).clamp(0, mx).round()
            out[v, z0:z1] = noisy.to(torch.int32).to(torch.int16) if bits == 16 else noisy.to(torch.uint8)
    return out


def views_torch(spec: dict, device="cuda", bits: int = 16, bead_density: float = 5e-5):
    """V x D x H x W views of one volume on the GPU (torch int16 holding
    uint16 bits for 16-bit samples, uint8 otherwise)."""
    gt, g = bead_volume_torch(spec["D"], spec["H"], spec["W"], spec["seed"], device, bead_density)
    gt = (gt - 100.0) * (spec["peak"] / float((gt - 100.0).max().clamp_min(1e-6))) * 0.9 + 0.1 * spec["peak"]
    return blur_noise_torch(gt, spec_psfs(spec), g, bits)


def warm_start_views_torch(D, H=512, W=512, views=4, seed=0, ksize=17, sigma=(1.5, 4.0), device="cuda"):
    """Training and test planes of the learned warm start: the small plain-RL
    generator (beads of width 1 voxel, amplitude U[500, 2000] on background
    100; 17 x 17 PSFs of sigma 1.5 x 4.0 px; Poisson noise; uint16) at
    H x W with ``views`` PSF orientations 180 v / views degrees.  Returns
    (views V x D x H x W int16, ground truth D x H x W float32, PSFs)."""
    psfs = [gaussian_psf(ksize, ksize, sigma[0], sigma[1], 180.0 * v / views) for v in range(views)]
    density = 200.0 / (256 * 256 * 64)
    gt, g = bead_volume_torch(D, H, W, seed, device, density)
    return blur_noise_torch(gt, psfs, g), gt, psfs
