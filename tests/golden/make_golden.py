"""Generate the golden fixtures of tests/golden/ from the reference library.

Runs the reference's own CUDA build (oracle/_ref/libfmvd_ref.so: the upstream
deconvolution sources compiled for sm_100a with cuFFT) and the texture-object
restatement of its resampler (oracle/_ref/libfmvd_reftex.so) on small seeded
inputs, and writes inputs and outputs as .npz files.  Needs a GPU; run as

    python tests/golden/make_golden.py <output dir>

(then copy the .npz files into tests/golden/).

The fixtures pin the CPU oracle (oracle/fmvd_oracle.py) in the CPU tests.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gpu_deconvolution_b200 import synth  # noqa: E402

from oracle.ref_lib import load_ref, ref_deconvolve  # noqa: E402,F401


def rl_cases():
    """(name, views, weights, kernels, psf, iterations list, nstreams)"""
    cases = []
    rng = np.random.default_rng(7)
    # 16-bit, two views, non-uniform weights (with zeros), 9x9 kernels
    views, psfs, _, _ = synth.plain_rl_views(shape=(3, 40, 48), n_views=2, n_beads=12, ksize=9, sigma=(1.2, 2.5),
                                            seed=11)
    weights = [rng.uniform(0.0, 1.0, (40, 48)).astype(np.float32) for _ in range(2)]
    weights[0][:5, :7] = 0.0
    weights[1][:5, :7] = 0.0
    cases.append(("rl16_v2", views, weights, psfs, 0, [1, 4], 1))
    for t in (1, 2, 3):
        cases.append((f"rl16_psf{t}", views, weights, psfs, t, [2], 1))
    # 8-bit, three views
    v8, p8, w8, _ = synth.plain_rl_views(shape=(2, 33, 37), n_views=3, n_beads=8, ksize=7, sigma=(1.0, 2.0), seed=12,
                                         bits=8)
    cases.append(("rl8_v3", v8, list(w8), p8, 0, [3], 1))
    # non-square kernels (pins the swapped data-padding borders)
    rng2 = np.random.default_rng(13)
    gt = synth.bead_volume((2, 30, 50), 10, rng2)
    kns = [synth.gaussian_psf(5, 11, 2.0, 1.0, 0.0), synth.gaussian_psf(5, 11, 1.0, 1.5, 30.0)]
    vns = np.stack([synth.quantise(synth.blur_planes(gt, k), rng2) for k in kns])
    cases.append(("rl16_nonsquare", vns, [np.ones((30, 50), np.float32)] * 2, kns, 0, [2], 1))
    # saturated and dark regions: clip at 65535 and negative estimates
    rng3 = np.random.default_rng(14)
    gt = synth.bead_volume((2, 32, 32), 6, rng3, amp=(40000.0, 60000.0), background=0.0)
    ks = [synth.gaussian_psf(9, 9, 1.0, 1.0, 0.0)] * 2
    vs = np.stack([synth.quantise(synth.blur_planes(gt, k), rng3, noise=False) for k in ks])
    vs[:, :, 10:14, 10:14] = 65535
    cases.append(("rl16_extremes", vs, [np.ones((32, 32), np.float32)] * 2, ks, 0, [5], 1))
    return cases


def stream_cases():
    """Plane-streaming call pattern: fewer planes than streams, and more."""
    views, psfs, weights, _ = synth.plain_rl_views(shape=(4, 24, 24), n_views=2, n_beads=6, ksize=5, seed=21)
    return [("stream_d1_s3", views[:, :1], list(weights), psfs, 3), ("stream_d4_s3", views, list(weights), psfs, 3)]


def transform_cases():
    rng = np.random.default_rng(31)
    d, h, w = 20, 24, 28
    zz, yy, xx = np.meshgrid(np.arange(d), np.arange(h), np.arange(w), indexing="ij")
    src = (20000 + 15000 * np.sin(xx / 3.0) * np.cos(yy / 4.0) + 8000 * np.sin(zz / 2.5)).astype(np.float64)
    src += rng.normal(0, 2000, src.shape)
    src = np.clip(src, 0, 65535).astype(np.uint16)
    src[5:8, 5:8, 5:8] = 65535
    mats = []
    mats.append(np.array([1, 0, 0, 2.25, 0, 1, 0, -1.5, 0, 0, 1, 0.75], np.float32))
    mats.append(synth.rotation_y_inverse(90.0, (24, 20, 28), (d, h, w), 2.0, (0.3, -0.7, 0.2)))
    a = np.eye(3) + rng.normal(0, 0.15, (3, 3))
    mats.append(np.concatenate([a, rng.uniform(-2, 2, (3, 1))], axis=1).astype(np.float32).reshape(-1))
    return src, mats, (24, 20, 28)  # (td, th, tw)


def main(out_dir: str) -> None:
    os.makedirs(out_dir, exist_ok=True)
    lib, tex = load_ref()
    for name, views, weights, kernels, psf, its, ns in rl_cases():
        rec = {"views": views, "weights": np.stack(weights), "kernels": np.stack(kernels).astype(np.float32),
               "psf": psf}
        for it in its:
            r = ref_deconvolve(lib, views, weights, [k.copy() for k in kernels], psf, it, ns, True)
            rec[f"out_it{it}"] = r["out"]
            rec[f"est_it{it}"] = r["est"]
            rec["fft"] = np.array([r["fftH"], r["fftW"]])
            rec["kernels_normalised"] = r["kernels_normalised"]
        np.savez_compressed(os.path.join(out_dir, name + ".npz"), **rec)
        print("wrote", name)
    for name, views, weights, kernels, ns in stream_cases():
        r = ref_deconvolve(lib, views, weights, [k.copy() for k in kernels], 0, 2, ns, False)
        np.savez_compressed(os.path.join(out_dir, name + ".npz"), views=views, weights=np.stack(weights),
                            kernels=np.stack(kernels), nstreams=ns, out=r["out"], source_calls=r["source_calls"],
                            sink_calls=r["sink_calls"])
        print("wrote", name, r["source_calls"], r["sink_calls"])
    src, mats, (td, th, tw) = transform_cases()
    rec = {"src": src, "mats": np.stack(mats), "shape": np.array([td, th, tw])}
    for i, m in enumerate(mats):
        for bits in (16, 8):
            s = src if bits == 16 else (src >> 8).astype(np.uint8)
            out = np.zeros((td, th, tw), s.dtype)
            raw = np.zeros((td, th, tw), np.float32)
            r = tex.reftex_transform(bits, np.ascontiguousarray(s).ctypes.data, src.shape[2], src.shape[1],
                                     src.shape[0], tw, th, td, np.ascontiguousarray(m).ctypes.data, out.ctypes.data,
                                     raw.ctypes.data, None)
            assert r == 0, r
            rec[f"out{bits}_m{i}"] = out
            rec[f"raw{bits}_m{i}"] = raw
    # filter calibration: a single bright texel, sampled at fine offsets
    vol = np.zeros((1, 1, 4), np.uint16)
    vol[0, 0, 2] = 65535
    fx = np.arange(0, 4096, dtype=np.float64) / 4096.0
    coords = np.zeros((fx.size, 3), np.float32)
    coords[:, 0] = (1.5 + fx).astype(np.float32)
    coords[:, 1] = 0.5
    coords[:, 2] = 0.5
    vals = np.zeros(fx.size, np.float32)
    assert tex.reftex_probe(16, vol.ctypes.data, 4, 1, 1, coords.ctypes.data, vals.ctypes.data, fx.size) == 0
    rec["probe_coords"] = coords
    rec["probe_vals"] = vals
    # conversion of the fetched maximum: every texel 65535
    full = np.full((2, 2, 2), 65535, np.uint16)
    outf = np.zeros((1, 1, 1), np.uint16)
    ident = np.array([1, 0, 0, 0.5, 0, 1, 0, 0.5, 0, 0, 1, 0.5], np.float32)
    tex.reftex_transform(16, full.ctypes.data, 2, 2, 2, 1, 1, 1, ident.ctypes.data, outf.ctypes.data, None, None)
    rec["saturation_out"] = outf
    np.savez_compressed(os.path.join(out_dir, "transform.npz"), **rec)
    print("wrote transform; saturated fetch ->", int(outf[0, 0, 0]))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <output dir>")
    main(sys.argv[1])
