"""CPU tests of the oracle: pinned against the reference's own CUDA build
(golden fixtures from tests/golden/make_golden.py) and cross-checked against
the independent C/OpenMP port (oracle/fmvd_cpu.c)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden, rel_l2
from gpu_deconvolution_b200 import synth
from oracle import fmvd_oracle as O

TOL = 1e-4


def test_snap_transform_size_table():
    # powers of two kept; next power of two up to 1024; multiples of 512 above
    cases = {1: 16, 16: 16, 17: 32, 272: 512, 512: 512, 541: 1024, 542: 1024, 1024: 1024, 1025: 1536,
             1054: 1536, 1536: 1536, 2048: 2048, 2110: 2560, 2560: 2560, 3000: 3072, 3500: 3584, 4096: 4096}
    for n, want in cases.items():
        assert O.snap_transform_size(n) == want, n


def test_config_fft_planes():
    assert O.snap_transform_size(256 + 17 - 1) == 512
    assert O.snap_transform_size(512 + 31 - 1) == 1024
    assert O.snap_transform_size(2048 + 63 - 1) == 2560


def test_clamp_map_regions():
    m = O.clamp_map(16, 10, 3)
    assert list(m) == list(range(10)) + [9, 9, 9] + [0, 0, 0]


def test_pad_kernel_centre_and_wrap():
    k = np.arange(9, dtype=np.float64).reshape(3, 3)
    p = O.pad_kernel(k, 8, 8)
    assert p[0, 0] == k[1, 1]
    assert p[7, 7] == k[0, 0]
    assert p[1, 1] == k[2, 2]
    assert p.sum() == k.sum()


def test_circular_convolution_matches_direct():
    rng = np.random.default_rng(0)
    img = rng.normal(size=(16, 16))
    k = rng.normal(size=(3, 5))
    spec = np.fft.rfft2(O.pad_kernel(k, 16, 16))
    got = O.circ_conv(img, spec)
    ref = np.zeros_like(img)
    for y in range(16):
        for x in range(16):
            for ky in range(3):
                for kx in range(5):
                    ref[y, x] += k[ky, kx] * img[(y - (ky - 1)) % 16, (x - (kx - 2)) % 16]
    assert np.allclose(got, ref)


# ---------------------------------------------------------------- golden pins
RL_FIXTURES = ["rl16_v2", "rl16_psf1", "rl16_psf2", "rl16_psf3", "rl8_v3", "rl16_nonsquare", "rl16_extremes"]


@pytest.mark.parametrize("name", RL_FIXTURES)
def test_oracle_matches_reference_build(name):
    g = golden(name)
    views, weights, kernels = g["views"], g["weights"], g["kernels"]
    bits = 16 if views.dtype == np.uint16 else 8
    plan = O.Plan(views.shape[2], views.shape[3], list(weights), list(kernels), int(g["psf"]), bits)
    assert [plan.fftH, plan.fftW] == list(g["fft"])
    # the caller's kernels come back normalised
    for k, kn in zip(kernels, g["kernels_normalised"]):
        assert np.allclose(O.normalize(k), kn, rtol=1e-6, atol=1e-9)
    its = sorted(int(k[len("est_it"):]) for k in g.files if k.startswith("est_it"))
    for it in its:
        est_ref = g[f"est_it{it}"]
        out_ref = g[f"out_it{it}"]
        for z in range(views.shape[1]):
            est = plan.deconvolve_plane([views[v, z] for v in range(views.shape[0])], it)
            assert rel_l2(est, est_ref[z]) < TOL, (name, it, z)
            d = np.abs(plan.unpad(est).astype(np.int64) - out_ref[z].astype(np.int64))
            assert d.max() <= 1 and (d > 0).mean() < 1e-2, (name, it, z)


@pytest.mark.parametrize("name", ["stream_d1_s3", "stream_d4_s3"])
def test_streaming_call_pattern_matches_reference(name):
    g = golden(name)
    D = g["views"].shape[1]
    sources, sinks = O.streaming_call_counts(D, int(g["nstreams"]))
    assert int(g["source_calls"]) == sources
    assert int(g["sink_calls"]) == sinks
    out = O.deconvolve_volume(g["views"], list(g["weights"]), list(g["kernels"]), 0, 2)
    d = np.abs(out.astype(np.int64) - g["out"][:D].astype(np.int64))
    assert d.max() <= 1


def test_texture_filter_model_matches_hardware():
    """The texture unit's weight for fractional offset f, measured on the
    B200: the oracle's quantisation model must reproduce it."""
    g = golden("transform")
    coords = g["probe_coords"].astype(np.float32)
    vals = g["probe_vals"]
    i, a = O.texture_weight(coords[:, 0], "round")
    assert np.all(i == 1)
    # the unit returns k/256 plus at most 128 * 2^-24 (its internal rounding)
    assert np.abs(a - vals).max() < 1e-5


def test_transform_oracle_matches_texture_unit():
    g = golden("transform")
    src, mats = g["src"], g["mats"]
    td, th, tw = (int(x) for x in g["shape"])
    for i, m in enumerate(mats):
        for bits in (16, 8):
            s = src if bits == 16 else (src >> 8).astype(np.uint8)
            ref = g[f"out{bits}_m{i}"]
            got = O.transform_volume(s, m, td, th, tw, bits=bits)
            top = 1 << bits
            d = np.abs(got.astype(np.int64) - ref.astype(np.int64))
            d = np.minimum(d, top - d)
            sens = O.transform_weight_sensitivity(s, m, td, th, tw, bits=bits)
            assert np.all(d <= sens + 1), (i, bits)
            raw = O.transform_volume(s, m, td, th, tw, bits=bits, out_float=True) * (top - 1)
            assert np.all(np.abs(raw - g[f"raw{bits}_m{i}"] * (top - 1)) <= sens + 1e-3), (i, bits)
            if i == 0:
                # weights that are exact multiples of 1/256: identical up to rounding
                assert d.max() <= 1


def test_saturated_fetch_conversion():
    """A fetch of value 1.0 converts (sample)(65536.5) through a 32-bit
    integer: the reference build gives 0, and so does the oracle."""
    g = golden("transform")
    assert int(g["saturation_out"][0, 0, 0]) == 0
    full = np.full((2, 2, 2), 65535, np.uint16)
    ident = np.array([1, 0, 0, 0.5, 0, 1, 0, 0.5, 0, 0, 1, 0.5], np.float32)
    assert int(O.transform_volume(full, ident, 1, 1, 1)[0, 0, 0]) == 0


# ---------------------------------------------------------- C port cross-check
def _cpu_lib():
    path = os.path.join(ROOT, "oracle", "_build", "libfmvd_cpu.so")
    if not os.path.exists(path):
        r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "cpu"], capture_output=True)
        if r.returncode != 0:
            pytest.skip("C port did not build")
    lib = C.CDLL(path)
    lib.fmvdcpu_deconvolve.restype = C.c_int
    return lib


@pytest.mark.parametrize("bits,ksize,shape", [(16, 9, (4, 48, 40)), (8, 7, (3, 33, 37)), (16, 17, (2, 64, 64))])
def test_c_port_matches_oracle(bits, ksize, shape):
    lib = _cpu_lib()
    views, psfs, weights, _ = synth.plain_rl_views(shape=shape, n_views=2, n_beads=10, ksize=ksize, seed=2, bits=bits)
    V, D, H, W = views.shape
    it = 3
    out, est = O.deconvolve_volume(views, weights, psfs, 0, it, bits=bits, return_float=True)
    k1 = np.stack([O.normalize(p) for p in psfs]).astype(np.float32)
    k2 = np.stack(O.compute_kernel2(psfs, 0)).astype(np.float32)
    kH, kW = psfs[0].shape
    fh, fw = O.snap_transform_size(H + kH - 1), O.snap_transform_size(W + kW - 1)
    out_c = np.zeros((D, H, W), views.dtype)
    est_c = np.zeros((D, fh, fw), np.float32)
    P = lambda a: C.c_void_p(a.ctypes.data)
    r = lib.fmvdcpu_deconvolve(bits, P(np.ascontiguousarray(views)), P(np.ascontiguousarray(weights)), P(k1), P(k2),
                               V, D, H, W, kH, kW, it, P(out_c), P(est_c), 2)
    assert r == 0
    assert rel_l2(est_c, est) < TOL
    assert np.abs(out_c.astype(np.int64) - out.astype(np.int64)).max() <= 1
