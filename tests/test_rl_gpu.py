"""Parity of the B200 deconvolution with the FP64 oracle through the C ABI:
small planes, every FFT length, all PSF types, 8 and 16 bit, non-square
kernels, the streaming, file and CLI entry points and the reference's
call-pattern quirks.  (The oracle itself is pinned to the reference's CUDA
build by the fixtures of tests/golden/; tests/test_parity_depth_gpu.py runs
the reference build beside the library at each configuration's depth.)

Tolerances: float estimates within 1e-4 relative L2 of the oracle after every
tested iteration count; sample outputs within one unit of the oracle
(truncation of values that differ in the last float bits), and identical in
almost every voxel.
"""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_deconvolution_b200 import api, synth
from oracle import fmvd_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-4


def device_estimates(views, weights, kernels, psf, iterations, pairs=0):
    import torch
    V, D, H, W = views.shape
    plan = api.DevicePlan(H, W, weights, [k.copy() for k in kernels], psf, bits=16 if views.dtype == np.uint16 else 8,
                          pairs_per_batch=pairs)
    tv = torch.from_numpy(np.ascontiguousarray(views).view(np.uint8).reshape(-1)).cuda()
    out = torch.zeros(D * H * W * views.dtype.itemsize, dtype=torch.uint8, device="cuda")
    est = torch.zeros((D, plan.fftH, plan.fftW), dtype=torch.float32, device="cuda")
    plan.run(tv, out, iterations, est, nplanes=D)
    torch.cuda.synchronize()
    res = out.cpu().numpy().view(views.dtype).reshape(D, H, W), est.cpu().numpy()
    plan.destroy()
    return res


def oracle_estimates(views, weights, kernels, psf, iterations):
    out, est = O.deconvolve_volume(views, list(weights), list(kernels), psf, iterations,
                                   bits=16 if views.dtype == np.uint16 else 8, return_float=True)
    return out, est


def check_outputs(out, ref_out):
    d = np.abs(out.astype(np.int64) - ref_out.astype(np.int64))
    assert d.max() <= 1, d.max()
    assert (d > 0).mean() < 1e-2


@pytest.mark.parametrize("iterations", [1, 2, 5])
def test_small_two_views_vs_oracle(iterations):
    views, psfs, weights, _ = synth.plain_rl_views(shape=(3, 40, 48), n_views=2, n_beads=12, ksize=9,
                                                  sigma=(1.2, 2.5), seed=3)
    out, est = device_estimates(views, weights, psfs, 0, iterations)
    oout, oest = oracle_estimates(views, weights, psfs, 0, iterations)
    assert rel_l2(est, oest) < TOL
    check_outputs(out, oout)


@pytest.mark.parametrize("psf", [1, 2, 3])
def test_psf_types_vs_oracle(psf):
    views, psfs, _, _ = synth.plain_rl_views(shape=(2, 36, 36), n_views=3, n_beads=10, ksize=7, sigma=(1.0, 2.0),
                                            seed=4)
    rng = np.random.default_rng(5)
    weights = [rng.uniform(0.1, 1.0, (36, 36)).astype(np.float32) for _ in range(3)]
    out, est = device_estimates(views, weights, psfs, psf, 3)
    oout, oest = oracle_estimates(views, weights, psfs, psf, 3)
    assert rel_l2(est, oest) < TOL
    check_outputs(out, oout)


def test_eight_bit_vs_oracle():
    views, psfs, weights, _ = synth.plain_rl_views(shape=(3, 33, 37), n_views=2, n_beads=8, ksize=7, seed=6, bits=8)
    out, est = device_estimates(views, weights, psfs, 0, 3)
    oout, oest = oracle_estimates(views, weights, psfs, 0, 3)
    assert rel_l2(est, oest) < TOL
    check_outputs(out, oout)


def test_nonsquare_kernel_borders():
    rng = np.random.default_rng(13)
    gt = synth.bead_volume((2, 30, 50), 10, rng)
    kns = [synth.gaussian_psf(5, 11, 2.0, 1.0, 0.0), synth.gaussian_psf(5, 11, 1.0, 1.5, 30.0)]
    views = np.stack([synth.quantise(synth.blur_planes(gt, k), rng) for k in kns])
    w = [np.ones((30, 50), np.float32)] * 2
    out, est = device_estimates(views, w, kns, 0, 2)
    oout, oest = oracle_estimates(views, w, kns, 0, 2)
    assert rel_l2(est, oest) < TOL
    check_outputs(out, oout)


# every supported FFT length, in the row role and in the column role
LENGTH_PAIRS = [(16, 4096), (32, 3584), (64, 3072), (128, 2560), (256, 2048), (512, 1536), (1024, 1024),
                (4096, 16), (3584, 32), (3072, 64), (2560, 128), (2048, 256), (1536, 512)]


@pytest.mark.parametrize("fh,fw", LENGTH_PAIRS)
def test_every_fft_length(fh, fw):
    k = 5
    H, W = fh - k + 1, fw - k + 1
    rng = np.random.default_rng(fh * 7 + fw)
    views = rng.integers(50, 3000, (1, 2, H, W)).astype(np.uint16)
    psf = [synth.gaussian_psf(k, k, 1.0, 1.6, 20.0)]
    w = [np.ones((H, W), np.float32)]
    out, est = device_estimates(views, w, psf, 0, 1)
    assert est.shape[1:] == (fh, fw)
    oout, oest = oracle_estimates(views, w, psf, 0, 1)
    assert rel_l2(est, oest) < TOL
    check_outputs(out, oout)


@pytest.mark.parametrize("fh,fw", [(1536, 64), (64, 2560)])
def test_line_engine_8bit_two_views(fh, fw):
    """8-bit samples, two views with uneven weights and an odd number of
    planes, on the line engine (rows or columns above 1024)."""
    k = 7
    H, W = fh - k + 1, fw - k + 1
    rng = np.random.default_rng(fh + 3 * fw)
    views = rng.integers(5, 250, (2, 3, H, W)).astype(np.uint8)
    psf = [synth.gaussian_psf(k, k, 1.0, 2.0, 30.0 * v) for v in range(2)]
    w = [rng.uniform(0.3, 1.7, (H, W)).astype(np.float32) for _ in range(2)]
    out, est = device_estimates(views, w, psf, 0, 2)
    assert est.shape[1:] == (fh, fw)
    oout, oest = oracle_estimates(views, w, psf, 0, 2)
    assert rel_l2(est, oest) < TOL
    check_outputs(out, oout)


def test_config_plane_512_vs_oracle():
    """The plain-RL workload's plane geometry (256^2 data, 17^2 kernels -> 512^2)."""
    views, psfs, weights, _ = synth.plain_rl_views(shape=(2, 256, 256), n_views=2, n_beads=40, ksize=17, seed=8)
    out, est = device_estimates(views, weights, psfs, 0, 3)
    oout, oest = oracle_estimates(views, weights, psfs, 0, 3)
    assert est.shape[1:] == (512, 512)
    assert rel_l2(est, oest) < TOL
    check_outputs(out, oout)


def test_batching_is_invisible():
    """Batch size changes only the schedule: results are bitwise identical."""
    views, psfs, weights, _ = synth.plain_rl_views(shape=(7, 40, 40), n_views=2, n_beads=10, ksize=9, seed=9)
    a, ea = device_estimates(views, weights, psfs, 0, 2, pairs=1)
    b, eb = device_estimates(views, weights, psfs, 0, 2, pairs=8)
    assert np.array_equal(a, b)
    assert np.array_equal(ea, eb)


def test_zero_iterations_returns_initial_estimate():
    views, psfs, weights, _ = synth.plain_rl_views(shape=(2, 20, 20), n_views=3, n_beads=4, ksize=5, seed=10)
    out, est = device_estimates(views, weights, psfs, 0, 0)
    assert np.all(out == 30)
    assert np.allclose(est, 30.0)


def test_streaming_api_matches_device_api():
    views, psfs, weights, _ = synth.plain_rl_views(shape=(5, 40, 44), n_views=2, n_beads=10, ksize=9, seed=12)
    dev, _ = device_estimates(views, weights, psfs, 0, 3)
    got, stats = api.deconvolve(views, weights, psfs, 0, 3, nstreams=3, pairs_per_batch=1, return_stats=True)
    assert np.array_equal(got, dev)
    assert stats["source_calls"] == 6 and stats["sink_calls"] == 5


def test_streaming_c_callbacks_match_device_api():
    """The streaming API driven by a C datasource and datasink
    (lib/libfmvd_host_feed.so) gives the device API's planes and the
    reference's call counts."""
    views, psfs, weights, _ = synth.plain_rl_views(shape=(13, 40, 44), n_views=3, n_beads=10, ksize=9, seed=16)
    dev, _ = device_estimates(views, weights, psfs, 0, 3)
    got, stats = api.deconvolve_c_callbacks(views, weights, [p.copy() for p in psfs], 0, 3, nstreams=3,
                                            return_stats=True)
    assert np.array_equal(got, dev)
    assert stats["source_calls"] == 14 and stats["sink_calls"] == 13


def test_streaming_plans_reuse_pinned_buffers():
    """Streaming plans hand their pinned batch buffers to a process-wide pool
    that later plans draw from without clearing them: a plan that follows
    plans over other data, including a source shorter than nstreams (whose
    missing planes the reference leaves as zeros), gives the same planes as
    the same plan run first."""
    a_views, psfs, weights, _ = synth.plain_rl_views(shape=(11, 40, 44), n_views=3, n_beads=10, ksize=9, seed=18)
    b_views, _, _, _ = synth.plain_rl_views(shape=(2, 40, 44), n_views=3, n_beads=10, ksize=9, seed=19)
    first_b = api.deconvolve_c_callbacks(b_views, weights, [p.copy() for p in psfs], 0, 3, nstreams=3)
    first_a = api.deconvolve_c_callbacks(a_views, weights, [p.copy() for p in psfs], 0, 3, nstreams=3)
    for _ in range(2):
        assert np.array_equal(api.deconvolve_c_callbacks(b_views, weights, [p.copy() for p in psfs], 0, 3,
                                                         nstreams=3), first_b)
        assert np.array_equal(api.deconvolve_c_callbacks(a_views, weights, [p.copy() for p in psfs], 0, 3,
                                                         nstreams=3), first_a)
    assert first_b.shape[0] == 3  # the quirk plane of a 2-plane source with nstreams 3


def test_streaming_strict_read_ahead(monkeypatch):
    """FMVD_STRICT_READ_AHEAD=1: the datasource never runs more than nstreams
    planes ahead of the datasink (the reference's read-ahead), and the planes
    are the same as with batched read-ahead."""
    views, psfs, weights, _ = synth.plain_rl_views(shape=(9, 40, 44), n_views=2, n_beads=10, ksize=9, seed=17)
    want = api.deconvolve(views, weights, [p.copy() for p in psfs], 0, 2, nstreams=3)
    monkeypatch.setenv("FMVD_STRICT_READ_AHEAD", "1")
    state = {"z": 0, "out": [], "ahead": 0}

    def source(bufs):
        if state["z"] >= views.shape[1]:
            return False
        for v in range(views.shape[0]):
            bufs[v][...] = views[v, state["z"]]
        state["z"] += 1
        state["ahead"] = max(state["ahead"], state["z"] - len(state["out"]))
        return True

    plan = api.StreamingPlan(40, 44, weights, [p.copy() for p in psfs], 0, 3, source, state["out"].append)
    try:
        plan.deconvolve_planes(2)
    finally:
        plan.destroy()
    assert np.array_equal(np.stack(state["out"]), want)
    assert state["ahead"] <= 3


def test_streaming_fewer_planes_than_streams():
    """Reference quirk: a source with 1 plane and nstreams = 3 gives 3 sink
    calls and 4 source calls; the first plane is the real result."""
    views, psfs, weights, _ = synth.plain_rl_views(shape=(1, 24, 24), n_views=2, n_beads=4, ksize=5, seed=13)
    got, stats = api.deconvolve(views, weights, psfs, 0, 2, nstreams=3, return_stats=True)
    assert stats["source_calls"] == 4 and stats["sink_calls"] == 3
    oout, _ = oracle_estimates(views, weights, psfs, 0, 2)
    check_outputs(got[:1], oout)


def test_kernels_normalised_in_place(lib):
    """The caller's kernels come back normalised (fmvd_deconvolve.impl.cpp:63-64)."""
    psf = synth.gaussian_psf(7, 7, 1.0, 2.0, 0.0) * 5.0
    ks = [psf.copy(), (psf * 3).copy()]
    plan = api.StreamingPlan(20, 20, [np.ones((20, 20), np.float32)] * 2, ks, 0, 3)
    for k in plan.kernels:
        assert abs(float(k.astype(np.float64).sum()) - 1.0) < 1e-5
    plan.destroy()


def test_files_entry_point(tmp_path):
    views, psfs, weights, _ = synth.plain_rl_views(shape=(4, 30, 34), n_views=2, n_beads=6, ksize=7, seed=14)
    paths = []
    for v in range(2):
        p = tmp_path / f"v{v}.raw"
        views[v].tofile(p)
        paths.append(str(p))
    outp = str(tmp_path / "out.raw")
    api.deconvolve_files(paths, outp, 34, 30, 4, weights, [k.copy() for k in psfs], 0, 2)
    got = np.fromfile(outp, np.uint16).reshape(-1, 30, 34)
    oout, _ = oracle_estimates(views, weights, psfs, 0, 2)
    assert got.shape[0] == 4
    check_outputs(got, oout)


def test_unsupported_size_reports_error():
    from gpu_deconvolution_b200.native import FmvdError
    with pytest.raises(FmvdError):
        api.DevicePlan(5000, 64, [np.ones((5000, 64), np.float32)], [np.ones((3, 3), np.float32)], 0)


def test_cli_matches_c_api(tmp_path):
    """The fmvd_deconvolve tool takes the reference CLI's flags
    (fmvd_deconvolve_hdd.cpp:22-180) and writes the same planes."""
    import os
    import subprocess
    from conftest import ROOT
    exe = os.path.join(ROOT, "gpu_deconvolution_b200", "bin", "fmvd_deconvolve")
    views, psfs, weights, _ = synth.plain_rl_views(shape=(4, 30, 34), n_views=2, n_beads=6, ksize=7, seed=15)
    args = [exe, "-v", "2", "-i", "2", "-t", "0", "-o", str(tmp_path / "out.raw"), "-d"]
    for v in range(2):
        views[v].tofile(tmp_path / f"v{v}.raw")
        args.append(str(tmp_path / f"v{v}.raw"))
    args.append("-w")
    for v in range(2):
        weights[v].tofile(tmp_path / f"w{v}.raw")
        args.append(str(tmp_path / f"w{v}.raw"))
    args.append("-k")
    for v in range(2):
        psfs[v].tofile(tmp_path / f"k{v}.raw")
        args.append(str(tmp_path / f"k{v}.raw"))
    args += ["-dw", "34", "-dh", "30", "-dd", "4", "-kw", "7", "-kh", "7"]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(tmp_path / "out.raw", np.uint16).reshape(-1, 30, 34)
    want = api.deconvolve(views, weights, [p.copy() for p in psfs], 0, 2, nstreams=3)
    assert np.array_equal(got, want)
