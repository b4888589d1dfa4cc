"""Resuming RL from a given estimate, warm-start padding and the FP64
per-plane convergence statistics (fmvd_b200_deconvolve_device_from,
fmvd_b200_pad_estimate, fmvd_b200_plane_stats) against the oracle and
against one uninterrupted run."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_deconvolution_b200 import api, synth
from oracle import fmvd_oracle as O

pytestmark = pytest.mark.gpu


def _case(torch, H=96, W=80, V=2, D=5, k=9, seed=4):
    rng = np.random.default_rng(seed)
    psfs = [synth.gaussian_psf(k, k, 1.0, 2.0, 50.0 * v) for v in range(V)]
    weights = [rng.uniform(0.5, 1.5, (H, W)).astype(np.float32) for _ in range(V)]
    views_np = rng.integers(100, 3000, (V, D, H, W)).astype(np.uint16)
    views = torch.from_numpy(views_np.view(np.int16)).cuda()
    return psfs, weights, views_np, views


def test_continuation_is_exact():
    torch = pytest.importorskip("torch")
    psfs, weights, _, views = _case(torch)
    V, D, H, W = views.shape
    plan = api.DevicePlan(H, W, weights, [p.copy() for p in psfs], 0, pairs_per_batch=2)
    try:
        fh, fw = plan.fftH, plan.fftW
        out_a = torch.zeros((D, H, W), dtype=torch.int16, device="cuda")
        est_a = torch.zeros((D, fh, fw), dtype=torch.float32, device="cuda")
        plan.run(views, out_a, 5, estimate=est_a)
        out_b = torch.zeros_like(out_a)
        est_b = torch.zeros_like(est_a)
        plan.run(views, out_b, 2, estimate=est_b)
        plan.run(views, out_b, 3, estimate=est_b, init=est_b)  # in place
        torch.cuda.synchronize()
        assert torch.equal(est_a, est_b)
        assert torch.equal(out_a, out_b)
    finally:
        plan.destroy()


def test_warm_start_from_oracle_estimate_matches_oracle():
    """Start from the oracle's 2-iteration estimate, run 2 more: the result is
    the oracle's 4-iteration estimate within the RL parity tolerance."""
    torch = pytest.importorskip("torch")
    psfs, weights, views_np, views = _case(torch, D=2)
    V, D, H, W = views.shape
    plan = api.DevicePlan(H, W, weights, [p.copy() for p in psfs], 0)
    oplan = O.Plan(H, W, weights, psfs, 0)
    try:
        fh, fw = plan.fftH, plan.fftW
        e2 = np.stack([oplan.deconvolve_plane([views_np[v, z] for v in range(V)], 2) for z in range(D)])
        e4 = np.stack([oplan.deconvolve_plane([views_np[v, z] for v in range(V)], 4) for z in range(D)])
        init = torch.from_numpy(e2.astype(np.float32)).cuda()
        est = torch.zeros((D, fh, fw), dtype=torch.float32, device="cuda")
        out = torch.zeros((D, H, W), dtype=torch.int16, device="cuda")
        plan.run(views, out, 2, estimate=est, init=init)
        torch.cuda.synchronize()
        assert rel_l2(est.cpu().numpy(), e4) < 1e-4
    finally:
        plan.destroy()


def test_pad_estimate_matches_oracle_padding():
    torch = pytest.importorskip("torch")
    H, W, kH, kW = 50, 37, 7, 11  # non-square kernel: the borders differ per axis
    psfs = [synth.gaussian_psf(kH, kW, 1.0, 1.5, 0.0)]
    plan = api.DevicePlan(H, W, [np.ones((H, W), np.float32)], psfs, 0)
    oplan = O.Plan(H, W, [np.ones((H, W), np.float32)], psfs, 0)
    try:
        rng = np.random.default_rng(1)
        planes = rng.uniform(0, 100, (3, H, W)).astype(np.float32)
        out = torch.zeros((3, plan.fftH, plan.fftW), dtype=torch.float32, device="cuda")
        plan.pad_estimate(torch.from_numpy(planes).cuda(), out)
        torch.cuda.synchronize()
        expect = np.stack([oplan.pad_data(p) for p in planes]).astype(np.float32)
        np.testing.assert_array_equal(out.cpu().numpy(), expect)
    finally:
        plan.destroy()


def test_plane_stats_fp64_against_oracle():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2)
    a = rng.uniform(0, 4000, (6, 130, 140)).astype(np.float32)
    b = (a + rng.normal(0, 1e-3, a.shape)).astype(np.float32)
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    for rows, cols, bb, tbb in ((130, 140, b, tb), (100, 77, b, tb), (130, 140, None, None)):
        got = api.plane_stats(ta, tbb, rows, cols)
        want = O.plane_stats(a, bb, rows, cols)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-9)
    # deterministic: the same bits on a second call
    np.testing.assert_array_equal(api.plane_stats(ta, tb), api.plane_stats(ta, tb))


def test_run_until_stops_on_tolerance_and_matches_fixed_count():
    torch = pytest.importorskip("torch")
    psfs, weights, _, views = _case(torch, D=4)
    V, D, H, W = views.shape
    plan = api.DevicePlan(H, W, weights, [p.copy() for p in psfs], 0)
    try:
        out = torch.zeros((D, H, W), dtype=torch.int16, device="cuda")
        n, hist = plan.run_until(views, out, tol=0.0, max_iterations=40, check_every=4)
        assert n == 40 and len(hist) == 9  # no check after the first chunk
        ref = torch.zeros_like(out)
        plan.run(views, ref, 40)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        # chunks continue each other exactly, so a rerun sees the same
        # changes and stops at the first check at or below the tolerance
        tol = hist[3]
        first = next(i for i, x in enumerate(hist) if x <= tol)
        n2, hist2 = plan.run_until(views, out, tol=tol, max_iterations=40, check_every=4)
        assert n2 == 4 * (first + 2) and hist2 == hist[:first + 1]
        plan.run(views, ref, n2)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    finally:
        plan.destroy()
