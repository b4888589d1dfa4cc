"""Many volumes in one graph launch (fmvd_b200_batch_*) and the schedule
autotuner.  CPU tests cover the tuner's cache and choice; GPU tests check
that a batched graph run and a tuned plan give exactly the per-volume
results of the default path, and that a batched volume matches the oracle."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_deconvolution_b200 import autotune, synth


def test_best_prefers_fastest_then_smaller():
    table = {(2, 4): 1.0, (4, 8): 0.8, (6, 2): 0.8, (1, 2): 3.0}
    assert autotune.best(table) == (4, 8)
    assert autotune.best({(3, 8): 1.0, (3, 4): 1.0}) == (3, 4)
    # with the radix schedule as the third knob
    assert autotune.best({(1, 0, 2): 0.5, (1, 0, 1): 0.6, (2, 0, 1): 0.5}) == (1, 0, 2)


def test_pair_candidates_bounded_by_memory():
    assert autotune.pair_candidates(512, 512) == list(autotune.PAIRS)
    big = autotune.pair_candidates(4096, 4096)
    assert big and all(p * 2 * 8 * 4096 * 4096 <= autotune.MAX_WORK_BYTES for p in big) or big == [1]


def test_cache_roundtrip(tmp_path):
    path = str(tmp_path / "tune.json")
    key = autotune.cache_key("B200", 1024, 1024, 4, 16)
    assert autotune.load_cache(path) == {}
    autotune.save_entry(key, {"pairs_per_batch": 6, "col_warps": 8}, path)
    autotune.save_entry("other", {"pairs_per_batch": 1, "col_warps": 2}, path)
    data = autotune.load_cache(path)
    assert data[key]["pairs_per_batch"] == 6 and "other" in data
    (tmp_path / "bad.json").write_text("not json")
    assert autotune.load_cache(str(tmp_path / "bad.json")) == {}


def test_batched_specs_follow_the_workload():
    specs = synth.batched_specs(0, 32)
    assert len(specs) == 32
    for s in specs:
        assert s["H"] == s["W"] and s["H"] in synth.BATCH_PLANE_SIZES
        assert 16 <= s["D"] <= 256 and 2 <= s["V"] <= 6
        assert s["k"] % 2 == 1 and 9 <= s["k"] <= 41
        assert 200 <= s["peak"] <= 5000 and len(s["sigma"]) == s["V"]
    assert synth.batched_specs(0, 32) == specs  # seeded


def _small_specs():
    return synth.batched_specs(5, 4, sizes=(64, 96, 128), depth=(3, 7), views=(2, 3), ksize=(5, 11),
                               iterations=6)


@pytest.mark.gpu
def test_batch_graph_matches_individual_runs():
    import torch
    from gpu_deconvolution_b200 import api
    specs = _small_specs()
    plans, views, outs, refs = [], [], [], []
    for s in specs:
        psfs = synth.spec_psfs(s)
        w = [np.ones((s["H"], s["W"]), np.float32)] * s["V"]
        plans.append(api.DevicePlan(s["H"], s["W"], w, psfs, 0))
        views.append(synth.views_torch(s))
        outs.append(torch.zeros((s["D"], s["H"], s["W"]), dtype=torch.int16, device="cuda"))
    # a fifth volume that shares the first plan (same branch, run in order)
    views.append(views[0].flip(1).contiguous())
    outs.append(torch.zeros_like(outs[0]))
    all_plans = plans + [plans[0]]
    its = [s["iterations"] for s in specs] + [specs[0]["iterations"]]
    try:
        for p, v, o, it in zip(all_plans, views, outs, its):
            ref = torch.zeros_like(o)
            p.run(v, ref, it)
            refs.append(ref)
        torch.cuda.synchronize()
        batch = api.Batch(all_plans, views, outs, its, max_branches=3)
        try:
            assert batch.branches == 3
            for _ in range(2):  # graph replay gives the same result
                for o in outs:
                    o.zero_()
                batch.run()
                torch.cuda.synchronize()
                for o, r in zip(outs, refs):
                    assert torch.equal(o, r)
        finally:
            batch.destroy()
        for p in plans:
            assert p.lib.fmvd_b200_plan_check(p.plan) == 0
    finally:
        for p in plans:
            p.destroy()


@pytest.mark.gpu
def test_batched_volume_against_oracle():
    """Per-volume error of a batched volume against the FP64 oracle on two
    planes (RL parity tolerance 1e-4 relative L2 on the estimate)."""
    import torch
    from gpu_deconvolution_b200 import api
    from oracle import fmvd_oracle as O
    s = _small_specs()[1]
    psfs = synth.spec_psfs(s)
    w = [np.ones((s["H"], s["W"]), np.float32)] * s["V"]
    plan = api.DevicePlan(s["H"], s["W"], w, [p.copy() for p in psfs], 0)
    try:
        views = synth.views_torch(s)
        out = torch.zeros((s["D"], s["H"], s["W"]), dtype=torch.int16, device="cuda")
        est = torch.zeros((s["D"], plan.fftH, plan.fftW), dtype=torch.float32, device="cuda")
        plan.run(views, out, s["iterations"], estimate=est)
        torch.cuda.synchronize()
        vnp = views.cpu().numpy().view(np.uint16)
        oplan = O.Plan(s["H"], s["W"], w, psfs, 0)
        for z in (0, s["D"] - 1):
            e = oplan.deconvolve_plane([vnp[v, z] for v in range(s["V"])], s["iterations"])
            assert rel_l2(est[z].cpu().numpy(), e) < 1e-4
    finally:
        plan.destroy()


@pytest.mark.gpu
def test_tuned_plan_is_bit_identical(tmp_path):
    import torch
    from gpu_deconvolution_b200 import api
    H, W, V, D, k = 120, 100, 3, 9, 9
    entry = autotune.tune(H, W, k, k, views=V, planes=12, iterations=1, repeats=1,
                          path=str(tmp_path / "t.json"))
    assert entry["pairs_per_batch"] in autotune.PAIRS and entry["col_warps"] in (2, 4, 8)
    assert autotune.load_cache(str(tmp_path / "t.json"))  # cached
    psfs = [synth.gaussian_psf(k, k, 1.0, 2.0, 30.0 * v) for v in range(V)]
    w = [np.ones((H, W), np.float32)] * V
    g = torch.Generator(device="cuda").manual_seed(3)
    views = torch.randint(50, 3000, (V, D, H, W), dtype=torch.int32, device="cuda", generator=g).to(torch.int16)
    tuned = autotune.tuned_plan(H, W, w, [p.copy() for p in psfs], path=str(tmp_path / "t.json"))
    default = api.DevicePlan(H, W, w, [p.copy() for p in psfs], 0)
    try:
        a = torch.zeros((D, H, W), dtype=torch.int16, device="cuda")
        b = torch.zeros_like(a)
        ea = torch.zeros((D, tuned.fftH, tuned.fftW), dtype=torch.float32, device="cuda")
        eb = torch.zeros_like(ea)
        tuned.run(views, a, 5, estimate=ea)
        default.run(views, b, 5, estimate=eb)
        torch.cuda.synchronize()
        assert torch.equal(ea, eb) and torch.equal(a, b)
        # every column width gives the same bits
        for cw in (2, 4, 8):
            p = api.DevicePlan(H, W, w, [q.copy() for q in psfs], 0, pairs_per_batch=2, col_warps=cw)
            try:
                p.run(views, a, 5, estimate=ea)
                torch.cuda.synchronize()
                assert p.col_warps == cw and torch.equal(ea, eb)
            finally:
                p.destroy()
    finally:
        tuned.destroy()
        default.destroy()


def _oracle_middle_plane(args):
    H, W, weights, psfs, planes, iterations = args
    from oracle import fmvd_oracle as Or
    return Or.Plan(H, W, weights, psfs, 0).deconvolve_plane(planes, iterations)


@pytest.mark.gpu
def test_batched_workload_volumes_against_oracle():
    """Per-volume error of the batched workload (32 volumes, seed 0) against
    the FP64 oracle, on the middle plane of every volume (padded planes 256
    to 1536), within the RL parity tolerance of 1e-4 relative L2.  The
    oracle's planes run in spawned processes."""
    import multiprocessing as mp

    import torch
    from gpu_deconvolution_b200 import api
    jobs, ests, idx = [], [], []
    for sp in synth.batched_specs(0, 32):
        psfs = synth.spec_psfs(sp)
        w = [np.ones((sp["H"], sp["W"]), np.float32)] * sp["V"]
        views = synth.views_torch(sp)
        z = sp["D"] // 2
        one = views[:, z:z + 1].contiguous()
        plan = api.DevicePlan(sp["H"], sp["W"], w, [p.copy() for p in psfs], 0)
        try:
            est = torch.zeros((1, plan.fftH, plan.fftW), dtype=torch.float32, device="cuda")
            out = torch.zeros((1, sp["H"], sp["W"]), dtype=torch.int16, device="cuda")
            plan.run(one, out, sp["iterations"], estimate=est)
            torch.cuda.synchronize()
        finally:
            plan.destroy()
        vv = one[:, 0].cpu().numpy().view(np.uint16)
        jobs.append((sp["H"], sp["W"], w, psfs, [vv[v] for v in range(sp["V"])], sp["iterations"]))
        ests.append(est[0].cpu().numpy())
        idx.append(sp["index"])
        del views
    with mp.get_context("spawn").Pool(min(16, len(jobs))) as pool:
        refs = pool.map(_oracle_middle_plane, jobs)
    errors = {i: rel_l2(e, r) for i, e, r in zip(idx, ests, refs)}
    print("per-volume rel L2 vs the FP64 oracle:", {i: f"{v:.2e}" for i, v in errors.items()})
    assert len(errors) == 32
    assert max(errors.values()) < 1e-4, errors


@pytest.mark.gpu
@pytest.mark.parametrize("fh,fw", [(1536, 64), (64, 2560), (3072, 64)])
def test_radix_schedules_match_oracle(fh, fw):
    """Both radix schedules of lines above 1024 (R-point DFTs per position,
    and weighted sums over the sub-lines) against the FP64 oracle, in the row
    and the column role."""
    import torch
    from gpu_deconvolution_b200 import api
    from oracle import fmvd_oracle as O
    k = 7
    H, W = fh - k + 1, fw - k + 1
    rng = np.random.default_rng(fh + fw)
    views = rng.integers(20, 3000, (2, 3, H, W)).astype(np.uint16)
    psfs = [synth.gaussian_psf(k, k, 1.0, 2.0, 40.0 * v) for v in range(2)]
    w = [rng.uniform(0.3, 1.5, (H, W)).astype(np.float32) for _ in range(2)]
    _, oest = O.deconvolve_volume(views, w, psfs, 0, 3, return_float=True)
    tv = torch.from_numpy(views.view(np.int16)).cuda()
    for rs in (1, 2):
        plan = api.DevicePlan(H, W, w, [p.copy() for p in psfs], 0, radix_step=rs)
        try:
            assert plan.radix_step == rs
            out = torch.zeros((3, H, W), dtype=torch.int16, device="cuda")
            est = torch.zeros((3, plan.fftH, plan.fftW), dtype=torch.float32, device="cuda")
            plan.run(tv, out, 3, estimate=est)
            torch.cuda.synchronize()
            assert rel_l2(est.cpu().numpy(), oest) < 1e-4, rs
        finally:
            plan.destroy()


@pytest.mark.gpu
def test_tuner_picks_radix_schedule(tmp_path):
    entry = autotune.tune(1400, 1400, 31, 31, views=2, planes=4, iterations=1, repeats=1,
                          path=str(tmp_path / "t.json"))
    assert entry["radix_step"] in (1, 2) and entry["fft"] == [1536, 1536]
    assert any(key.endswith(",2") for key in entry["table"]) and any(key.endswith(",1") for key in entry["table"])
