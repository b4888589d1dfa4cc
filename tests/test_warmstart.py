"""The learned warm start: the network's forward pass and gradients against
the FP64 oracle, and what a briefly trained network gains over plain RL
started from the reference's constant initialisation.

The oracle (oracle/unet_oracle.py) is itself pinned by finite differences
of its exact FP64 mode on a small network."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import unet_oracle as U


def _random_params(V, base, seed=0, scale=0.2):
    shapes = U.layer_shapes(V, base)
    n = sum(co * t * ci + co for ci, co, t in shapes) + base + 1
    return np.random.default_rng(seed).normal(0, scale, n)


def test_oracle_gradient_finite_differences():
    V, base = 2, 8
    rng = np.random.default_rng(1)
    p = _random_params(V, base)
    views = rng.integers(100, 2000, (V, 1, 16, 16)).astype(np.uint16)
    tgt = rng.uniform(100, 2000, (1, 16, 16))
    _, g = U.network_grads(p, views, tgt, base, quantise=False)
    for i in rng.choice(p.size, 12, replace=False):
        e = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += e
        pm[i] -= e
        lp, _ = U.network_grads(pp, views, tgt, base, quantise=False)
        lm, _ = U.network_grads(pm, views, tgt, base, quantise=False)
        assert abs(g[i] - (lp - lm) / (2 * e)) <= 1e-6 + 1e-4 * abs(g[i])


def test_oracle_layer_list():
    shapes = U.layer_shapes(4)
    assert len(shapes) == 14 and shapes[0] == (64, 32, 1) and shapes[7] == (256, 256, 9)
    assert shapes[8] == (256, 128, 9) and shapes[13] == (32, 32, 9)


@pytest.mark.gpu
def test_network_forward_and_gradients_match_oracle():
    import torch
    from gpu_deconvolution_b200.warmstart import WarmStartNet
    V, N, H, W = 4, 2, 128, 128
    net = WarmStartNet(H, W, V, max_batch=N, seed=3)
    try:
        rng = np.random.default_rng(2)
        views_np = rng.integers(100, 2000, (V, N, H, W)).astype(np.uint16)
        target_np = rng.uniform(100, 2000, (N, H, W)).astype(np.float32)
        views = torch.from_numpy(views_np.view(np.int16)).cuda()
        target = torch.from_numpy(target_np).cuda()
        p = net.params()
        est = net.forward(views)
        torch.cuda.synchronize()
        ref, _ = U.network_forward(p, views_np)
        assert rel_l2(est.cpu().numpy(), ref) < 1e-2
        loss = net.train_step(views, target, 0.0)  # gradients only
        g = net.grads()
        assert np.array_equal(net.params(), p)
        ref_loss, ref_g = U.network_grads(p, views_np, target_np)
        assert abs(loss - ref_loss) < 1e-3 * ref_loss
        # per layer: bf16 storage between layers lets a few roundings differ
        off = 0
        for cin, cout, taps in U.layer_shapes(V):
            n = cout * taps * cin
            assert rel_l2(g[off:off + n], ref_g[off:off + n]) < 5e-2
            assert rel_l2(g[off + n:off + n + cout], ref_g[off + n:off + n + cout]) < 5e-2
            off += n + cout
        assert rel_l2(g[off:], ref_g[off:]) < 1e-2
        net.check()
    finally:
        net.destroy()


@pytest.mark.gpu
def test_trained_network_gains_over_plain_start():
    """Train briefly on 128 x 128 planes against plain RL-20; on held-out
    planes, 3 RL iterations from the network's estimate are closer to plain
    RL-20 than 3 iterations from the constant start."""
    import torch
    from gpu_deconvolution_b200 import api
    from gpu_deconvolution_b200 import warmstart as WS
    H = W = 128
    V, n_train, n_test, N_RL = 4, 192, 16, 20
    views, targets, _, psfs = WS.training_pairs(n_train + n_test, H, W, V, N_RL, seed=77, planes_per_volume=52)
    tr_v, te_v = views[:, :n_train].contiguous(), views[:, n_train:].contiguous()
    tr_t, te_t = targets[:n_train].contiguous(), targets[n_train:].contiguous()
    net = WS.WarmStartNet(H, W, V, max_batch=16, seed=0)
    plan = api.DevicePlan(H, W, WS.equal_weights(H, W, V), [p.copy() for p in psfs], 0)
    try:
        hist = WS.train(net, tr_v, tr_t, epochs=25, batch=16, lr=1e-3)
        assert hist[-1] < 0.6 * hist[0]
        warm, _ = WS.warm_deconvolve(net, plan, te_v, 3)
        plain, _ = WS.rl_planes(plan, te_v, 3)
        err_warm = float(np.mean(WS.rel_l2_planes(warm.contiguous(), te_t)))
        err_plain = float(np.mean(WS.rel_l2_planes(plain.contiguous(), te_t)))
        assert err_warm < err_plain, (err_warm, err_plain)
        # the convergence check with a tolerance nothing meets sends every
        # plane to the plain-RL fallback, which reproduces plain RL-20
        fb, idx = WS.warm_deconvolve(net, plan, te_v, 3, check_tol=0.0, fallback_iterations=N_RL)
        assert idx.size == n_test
        assert float(np.max(WS.rel_l2_planes(fb.contiguous(), te_t))) < 1e-6
        net.check()
    finally:
        plan.destroy()
        net.destroy()
