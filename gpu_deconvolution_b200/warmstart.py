"""Learned warm start for plain Richardson-Lucy (no reference counterpart).

A small 2-D U-Net (fmvd_b200_unet_*: hand-written BF16 tcgen05 convolutions,
FP32 accumulation) maps the registered view planes of a z-plane and their
mean to an estimate of that plane.  It is trained only on pairs the method
itself produces: views and the plain RL-N result from the reference's
initialisation.  At inference the network's estimate, padded like the views,
starts RL (``DevicePlan.run(init=...)``) for k iterations instead of N;
plain RL-N remains the measure of its error and the fallback:

* ``WarmStartNet``      the network (train_step, forward, parameters)
* ``training_pairs``    views + plain RL-N targets on the GPU
* ``train``             Adam on the L1 loss over shuffled batches
* ``warm_deconvolve``   network -> padding -> RL-k, with the FP64
                        convergence check and the plain-RL fallback
* ``tune_k``            the smallest k whose result is within a relative L2
                        tolerance of plain RL-N on held-out planes
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import api, native, synth
from .native import FmvdError


class WarmStartNet:
    def __init__(self, H: int, W: int, views: int = 4, max_batch: int = 16, seed: int = 0):
        self.lib = native.load()
        native.clear_errors()
        self.net = self.lib.fmvd_b200_unet_create(H, W, views, max_batch, seed)
        native.check("fmvd_b200_unet_create")
        if not self.net:
            raise FmvdError("warm-start network creation failed")
        self.H, self.W, self.views, self.max_batch = H, W, views, max_batch
        self.nparams = int(self.lib.fmvd_b200_unet_param_count(self.net))

    def params(self) -> np.ndarray:
        p = np.empty(self.nparams, np.float32)
        if self.lib.fmvd_b200_unet_get_params(self.net, p.ctypes.data) != 0:
            raise FmvdError("fmvd_b200_unet_get_params failed")
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams
        native.clear_errors()
        r = self.lib.fmvd_b200_unet_set_params(self.net, p.ctypes.data)
        native.check("fmvd_b200_unet_set_params")
        if r != 0:
            raise FmvdError("fmvd_b200_unet_set_params failed")

    def grads(self) -> np.ndarray:
        g = np.empty(self.nparams, np.float32)
        if self.lib.fmvd_b200_unet_get_grads(self.net, g.ctypes.data) != 0:
            raise FmvdError("fmvd_b200_unet_get_grads failed")
        return g

    def train_step(self, views, target, lr: float, stream: int = 0) -> float:
        """views: CUDA int16 V x N x H x W (uint16 samples); target: CUDA
        float32 N x H x W.  lr = 0 computes the gradients only."""
        V, N, H, W = views.shape
        loss = C.c_float(0.0)
        native.clear_errors()
        r = self.lib.fmvd_b200_unet_train_step(self.net, views.data_ptr(), views.stride(0), N, target.data_ptr(),
                                               float(lr), C.byref(loss), stream)
        native.check("fmvd_b200_unet_train_step")
        if r != 0:
            raise FmvdError("fmvd_b200_unet_train_step failed")
        return float(loss.value)

    def forward(self, views, out=None, stream: int = 0):
        import torch
        V, N, H, W = views.shape
        if out is None:
            out = torch.empty((N, H, W), dtype=torch.float32, device=views.device)
        native.clear_errors()
        r = self.lib.fmvd_b200_unet_forward(self.net, views.data_ptr(), views.stride(0), N, out.data_ptr(), stream)
        native.check("fmvd_b200_unet_forward")
        if r != 0:
            raise FmvdError("fmvd_b200_unet_forward failed")
        return out

    def check(self) -> None:
        native.clear_errors()
        r = self.lib.fmvd_b200_unet_check(self.net)
        native.check("fmvd_b200_unet_check")
        if r != 0:
            raise FmvdError("warm-start network kernel reported a timeout")

    def save(self, path: str) -> None:
        np.savez(path, params=self.params(), H=self.H, W=self.W, views=self.views)

    def load(self, path: str) -> None:
        self.set_params(np.load(path)["params"])

    def destroy(self) -> None:
        if self.net:
            self.lib.fmvd_b200_unet_destroy(self.net)
            self.net = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def equal_weights(H, W, V):
    return [np.ones((H, W), np.float32)] * V


def rl_planes(plan: api.DevicePlan, views, iterations: int, init=None):
    """Plain RL of V x N x H x W views: (data-plane float estimates N x H x W,
    padded estimates N x fftH x fftW)."""
    import torch
    V, N, H, W = views.shape
    out = torch.empty((N, H, W), dtype=torch.int16, device=views.device)
    est = torch.empty((N, plan.fftH, plan.fftW), dtype=torch.float32, device=views.device)
    plan.run(views, out, iterations, estimate=est, init=init, view_stride=views.stride(0))
    return est[:, :H, :W], est


def training_pairs(n_planes: int, H: int = 512, W: int = 512, views: int = 4, iterations: int = 50,
                   seed: int = 1000, planes_per_volume: int = 64):
    """Views and plain RL-N targets (data region), all on the GPU, from the
    warm-start generator with fresh seeds.  Returns (views V x n x H x W,
    targets n x H x W, ground truth n x H x W, psfs)."""
    import torch
    vs, ts, gts = [], [], []
    psfs = None
    plan = None
    done = 0
    vol = 0
    while done < n_planes:
        D = min(planes_per_volume, n_planes - done)
        v, gt, psfs = synth.warm_start_views_torch(D, H, W, views, seed=seed + vol)
        if plan is None:
            plan = api.DevicePlan(H, W, equal_weights(H, W, views), [p.copy() for p in psfs], 0)
        est, _ = rl_planes(plan, v, iterations)
        vs.append(v)
        ts.append(est.clone())
        gts.append(gt)
        done += D
        vol += 1
    torch.cuda.synchronize()
    plan.destroy()
    return torch.cat(vs, dim=1).contiguous(), torch.cat(ts).contiguous(), torch.cat(gts).contiguous(), psfs


def train(net: WarmStartNet, views, targets, epochs: int = 10, batch: int = 16, lr: float = 1e-3, seed: int = 0,
          log=None, final_lr_fraction: float = 0.02):
    """Adam on the L1 loss over shuffled batches, the step size decaying on a
    cosine from ``lr`` to ``final_lr_fraction * lr``; returns the per-epoch
    mean losses."""
    import torch
    V, N, H, W = views.shape
    rng = np.random.default_rng(seed)
    history = []
    per_epoch = max(1, N // batch)
    total = max(1, epochs * per_epoch - 1)
    step = 0
    for ep in range(epochs):
        order = rng.permutation(N)
        losses = []
        for b0 in range(0, N - batch + 1, batch):
            idx = torch.from_numpy(order[b0:b0 + batch]).to(views.device)
            bv = views.index_select(1, idx).contiguous()
            bt = targets.index_select(0, idx).contiguous()
            f = final_lr_fraction + (1.0 - final_lr_fraction) * 0.5 * (1.0 + np.cos(np.pi * step / total))
            losses.append(net.train_step(bv, bt, lr * f))
            step += 1
        history.append(float(np.mean(losses)))
        if log:
            log(f"epoch {ep}: loss {history[-1]:.5f}")
    return history


def rel_l2_planes(a, b):
    """Per-plane relative L2 distance of CUDA tensors N x H x W (FP64 sums)."""
    st = api.plane_stats(a.contiguous(), b.contiguous())
    ref = api.plane_stats(b.contiguous())
    return np.sqrt(st[:, 2] / np.maximum(ref[:, 1], 1e-300))


def warm_deconvolve(net: WarmStartNet, plan: api.DevicePlan, views, k: int, check_tol: float | None = None,
                    fallback_iterations: int = 50, floor: float = 1.0):
    """Network estimate -> padding (values below ``floor`` samples raised to
    it: RL needs a positive start) -> k RL iterations.  With ``check_tol``,
    planes whose estimate still changes by more than check_tol (relative L2
    over one more iteration, FP64 sums) are redone with plain RL.  Returns
    (data-plane estimates N x H x W, indices of planes that fell back)."""
    import torch
    V, N, H, W = views.shape
    guess = net.forward(views)
    init = torch.empty((N, plan.fftH, plan.fftW), dtype=torch.float32, device=views.device)
    plan.pad_estimate(guess, init, floor)
    est, padded = rl_planes(plan, views, k, init=init)
    fell_back = np.zeros(0, np.int64)
    if check_tol is not None:
        nxt, _ = rl_planes(plan, views, 1, init=padded)
        change = rel_l2_planes(nxt.contiguous(), est.contiguous())
        fell_back = np.nonzero(change > check_tol)[0]
        if fell_back.size:
            idx = torch.from_numpy(fell_back).to(views.device)
            sub = views.index_select(1, idx).contiguous()
            plain, _ = rl_planes(plan, sub, fallback_iterations)
            est = est.contiguous()
            est[idx] = plain
    return est, fell_back


def tune_k(net: WarmStartNet, plan: api.DevicePlan, views, reference, tol: float = 1e-2,
           candidates=(0, 1, 2, 3, 4, 6, 8, 10, 12, 16, 20, 25, 30, 40)):
    """Smallest k whose warm-start result is within ``tol`` relative L2 of
    ``reference`` (plain RL-N) on every plane; None if none is."""
    errors = {}
    for k in candidates:
        est, _ = warm_deconvolve(net, plan, views, k)
        err = float(np.max(rel_l2_planes(est.contiguous(), reference)))
        errors[k] = err
        if err <= tol:
            return k, errors
    return None, errors


def time_cuda(fn, repeats: int = 3):
    """Median device time (ms) of fn() with CUDA events."""
    import torch
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def psnr(a, gt):
    """PSNR (dB) of estimate a against ground truth gt (peak = max of gt)."""
    a = a.double()
    gt = gt.double()
    mse = float(((a - gt) ** 2).mean())
    return 10.0 * np.log10(float(gt.max()) ** 2 / max(mse, 1e-300))


def wall(fn):
    t0 = time.perf_counter()
    r = fn()
    return r, time.perf_counter() - t0
