"""Schedule autotuner for the fused RL passes.

Three knobs decide how a padded plane geometry runs:

* ``pairs_per_batch``: plane pairs deconvolved together.  Larger batches give
  each launch more blocks; smaller ones keep the batch's work planes resident
  in L2 between the four passes of a view update.
* ``col_warps`` (tile schedule): warps (columns) per column-pass block, 2, 4
  or 8 (planes up to 1024 rows), which trades shared memory per block against
  blocks per SM.
* ``radix_step`` (radix schedule, lines longer than 1024 = R x 512): the
  radix-R step of the line transforms as R-point DFTs per position in shared
  memory (1) or as each sub-line group's weighted sum over the R sub-lines
  (2): the same transform with different instruction and shared-memory mixes.

The first two never change any plane's arithmetic (results are bit-identical
across settings); the radix schedule changes only the rounding of the FFT
(both stay within the parity tolerance of the FP64 oracle).

``tune`` times every candidate on synthetic planes of the geometry with CUDA
events and keeps the fastest in a JSON cache keyed by device, padded plane,
view count and sample size; ``tuned_plan`` builds a plan with the cached (or
freshly measured) choice.
"""
from __future__ import annotations

import json
import os
import threading

import numpy as np

PAIRS = (1, 2, 3, 4, 6, 8, 12, 16)
COL_WARPS = (2, 4, 8)
RADIX_STEPS = (1, 2)
MAX_WORK_BYTES = 1 << 29  # work planes of one candidate plan (C + estimate)

_lock = threading.Lock()


def cache_path() -> str:
    return os.environ.get("FMVD_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "gpu_deconvolution_b200", "tune.json")


def cache_key(device: str, fftH: int, fftW: int, views: int, bits: int) -> str:
    return f"{device}|{fftH}x{fftW}|V{views}|u{bits}"


def load_cache(path: str | None = None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def save_entry(key: str, entry: dict, path: str | None = None) -> None:
    path = path or cache_path()
    with _lock:
        data = load_cache(path)
        data[key] = entry
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        tmp = path + f".tmp{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def pair_candidates(fftH: int, fftW: int) -> list[int]:
    per_pair = 2 * 8 * fftH * fftW
    return [p for p in PAIRS if p * per_pair <= MAX_WORK_BYTES] or [1]


def best(table: dict) -> tuple:
    """The fastest (pairs, col_warps, radix_step) of a {key: ms} table; ties
    go to the smaller batch, then the narrower block, then schedule 1."""
    return min(table, key=lambda k: (table[k],) + tuple(k))


def _time_candidate(plan, views, out, iterations, repeats):
    import torch
    plan.run(views, out, 1)  # warm-up: first launches configure shared memory
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(repeats):
        plan.run(views, out, iterations)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / repeats


def tune(dataH, dataW, kH, kW, views=4, bits=16, planes=48, iterations=2, repeats=2, use_cache=True,
         path=None) -> dict:
    """Measure (or read from the cache) the best schedule for a geometry.
    Returns {"pairs_per_batch", "col_warps", "radix_step", "ms", "fft",
    "table"}."""
    import torch

    from . import api, native, synth

    probe = api.DevicePlan(dataH, dataW, [np.ones((dataH, dataW), np.float32)] * views,
                           [synth.gaussian_psf(kH, kW, 1.0, 2.0, 0.0)] * views, 0, bits=bits)
    fftH, fftW = probe.fftH, probe.fftW
    probe.destroy()
    device = torch.cuda.get_device_name()
    key = cache_key(device, fftH, fftW, views, bits)
    if use_cache:
        hit = load_cache(path).get(key)
        if hit:
            return hit

    g = torch.Generator(device="cuda").manual_seed(7)
    hi = 3000 if bits == 16 else 200
    dt = torch.int16 if bits == 16 else torch.uint8
    vols = torch.randint(10, hi, (views, planes, dataH, dataW), dtype=torch.int32, device="cuda",
                         generator=g).to(dt)
    out = torch.empty((planes, dataH, dataW), dtype=dt, device="cuda")
    psfs = [synth.gaussian_psf(kH, kW, 1.2, 3.0, 40.0 * v) for v in range(views)]
    weights = [np.ones((dataH, dataW), np.float32)] * views
    cws = COL_WARPS if fftH <= 1024 else (0,)
    radix = RADIX_STEPS if max(fftH, fftW) > 1024 else (1,)
    table = {}
    for pairs in pair_candidates(fftH, fftW):
        for cw in cws:
            for rs in radix:
                try:
                    plan = api.DevicePlan(dataH, dataW, weights, [p.copy() for p in psfs], 0, bits=bits,
                                          pairs_per_batch=pairs, col_warps=cw, radix_step=rs)
                except native.FmvdError:
                    continue  # this column width does not fit the plane
                try:
                    table[(pairs, plan.col_warps, rs)] = _time_candidate(plan, vols, out, iterations, repeats)
                finally:
                    plan.destroy()
    pairs, cw, rs = best(table)
    entry = {"pairs_per_batch": pairs, "col_warps": cw, "radix_step": rs, "ms": table[(pairs, cw, rs)],
             "fft": [fftH, fftW], "planes": planes, "iterations": iterations,
             "table": {f"{p},{c},{r}": round(ms, 4) for (p, c, r), ms in sorted(table.items())}}
    if use_cache:
        save_entry(key, entry, path)
    return entry


def tuned_plan(dataH, dataW, weights, kernels, psf_type=0, bits=16, **tune_args):
    """A DevicePlan with the autotuned schedule for its geometry."""
    from . import api
    kH, kW = np.asarray(kernels[0]).shape
    t = tune(dataH, dataW, kH, kW, views=len(kernels), bits=bits, **tune_args)
    return api.DevicePlan(dataH, dataW, weights, kernels, psf_type, bits=bits,
                          pairs_per_batch=t["pairs_per_batch"], col_warps=t["col_warps"],
                          radix_step=t.get("radix_step", 0))
