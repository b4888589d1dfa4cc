"""Python host API over the C ABI, mirroring the reference's operator
interface for the reconstruction path (fmvd_initialize / deconvolve_planes /
destroy with a datasource and datasink, the file entry point, transform_cuda)
plus device-resident variants for torch tensors.  Every call goes through the
native library; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import native
from .native import FmvdError

PSF_TYPES = {"independent": 0, "efficient_bayesian": 1, "optimization_1": 2, "optimization_2": 3}


def _sample_info(bits: int):
    if bits == 16:
        return np.uint16, C.c_uint16, native.SOURCE16, native.SINK16
    if bits == 8:
        return np.uint8, C.c_uint8, native.SOURCE8, native.SINK8
    raise ValueError("bits must be 8 or 16")


def _kernel_arrays(kernels, V):
    ks = [np.ascontiguousarray(np.asarray(k, np.float32)) for k in kernels]
    if len(ks) != V:
        raise ValueError("one kernel per view")
    return ks


class StreamingPlan:
    """fmvd_initialize_cuda_* / fmvd_deconvolve_planes_cuda_* / fmvd_destroy_cuda_*
    with Python callables as datasource and datasink.

    ``source(views: list[np.ndarray]) -> bool`` fills one plane per view
    (arrays of dataH x dataW, written in place) and returns False when no more
    planes exist; ``sink(plane: np.ndarray)`` receives each result plane.
    ``kernels`` are normalised in place, as the reference does.
    """

    def __init__(self, dataH, dataW, weights, kernels, psf_type=0, nstreams=3, source=None, sink=None, bits=16,
                 pairs_per_batch=0):
        self.lib = native.load()
        self.bits = bits
        self.dataH, self.dataW = dataH, dataW
        self.V = len(kernels)
        dtype, ctype, SRC, SNK = _sample_info(bits)
        self._dtype, self._ctype = dtype, ctype
        self.weights = [np.ascontiguousarray(np.asarray(w, np.float32)) for w in weights]
        self.kernels = _kernel_arrays(kernels, self.V)
        kH, kW = self.kernels[0].shape
        self._wp = native.pointer_array(self.weights)
        self._kp = native.pointer_array(self.kernels)
        self.source_calls = 0
        self.sink_calls = 0
        self._source = source
        self._sink = sink
        plane = dataH * dataW

        def c_source(buf, offset):
            self.source_calls += 1
            if self._source is None:
                return 0
            isz = np.dtype(dtype).itemsize
            views = [np.ctypeslib.as_array((ctype * plane).from_address(C.cast(buf[v], C.c_void_p).value + offset * isz))
                     .reshape(dataH, dataW) for v in range(self.V)]
            return 1 if self._source(views) else 0

        def c_sink(p):
            self.sink_calls += 1
            if self._sink is not None:
                self._sink(np.ctypeslib.as_array(p, shape=(dataH, dataW)).copy())

        self._c_source = SRC(c_source)
        self._c_sink = SNK(c_sink)
        native.clear_errors()
        fn = self.lib.fmvd_b200_initialize_cuda_16 if bits == 16 else self.lib.fmvd_b200_initialize_cuda_8
        self.plan = fn(dataH, dataW, self._wp, self._kp, kH, kW, int(psf_type), self.V, int(nstreams),
                       self._c_source, self._c_sink, int(pairs_per_batch))
        native.check("fmvd_initialize_cuda")
        if not self.plan:
            raise FmvdError("plan creation failed")
        fields = (C.c_int * 8).from_address(self.plan)
        self.fftH, self.fftW = fields[2], fields[3]
        self.nstreams = fields[7]

    def deconvolve_planes(self, iterations: int) -> None:
        fn = self.lib.fmvd_deconvolve_planes_cuda_16 if self.bits == 16 else self.lib.fmvd_deconvolve_planes_cuda_8
        fn(self.plan, int(iterations))
        native.check("fmvd_deconvolve_planes_cuda")

    def destroy(self) -> None:
        if self.plan:
            fn = self.lib.fmvd_destroy_cuda_16 if self.bits == 16 else self.lib.fmvd_destroy_cuda_8
            fn(self.plan)
            self.plan = None
            native.check("fmvd_destroy_cuda")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()


def deconvolve(views: np.ndarray, weights, kernels, psf_type=0, iterations=10, nstreams=3, pairs_per_batch=0,
               return_stats=False):
    """Deconvolve host views (V x D x H x W, uint16 or uint8) through the
    streaming C API; returns the planes the sink received (max(D, nstreams)
    planes, as the reference)."""
    views = np.asarray(views)
    bits = 16 if views.dtype == np.uint16 else 8
    V, D, H, W = views.shape
    state = {"z": 0}
    out = []

    def source(bufs):
        z = state["z"]
        if z >= D:
            return False
        for v in range(V):
            bufs[v][...] = views[v, z]
        state["z"] = z + 1
        return True

    plan = StreamingPlan(H, W, weights, [np.array(k, np.float32, copy=True) for k in kernels], psf_type, nstreams,
                         source, out.append, bits, pairs_per_batch)
    try:
        plan.deconvolve_planes(iterations)
    finally:
        plan.destroy()
    res = np.stack(out) if out else np.zeros((0, H, W), views.dtype)
    if return_stats:
        return res, {"source_calls": plan.source_calls, "sink_calls": plan.sink_calls, "fftH": plan.fftH,
                     "fftW": plan.fftW}
    return res


def deconvolve_c_callbacks(views: np.ndarray, weights, kernels, psf_type=0, iterations=10, nstreams=3,
                           return_stats=False):
    """``deconvolve`` with the datasource and datasink written in C
    (lib/libfmvd_host_feed.so): the drop-in streaming API as a C program
    drives it, without Python in the per-plane callbacks.  16-bit views
    (V x D x H x W); returns the planes the sink received."""
    views = np.ascontiguousarray(views, np.uint16)
    V, D, H, W = views.shape
    feed = native.load_host_feed()
    ks = np.ascontiguousarray(np.stack([np.asarray(k, np.float32) for k in kernels]))
    ws = np.ascontiguousarray(np.stack([np.asarray(w, np.float32) for w in weights]))
    kH, kW = ks.shape[1:]
    n_out = max(D, nstreams)
    out = np.zeros((n_out, H, W), np.uint16)
    counts = np.zeros(2, np.int32)
    native.clear_errors()
    got = feed.fmvd_feed_deconvolve_16(views.ctypes.data, V, D, H, W, ws.ctypes.data, ks.ctypes.data, kH, kW,
                                       int(psf_type), int(iterations), int(nstreams), out.ctypes.data, n_out,
                                       counts.ctypes.data)
    native.check("fmvd_feed_deconvolve_16")
    if got < 0:
        raise FmvdError("plan creation failed")
    res = out[:min(got, n_out)]
    if return_stats:
        return res, {"source_calls": int(counts[0]), "sink_calls": int(counts[1])}
    return res


def deconvolve_files(view_paths, out_path, dataW, dataH, dataD, weights, kernels, psf_type=0, iterations=10, bits=16):
    """fmvd_deconvolve_files_cuda_*: raw view files in, raw result file out."""
    lib = native.load()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    V = len(view_paths)
    files = [libc.fopen(p.encode(), b"rb") for p in view_paths]
    if not all(files):
        raise FmvdError("could not open a view file")
    res = libc.fopen(out_path.encode(), b"wb")
    ws = [np.ascontiguousarray(np.asarray(w, np.float32)) for w in weights]
    ks = _kernel_arrays(kernels, V)
    kH, kW = ks[0].shape
    fa = (C.c_void_p * V)(*files)
    fn = lib.fmvd_deconvolve_files_cuda_16 if bits == 16 else lib.fmvd_deconvolve_files_cuda_8
    native.clear_errors()
    fn(fa, res, dataW, dataH, dataD, native.pointer_array(ws), native.pointer_array(ks), kH, kW, int(psf_type), V,
       int(iterations))
    for f in files:
        libc.fclose(f)
    libc.fclose(res)
    native.check("fmvd_deconvolve_files_cuda")


class DevicePlan:
    """Device-resident deconvolution of torch CUDA tensors (fmvd_b200.h)."""

    def __init__(self, dataH, dataW, weights, kernels, psf_type=0, bits=16, pairs_per_batch=0, col_warps=0,
                 radix_step=0):
        """pairs_per_batch, col_warps and radix_step are the schedule knobs
        (0 = automatic; radix_step 1 or 2 selects the radix-R step of lines
        above 1024); ``autotune.tuned_plan`` picks them by measurement."""
        self.lib = native.load()
        self.bits = bits
        self.dataH, self.dataW = dataH, dataW
        self.V = len(kernels)
        self.weights = [np.ascontiguousarray(np.asarray(w, np.float32)) for w in weights]
        self.kernels = _kernel_arrays(kernels, self.V)
        kH, kW = self.kernels[0].shape
        native.clear_errors()
        self.plan = None
        if radix_step:
            self.plan = self.lib.fmvd_b200_plan_create_scheduled(bits, dataH, dataW,
                                                                 native.pointer_array(self.weights),
                                                                 native.pointer_array(self.kernels), kH, kW,
                                                                 int(psf_type), self.V, int(pairs_per_batch),
                                                                 int(col_warps), int(radix_step))
        elif col_warps:
            self.plan = self.lib.fmvd_b200_plan_create_tuned(bits, dataH, dataW, native.pointer_array(self.weights),
                                                             native.pointer_array(self.kernels), kH, kW,
                                                             int(psf_type), self.V, int(pairs_per_batch),
                                                             int(col_warps))
        else:
            self.plan = self.lib.fmvd_b200_plan_create(bits, dataH, dataW, native.pointer_array(self.weights),
                                                       native.pointer_array(self.kernels), kH, kW, int(psf_type),
                                                       self.V, int(pairs_per_batch))
        native.check("fmvd_b200_plan_create")
        if not self.plan:
            raise FmvdError("plan creation failed")
        h, w, p = C.c_int(), C.c_int(), C.c_int()
        self.lib.fmvd_b200_plan_query(self.plan, C.byref(h), C.byref(w), C.byref(p))
        self.fftH, self.fftW, self.pairs_per_batch = h.value, w.value, p.value
        self.col_warps = self.lib.fmvd_b200_plan_col_warps(self.plan)
        self.radix_step = self.lib.fmvd_b200_plan_radix_step(self.plan)

    def run(self, views, out, iterations, estimate=None, stream=0, view_stride=None, nplanes=None, init=None):
        """views: CUDA tensor holding V x D x dataH x dataW samples;
        out: CUDA tensor with room for D x dataH x dataW samples; estimate:
        optional float32 D x fftH x fftW that receives the final estimate;
        init: optional float32 D x fftH x fftW to start from instead of the
        reference's constant (continuing a run, or a warm start).
        ``nplanes`` defaults to out.shape[0].  Asynchronous on ``stream``
        (an int handle)."""
        D = nplanes if nplanes is not None else out.shape[0]
        vs = view_stride if view_stride is not None else D * self.dataH * self.dataW
        est = estimate.data_ptr() if estimate is not None else None
        native.clear_errors()
        if init is None:
            name = "fmvd_b200_deconvolve_device"
            r = self.lib.fmvd_b200_deconvolve_device(self.plan, views.data_ptr(), vs, out.data_ptr(), D,
                                                     int(iterations), est, stream)
        else:
            name = "fmvd_b200_deconvolve_device_from"
            r = self.lib.fmvd_b200_deconvolve_device_from(self.plan, views.data_ptr(), vs, out.data_ptr(), D,
                                                          int(iterations), init.data_ptr(), est, stream)
        native.check(name)
        if r != 0:
            raise FmvdError(name + " failed")

    def pad_estimate(self, planes, out, floor=float("-inf"), stream=0):
        """Data-plane float estimates (D x dataH x dataW CUDA tensor) onto the
        FFT plane (``out``: D x fftH x fftW) with the views' border padding,
        raised to ``floor``."""
        native.clear_errors()
        r = self.lib.fmvd_b200_pad_estimate(self.plan, planes.data_ptr(), out.data_ptr(), planes.shape[0],
                                            float(floor), stream)
        native.check("fmvd_b200_pad_estimate")
        if r != 0:
            raise FmvdError("fmvd_b200_pad_estimate failed")

    def run_until(self, views, out, tol, max_iterations, check_every=5, init=None, stream=0):
        """Plain RL in chunks of ``check_every`` iterations until the relative
        change of every plane's estimate over one chunk,
        ||e_k - e_(k-c)|| / ||e_k|| on the data region (FP64 sums on the
        GPU), is at most ``tol``, or ``max_iterations`` ran.  Chunks continue
        each other exactly.  Returns (iterations run, list of the largest
        per-plane change after each chunk)."""
        import torch
        D = out.shape[0]
        a = torch.empty((D, self.fftH, self.fftW), dtype=torch.float32, device=out.device)
        b = torch.empty_like(a)
        done, history = 0, []
        cur = init
        while done < max_iterations:
            k = min(check_every, max_iterations - done)
            self.run(views, out, k, estimate=a, stream=stream, init=cur)
            done += k
            if cur is not None:
                st = plane_stats(a, cur, self.dataH, self.dataW, stream=stream)
                change = float(np.max(np.sqrt(st[:, 2] / np.maximum(st[:, 1], 1e-300))))
                history.append(change)
                if change <= tol:
                    break
            a, b = b, a
            cur = b
        return done, history

    def destroy(self):
        if self.plan:
            self.lib.fmvd_b200_plan_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Reconstructor:
    """Host source volumes -> resampling -> plain RL -> host result, with the
    resampled frame kept on the device (fmvd_b200_reconstruct_host).
    ``plan`` is a DevicePlan for the frame's th x tw planes and V views."""

    def __init__(self, plan, views: int, src_shape, frame, chunk_planes: int = 0):
        self.lib = native.load()
        d, h, w = src_shape
        td, th, tw = frame
        self.plan, self.V, self.src_shape, self.frame = plan, views, tuple(src_shape), tuple(frame)
        native.clear_errors()
        self.rec = self.lib.fmvd_b200_reconstructor_create(plan.plan, views, w, h, d, tw, th, td, int(chunk_planes))
        native.check("fmvd_b200_reconstructor_create")
        if not self.rec:
            raise FmvdError("reconstructor creation failed")

    def run(self, views, inverses, iterations: int, out: np.ndarray | None = None) -> np.ndarray:
        """views: V host arrays d x h x w (uint16 or uint8, contiguous);
        inverses: V 3x4 target->source matrices."""
        vs = [np.ascontiguousarray(v) for v in views]
        assert len(vs) == self.V and all(v.shape == self.src_shape for v in vs)
        m = np.ascontiguousarray(np.stack([np.asarray(x, np.float32).reshape(12) for x in inverses]))
        if out is None:
            out = np.empty(self.frame, vs[0].dtype)
        ptrs = (C.c_void_p * self.V)(*[v.ctypes.data for v in vs])
        native.clear_errors()
        r = self.lib.fmvd_b200_reconstruct_host(self.rec, ptrs, m.ctypes.data, int(iterations), out.ctypes.data)
        native.check("fmvd_b200_reconstruct_host")
        if r != 0:
            raise FmvdError("fmvd_b200_reconstruct_host failed")
        return out

    def destroy(self):
        if self.rec:
            self.lib.fmvd_b200_reconstructor_destroy(self.rec)
            self.rec = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Batch:
    """Several device-resident volumes (each with its own ``DevicePlan``)
    deconvolved by one CUDA graph launch (fmvd_b200_batch_*).  The plans and
    tensors must outlive the batch."""

    def __init__(self, plans, views, outs, iterations, max_branches=1):
        self.lib = native.load()
        n = len(plans)
        its = iterations if isinstance(iterations, (list, tuple)) else [iterations] * n
        self._keep = (plans, views, outs)
        P = (C.c_void_p * n)(*[p.plan for p in plans])
        Vp = (C.c_void_p * n)(*[v.data_ptr() for v in views])
        S = (C.c_size_t * n)(*[o.shape[0] * p.dataH * p.dataW for p, o in zip(plans, outs)])
        O = (C.c_void_p * n)(*[o.data_ptr() for o in outs])
        D = (C.c_int * n)(*[o.shape[0] for o in outs])
        I = (C.c_int * n)(*[int(i) for i in its])
        native.clear_errors()
        self.batch = self.lib.fmvd_b200_batch_create(n, P, Vp, S, O, D, I, int(max_branches))
        native.check("fmvd_b200_batch_create")
        if not self.batch:
            raise FmvdError("batch creation failed")
        self.branches = self.lib.fmvd_b200_batch_branches(self.batch)

    def run(self, stream=0):
        native.clear_errors()
        r = self.lib.fmvd_b200_batch_run(self.batch, stream)
        native.check("fmvd_b200_batch_run")
        if r != 0:
            raise FmvdError("fmvd_b200_batch_run failed")

    def destroy(self):
        if self.batch:
            self.lib.fmvd_b200_batch_destroy(self.batch)
            self.batch = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def plane_stats(a, b=None, rows=None, cols=None, stream=0) -> np.ndarray:
    """FP64 per-plane sums of CUDA float32 planes ``a`` (D x H x W) over the
    top-left rows x cols region: columns sum a, sum a^2, sum (a-b)^2,
    sum |a-b| (zero without ``b``).  Returns a D x 4 float64 array."""
    import torch
    D, H, W = a.shape
    rows = H if rows is None else rows
    cols = W if cols is None else cols
    out = torch.empty((D, 4), dtype=torch.float64, device=a.device)
    lib = native.load()
    native.clear_errors()
    r = lib.fmvd_b200_plane_stats(a.data_ptr(), b.data_ptr() if b is not None else None, D, H, W, rows, cols,
                                  out.data_ptr(), stream)
    native.check("fmvd_b200_plane_stats")
    if r != 0:
        raise FmvdError("fmvd_b200_plane_stats failed")
    torch.cuda.synchronize(a.device)
    return out.cpu().numpy()


def transform_file(src: np.ndarray, inv, tw, th, td, outfile, mask=False, border=0, zspacing=1.0, maskfile=None):
    """transform_cuda_*: src is a d x h x w uint16/uint8 volume (one pointer per plane)."""
    lib = native.load()
    src = np.ascontiguousarray(src)
    bits = 16 if src.dtype == np.uint16 else 8
    d, h, w = src.shape
    planes = (C.c_void_p * d)(*[src[z].ctypes.data for z in range(d)])
    m = np.ascontiguousarray(np.asarray(inv, np.float32).reshape(12))
    fn = lib.transform_cuda_16 if bits == 16 else lib.transform_cuda_8
    native.clear_errors()
    fn(planes, w, h, d, tw, th, td, m.ctypes.data_as(native.c_float_p), outfile.encode(), int(bool(mask)),
       int(border), float(zspacing), (maskfile or "").encode())
    native.check("transform_cuda")


def transform_host(src: np.ndarray, inv, tw, th, td, out: np.ndarray | None = None) -> np.ndarray:
    """Resample into host memory (fmvd_b200_transform_host); ``out``
    (td x th x tw, the source's sample type, contiguous) is filled if given."""
    lib = native.load()
    src = np.ascontiguousarray(src)
    bits = 16 if src.dtype == np.uint16 else 8
    d, h, w = src.shape
    planes = (C.c_void_p * d)(*[src[z].ctypes.data for z in range(d)])
    m = np.ascontiguousarray(np.asarray(inv, np.float32).reshape(12))
    if out is None:
        out = np.zeros((td, th, tw), src.dtype)
    assert out.shape == (td, th, tw) and out.dtype == src.dtype and out.flags.c_contiguous
    native.clear_errors()
    r = lib.fmvd_b200_transform_host(bits, planes, w, h, d, tw, th, td, m.ctypes.data_as(native.c_float_p),
                                     out.ctypes.data)
    native.check("fmvd_b200_transform_host")
    if r != 0:
        raise FmvdError("transform failed")
    return out


def transform_device(src, pitch, w, h, d, inv, tw, th, z0, nz, out=None, out_f32=None, stream=0, bits=16):
    """Resample target planes [z0, z0+nz) of device source ``src`` (torch
    tensor, d x h x pitch samples) into device tensors."""
    lib = native.load()
    m = np.ascontiguousarray(np.asarray(inv, np.float32).reshape(12))
    native.clear_errors()
    r = lib.fmvd_b200_transform_device(bits, src.data_ptr(), pitch, w, h, d, tw, th, z0, nz,
                                       m.ctypes.data_as(native.c_float_p),
                                       out.data_ptr() if out is not None else None,
                                       out_f32.data_ptr() if out_f32 is not None else None, stream)
    native.check("fmvd_b200_transform_device")
    if r != 0:
        raise FmvdError("transform failed")


def mask_device(out, z, w, h, d, zspacing, tw, th, border, inv, stream=0):
    lib = native.load()
    m = np.ascontiguousarray(np.asarray(inv, np.float32).reshape(12))
    native.clear_errors()
    r = lib.fmvd_b200_mask_device(out.data_ptr(), z, w, h, d, float(zspacing), tw, th, float(border),
                                  m.ctypes.data_as(native.c_float_p), stream)
    native.check("fmvd_b200_mask_device")
    if r != 0:
        raise FmvdError("mask failed")


def source_pitch(bits: int, w: int) -> int:
    return native.load().fmvd_b200_source_pitch(bits, w)
