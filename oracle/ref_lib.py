"""ctypes access to the reference library built from the upstream sources
(TEST INFRASTRUCTURE: the checker and the reference arm, never the product).

``oracle/_ref/libfmvd_ref.so`` is the reference's deconvolution sources
(fmvd_deconvolve*.cpp, fmvd_deconvolve_cuda.cu, fmvd_cuda_utils.cpp) compiled
unmodified for sm_100a with cuFFT, plus ``oracle/ref_harness.cpp``, which feeds
the reference's public C API (fmvd_initialize / deconvolve_planes / destroy,
fmvd_deconvolve.impl.cpp:130-336) from host arrays through C datasource and
datasink callbacks.  ``oracle/_ref/libfmvd_reftex.so`` restates the reference
resampler (fmvd_transform.impl.cu:22-56) and mask kernel (fmvd_transform.cu:
19-67) with a texture object, because the upstream file binds legacy texture
references that CUDA 12 removed.

Only ``tests/``, ``tests/golden/make_golden.py`` and ``bench.py``'s reference
arm load these libraries; nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import fmvd_oracle as O

REF_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")
REF_LIB = os.path.join(REF_DIR, "libfmvd_ref.so")
TEX_LIB = os.path.join(REF_DIR, "libfmvd_reftex.so")


def available() -> bool:
    return os.path.exists(REF_LIB) and os.path.exists(TEX_LIB)


def load_ref():
    """(deconvolution library, texture resampler library)."""
    lib = C.CDLL(REF_LIB)
    lib.ref_deconvolve.restype = C.c_int
    lib.ref_deconvolve.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                   C.c_void_p]
    lib.ref_last_error.restype = C.c_char_p
    tex = C.CDLL(TEX_LIB)
    tex.reftex_transform.restype = C.c_int
    tex.reftex_transform.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    tex.reftex_probe.restype = C.c_int
    tex.reftex_probe.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    tex.reftex_mask.restype = C.c_int
    tex.reftex_mask.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                                C.c_float, C.c_void_p]
    return lib, tex


def ref_deconvolve(lib, views, weights, kernels, psf, iterations, nstreams, want_est, max_returned=None):
    """Deconvolve V x D x H x W host views through the reference library.

    Returns the sample planes the datasink received (``out``), the call counts,
    the FFT plane and, with ``want_est`` (nstreams must be 1), the float
    estimate of every returned plane on the FFT plane (``est``).  ``kernels``
    are copied; the normalised copies come back as ``kernels_normalised``."""
    views = np.ascontiguousarray(views)
    bits = 16 if views.dtype == np.uint16 else 8
    V, D, H, W = views.shape
    kH, kW = kernels[0].shape
    k = np.ascontiguousarray(np.stack(kernels).astype(np.float32))
    w = np.ascontiguousarray(np.stack(weights).astype(np.float32))
    mr = max_returned or max(D, nstreams)
    out = np.zeros((mr, H, W), views.dtype)
    stats = np.zeros(4, np.int32)
    est = None
    fh, fw = O.snap_transform_size(H + kH - 1), O.snap_transform_size(W + kW - 1)
    if want_est:
        est = np.zeros((mr, fh, fw), np.float32)
    r = lib.ref_deconvolve(bits, views.ctypes.data, V, D, H, W, w.ctypes.data, k.ctypes.data, kH, kW, psf,
                           iterations, nstreams, out.ctypes.data, mr, est.ctypes.data if est is not None else None,
                           stats.ctypes.data)
    if r != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    assert (int(stats[2]), int(stats[3])) == (fh, fw)
    res = {"out": out[:min(mr, int(stats[1]))], "source_calls": int(stats[0]), "sink_calls": int(stats[1]),
           "fftH": fh, "fftW": fw, "kernels_normalised": k}
    if est is not None:
        res["est"] = est[:min(mr, int(stats[1]))]
    return res


def ref_transform(tex, src, inv, tw, th, td, raw=None):
    """The reference resampler (texture-unit restatement) on a d x h x w host
    volume; returns td x th x tw samples."""
    src = np.ascontiguousarray(src)
    bits = 16 if src.dtype == np.uint16 else 8
    d, h, w = src.shape
    m = np.ascontiguousarray(np.asarray(inv, np.float32).reshape(12))
    out = np.zeros((td, th, tw), src.dtype)
    r = tex.reftex_transform(bits, src.ctypes.data, w, h, d, tw, th, td, m.ctypes.data, out.ctypes.data,
                             raw.ctypes.data if raw is not None else None, None)
    if r != 0:
        raise RuntimeError(f"reftex_transform failed ({r})")
    return out


def ref_mask(tex, inv, z, w, h, d, zspacing, tw, th, border):
    """The reference's transformed mask of target plane z (texture library's
    restatement of create_transformed_mask_kernel); th x tw float32."""
    m = np.ascontiguousarray(np.asarray(inv, np.float32).reshape(12))
    out = np.zeros((th, tw), np.float32)
    r = tex.reftex_mask(m.ctypes.data, z, w, h, d, float(zspacing), tw, th, float(border), out.ctypes.data)
    if r != 0:
        raise RuntimeError(f"reftex_mask failed ({r})")
    return out
