"""ctypes binding of the native library (libNativeSPIMReconstructionCuda.so).

This is the Python-side mirror of the reference's C API for the
reconstruction path: the same entry points, argument meaning and error
behaviour (errors are raised as ``FmvdError`` instead of terminating the
process, which is what the reference's default handler does).  There is no
fallback: if the library cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from .build import FEED_NAME, LIB_DIR, LIB_NAME

_lib = None
_lock = threading.Lock()
_errors: list[str] = []

c_p = C.c_void_p
c_int = C.c_int
c_float_p = C.POINTER(C.c_float)

SOURCE16 = C.CFUNCTYPE(c_int, C.POINTER(C.POINTER(C.c_uint16)), c_int)
SOURCE8 = C.CFUNCTYPE(c_int, C.POINTER(C.POINTER(C.c_uint8)), c_int)
SINK16 = C.CFUNCTYPE(None, C.POINTER(C.c_uint16))
SINK8 = C.CFUNCTYPE(None, C.POINTER(C.c_uint8))
HANDLER = C.CFUNCTYPE(None, c_p, C.c_char_p)


class FmvdError(RuntimeError):
    """An error reported by the native library through its error handler."""


@HANDLER
def _record_error(param, msg):
    _errors.append(msg.decode(errors="replace") if msg else "unknown error")


# the exported functions and their signatures (include/*.h)
SIGNATURES = {
    # fmvd_cuda_utils.h
    "setErrorHandler": (None, [HANDLER, c_p]),
    "iDivUp": (c_int, [c_int, c_int]),
    "__getLastCudaError": (None, [C.c_char_p, C.c_char_p, c_int]),
    "__gpuAssert": (None, [C.c_uint, C.c_char_p, c_int]),
    "getNumCUDADevices": (c_int, []),
    "getCudaDeviceName": (None, [c_int, C.c_char_p]),
    "setCudaDevice": (None, [c_int]),
    # fmvd_deconvolve.h
    "fmvd_malloc": (c_p, [C.c_size_t]),
    "fmvd_free": (None, [c_p]),
    "fmvd_initialize_cuda_16": (c_p, [c_int, c_int, c_p, c_p, c_int, c_int, c_int, c_int, c_int, SOURCE16, SINK16]),
    "fmvd_deconvolve_planes_cuda_16": (None, [c_p, c_int]),
    "fmvd_destroy_cuda_16": (None, [c_p]),
    "fmvd_deconvolve_files_cuda_16": (None, [c_p, c_p, c_int, c_int, c_int, c_p, c_p, c_int, c_int, c_int, c_int,
                                             c_int]),
    "fmvd_initialize_cuda_8": (c_p, [c_int, c_int, c_p, c_p, c_int, c_int, c_int, c_int, c_int, SOURCE8, SINK8]),
    "fmvd_deconvolve_planes_cuda_8": (None, [c_p, c_int]),
    "fmvd_destroy_cuda_8": (None, [c_p]),
    "fmvd_deconvolve_files_cuda_8": (None, [c_p, c_p, c_int, c_int, c_int, c_p, c_p, c_int, c_int, c_int, c_int,
                                            c_int]),
    # fmvd_transform.h
    "transform_cuda_16": (None, [c_p, c_int, c_int, c_int, c_int, c_int, c_int, c_float_p, C.c_char_p, c_int, c_int,
                                 C.c_float, C.c_char_p]),
    "transform_cuda_8": (None, [c_p, c_int, c_int, c_int, c_int, c_int, c_int, c_float_p, C.c_char_p, c_int, c_int,
                                C.c_float, C.c_char_p]),
    # fmvd_deconvolve_cuda.h
    "padKernel": (None, [c_p, c_p, c_int, c_int, c_int, c_int, c_p]),
    "padWeights": (None, [c_p, c_p, c_p, c_int, c_int, c_int, c_int, c_int, c_int, c_p]),
    "normalizeWeights": (None, [c_p, c_p, c_int, c_int, c_p]),
    "padDataClampToBorder32": (None, [c_p, c_p, c_int, c_int, c_int, c_int, c_int, c_int, c_p]),
    "unpadData32": (None, [c_p, c_p, c_int, c_int, c_int, c_int, c_p]),
    "modulateAndNormalize": (None, [c_p, c_p, c_int, c_int, c_int, c_p]),
    "multiply32": (None, [c_p, c_p, c_p, c_p, c_int, c_int, c_p]),
    "padDataClampToBorderAndInitialize_16": (None, [c_p, c_p, c_p, c_p, c_int, c_int, c_int, c_int, c_int, c_int,
                                                    c_p]),
    "unpadData_16": (None, [c_p, c_p, c_int, c_int, c_int, c_int, c_p]),
    "divide_16": (None, [c_p, c_p, c_p, c_int, c_int, c_p]),
    "padDataClampToBorderAndInitialize_8": (None, [c_p, c_p, c_p, c_p, c_int, c_int, c_int, c_int, c_int, c_int,
                                                   c_p]),
    "unpadData_8": (None, [c_p, c_p, c_int, c_int, c_int, c_int, c_p]),
    "divide_8": (None, [c_p, c_p, c_p, c_int, c_int, c_p]),
    # fmvd_b200.h
    "fmvd_b200_plan_create": (c_p, [c_int, c_int, c_int, c_p, c_p, c_int, c_int, c_int, c_int, c_int]),
    "fmvd_b200_plan_query": (c_int, [c_p, C.POINTER(c_int), C.POINTER(c_int), C.POINTER(c_int)]),
    "fmvd_b200_deconvolve_device": (c_int, [c_p, c_p, C.c_size_t, c_p, c_int, c_int, c_p, c_p]),
    "fmvd_b200_plan_destroy": (None, [c_p]),
    "fmvd_b200_plan_check": (c_int, [c_p]),
    "fmvd_b200_deconvolve_device_noalloc": (c_int, [c_p, c_p, C.c_size_t, c_p, c_int, c_int, c_p, c_p]),
    "fmvd_b200_conv_bf16": (c_int, [c_p, c_p, c_int, c_int, c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_p, c_p,
                                    c_int, c_p, c_p]),
    "fmvd_b200_conv_wgrad_bf16": (c_int, [c_p, c_p, c_int, c_int, c_int, c_int, c_int, c_int, c_p, c_p, c_p]),
    "fmvd_b200_unet_create": (c_p, [c_int, c_int, c_int, c_int, C.c_uint]),
    "fmvd_b200_unet_destroy": (None, [c_p]),
    "fmvd_b200_unet_param_count": (C.c_size_t, [c_p]),
    "fmvd_b200_unet_get_params": (c_int, [c_p, c_p]),
    "fmvd_b200_unet_set_params": (c_int, [c_p, c_p]),
    "fmvd_b200_unet_get_grads": (c_int, [c_p, c_p]),
    "fmvd_b200_unet_forward": (c_int, [c_p, c_p, C.c_size_t, c_int, c_p, c_p]),
    "fmvd_b200_unet_train_step": (c_int, [c_p, c_p, C.c_size_t, c_int, c_p, C.c_float, c_p, c_p]),
    "fmvd_b200_unet_check": (c_int, [c_p]),
    "fmvd_b200_reconstructor_create": (c_p, [c_p, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int]),
    "fmvd_b200_reconstruct_host": (c_int, [c_p, c_p, c_p, c_int, c_p]),
    "fmvd_b200_reconstructor_destroy": (None, [c_p]),
    "fmvd_b200_batch_create": (c_p, [c_int, c_p, c_p, c_p, c_p, c_p, c_p, c_int]),
    "fmvd_b200_batch_run": (c_int, [c_p, c_p]),
    "fmvd_b200_batch_branches": (c_int, [c_p]),
    "fmvd_b200_batch_destroy": (None, [c_p]),
    "fmvd_b200_plan_create_tuned": (c_p, [c_int, c_int, c_int, c_p, c_p, c_int, c_int, c_int, c_int, c_int, c_int]),
    "fmvd_b200_plan_col_warps": (c_int, [c_p]),
    "fmvd_b200_plan_create_scheduled": (c_p, [c_int, c_int, c_int, c_p, c_p, c_int, c_int, c_int, c_int, c_int,
                                             c_int, c_int]),
    "fmvd_b200_plan_radix_step": (c_int, [c_p]),
    "fmvd_b200_deconvolve_device_from": (c_int, [c_p, c_p, C.c_size_t, c_p, c_int, c_int, c_p, c_p, c_p]),
    "fmvd_b200_pad_estimate": (c_int, [c_p, c_p, c_p, c_int, C.c_float, c_p]),
    "fmvd_b200_plane_stats": (c_int, [c_p, c_p, c_int, c_int, c_int, c_int, c_int, c_p, c_p]),
    "fmvd_b200_initialize_cuda_16": (c_p, [c_int, c_int, c_p, c_p, c_int, c_int, c_int, c_int, c_int, SOURCE16,
                                           SINK16, c_int]),
    "fmvd_b200_initialize_cuda_8": (c_p, [c_int, c_int, c_p, c_p, c_int, c_int, c_int, c_int, c_int, SOURCE8, SINK8,
                                          c_int]),
    "fmvd_b200_source_pitch": (C.c_size_t, [c_int, c_int]),
    "fmvd_b200_transform_device": (c_int, [c_int, c_p, C.c_size_t, c_int, c_int, c_int, c_int, c_int, c_int, c_int,
                                           c_float_p, c_p, c_p, c_p]),
    "fmvd_b200_mask_device": (c_int, [c_p, c_int, c_int, c_int, c_int, C.c_float, c_int, c_int, C.c_float, c_float_p,
                                      c_p]),
    "fmvd_b200_transform_host": (c_int, [c_int, c_p, c_int, c_int, c_int, c_int, c_int, c_int, c_float_p, c_p]),
    "fmvd_b200_launch_count": (C.c_ulonglong, []),
}


def library_path() -> str:
    return os.path.join(LIB_DIR, LIB_NAME)


def load(path: str | None = None):
    """Load the native library (once) and install the raising error handler."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or library_path()
        if not os.path.exists(p):
            raise FmvdError(f"native library not built: {p} (run gpu_deconvolution_b200/build.py)")
        lib = C.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        lib.setErrorHandler(_record_error, None)
        _lib = lib
        return lib


_feed = None


def load_host_feed():
    """The C caller of the streaming API over host memory
    (lib/libfmvd_host_feed.so, linked against the main library)."""
    global _feed
    load()
    with _lock:
        if _feed is None:
            p = os.path.join(LIB_DIR, FEED_NAME)
            if not os.path.exists(p):
                raise FmvdError(f"host feed library not built: {p} (run gpu_deconvolution_b200/build.py)")
            f = C.CDLL(p)
            f.fmvd_feed_deconvolve_16.restype = c_int
            f.fmvd_feed_deconvolve_16.argtypes = [c_p, c_int, c_int, c_int, c_int, c_p, c_p, c_int, c_int, c_int,
                                                  c_int, c_int, c_p, c_int, c_p]
            _feed = f
        return _feed


def check(context: str = "") -> None:
    """Raise the errors the library reported since the last check."""
    if _errors:
        msgs = list(_errors)
        _errors.clear()
        raise FmvdError((context + ": " if context else "") + "; ".join(msgs))


def clear_errors() -> None:
    _errors.clear()


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def pointer_array(arrays) -> C.Array:
    arr = (c_p * len(arrays))(*[a.ctypes.data for a in arrays])
    return arr
