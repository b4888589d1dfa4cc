"""B200-native multi-view reconstruction (affine resampling + plane-wise
multi-view Richardson-Lucy), a drop-in for bene51/gpu_deconvolution's
native library.  The product is the shared library built from ``csrc/``;
this package holds its build recipe and a ctypes host API."""
from .native import FmvdError, library_path, load  # noqa: F401
