"""Build recipe for the native library (sm_100a), in-tree.

Produces ``gpu_deconvolution_b200/lib/libNativeSPIMReconstructionCuda.so``
(the reference's library name, so the Fiji plugin and C/C++ callers load it
unchanged) and the ``fmvd_deconvolve`` command-line tool in
``gpu_deconvolution_b200/bin/``.  Objects go to ``gpu_deconvolution_b200/_build``
and are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB_DIR = os.path.join(PKG, "lib")
BIN_DIR = os.path.join(PKG, "bin")
LIB_NAME = "libNativeSPIMReconstructionCuda.so"
FEED_NAME = "libfmvd_host_feed.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "-I" + INCLUDE, "-I" + CSRC] + ARCH

LIB_SOURCES = [
    "fmvd_cuda_utils.cpp",
    "engine.cpp",
    "deconvolve.cpp",
    "c_api.cpp",
    "cxx_api.cpp",
    "compat_launchers.cu",
    "transform.cu",
    "rl_kernels.cu",
    "noalloc.cu",
    "stats.cu",
    "batch.cpp",
    "reconstruct.cpp",
    "unet_gemm.cu",
    "unet_capi.cpp",
    "unet_layers.cu",
    "unet_model.cpp",
]
JNI_SOURCE = "jni/fastspim_NativeSPIMReconstructionCuda.cpp"


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    out = []
    for d in (CSRC, INCLUDE, os.path.join(CSRC, "jni")):
        if os.path.isdir(d):
            out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, extra: list[str]) -> str:
    obj = os.path.join(BUILD, src.replace("/", "_") + ".o")
    path = os.path.join(CSRC, src)
    if _stale(obj, [path] + _headers()):
        cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", path, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def jni_include_dirs() -> list[str] | None:
    """Directories holding jni.h: $JAVA_HOME/include(+/linux), else none."""
    home = os.environ.get("JAVA_HOME")
    if home and os.path.exists(os.path.join(home, "include", "jni.h")):
        return [os.path.join(home, "include"), os.path.join(home, "include", "linux")]
    return None


def build(verbose: bool = False, jobs: int = 8) -> str:
    """Compile every source for sm_100a and link the shared library and CLI."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(BIN_DIR, exist_ok=True)
    sources = list(LIB_SOURCES)
    extra_by_src = {s: [] for s in sources}
    jni = jni_include_dirs()
    if jni and os.path.exists(os.path.join(CSRC, JNI_SOURCE)):
        sources.append(JNI_SOURCE)
        extra_by_src[JNI_SOURCE] = ["-I" + d for d in jni]
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra_by_src[s]), sources))
    lib = os.path.join(LIB_DIR, LIB_NAME)
    if _stale(lib, objs):
        cmd = [nvcc(), "--shared"] + ARCH + objs + ["-o", lib, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    # a C caller of the streaming API over host memory (benchmark and tests)
    feed_src = os.path.join(CSRC, "host_feed.cpp")
    feed = os.path.join(LIB_DIR, FEED_NAME)
    if os.path.exists(feed_src) and _stale(feed, [feed_src, lib] + _headers()):
        cmd = [nvcc()] + NVCC_FLAGS + ["--shared", feed_src, "-o", feed, "-L" + LIB_DIR,
                                       "-lNativeSPIMReconstructionCuda", "-Xlinker", "-rpath=$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"host feed build failed:\n{r.stdout}\n{r.stderr}")
    cli_src = os.path.join(CSRC, "cli_main.cpp")
    cli = os.path.join(BIN_DIR, "fmvd_deconvolve")
    if os.path.exists(cli_src) and _stale(cli, [cli_src, lib]):
        cmd = [nvcc()] + NVCC_FLAGS + [cli_src, "-o", cli, "-L" + LIB_DIR, "-lNativeSPIMReconstructionCuda",
                                       "-Xlinker", "-rpath=$ORIGIN/../lib"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", lib)
    return lib


if __name__ == "__main__":
    build(verbose=True, jobs=int(sys.argv[1]) if len(sys.argv) > 1 else 8)
