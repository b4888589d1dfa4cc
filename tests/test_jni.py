"""The JNI layer the Fiji plugin binds (gpu_deconvolution_b200/csrc/jni).

No JDK exists here, so the layer is compiled against tests/jni/jni.h (the
subset of the JNI interface it uses, with the specification's names and
signatures) and driven by tests/jni/mock_jvm.cpp, which plays the Java side:
Java arrays, the static callbacks getNextPlane() / returnNextPlane(Object),
and exceptions thrown with ThrowNew."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

JNI_SRC = os.path.join(ROOT, "gpu_deconvolution_b200", "csrc", "jni", "fastspim_NativeSPIMReconstructionCuda.cpp")
MOCK = os.path.join(ROOT, "tests", "jni")
LIB_DIR = os.path.join(ROOT, "gpu_deconvolution_b200", "lib")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("jni") / "jni_driver")
    cmd = ["g++", "-std=c++17", "-O1", "-I" + MOCK, "-I" + os.path.join(ROOT, "include"),
           "-I/usr/local/cuda/include", JNI_SRC, os.path.join(MOCK, "mock_jvm.cpp"), "-o", exe,
           os.path.join(LIB_DIR, "libNativeSPIMReconstructionCuda.so"), "-Wl,-rpath," + LIB_DIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_jni_exports_and_error_paths(driver):
    out = subprocess.run([driver, "errors"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    lines = dict(l.split(" ", 1) for l in out.stdout.strip().splitlines())
    assert "[deconvolution already quit]" in lines["quit16_without_init"]
    assert "[deconvolution already quit]" in lines["quit8_without_init"]
    assert "[deconvolution not initialized]" in lines["interactive16_without_init"]
    assert "[Unsupported bit depth]" in lines["init_bad_bitdepth"]
    nm = subprocess.run(["nm", "--defined-only", driver], capture_output=True, text=True).stdout
    for name in ["getNumCudaDevices", "getCudaDeviceName", "setCudaDevice", "transform8", "transform16", "deconvolve",
                 "deconvolve_1init", "deconvolve_1interactive8", "deconvolve_1interactive16", "deconvolve_1quit8",
                 "deconvolve_1quit16"]:
        assert "Java_fastspim_NativeSPIMReconstructionCuda_" + name in nm


@pytest.mark.gpu
@pytest.mark.parametrize("bits", [16, 8])
def test_jni_streaming_and_files_match_c_api(driver, tmp_path, bits):
    from gpu_deconvolution_b200 import api, synth
    views, psfs, weights, _ = synth.plain_rl_views(shape=(5, 36, 40), n_views=2, n_beads=8, ksize=7, seed=21,
                                                  bits=bits)
    V, D, H, W = views.shape
    views.tofile(tmp_path / "views.raw")
    np.stack(weights).astype(np.float32).tofile(tmp_path / "weights.raw")
    np.stack(psfs).astype(np.float32).tofile(tmp_path / "kernels.raw")
    r = subprocess.run([driver, str(bits), str(W), str(H), str(D), str(V), "7", "7", "3", "0",
                        str(tmp_path / "views.raw"), str(tmp_path / "weights.raw"), str(tmp_path / "kernels.raw"),
                        str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    log = {l.split(" ", 1)[0]: l for l in lines}
    assert log["deconvolve_init"].endswith("exceptions=0")
    assert "[deconvolution already initialized]" in log["deconvolve_init_twice"]
    assert log["deconvolve_interactive"].endswith("exceptions=0")
    assert log["deconvolve_quit"].endswith("exceptions=0")
    assert log["deconvolve_files"].endswith("exceptions=0")
    ret = [l for l in lines if l.startswith("returned=")][0]
    assert ret.startswith(f"returned={D} ")
    dtype = np.uint16 if bits == 16 else np.uint8
    want = api.deconvolve(views, weights, [p.copy() for p in psfs], 0, 3, nstreams=3)
    got = np.fromfile(tmp_path / "interactive.raw", dtype).reshape(-1, H, W)
    assert np.array_equal(got, want[:D])
    got_f = np.fromfile(tmp_path / "files.raw", dtype).reshape(-1, H, W)
    assert np.array_equal(got_f[:D], want[:D])
