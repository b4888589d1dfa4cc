"""CPU tests of the C-ABI boundary: the library loads (no GPU needed to load
it) and exports every function the public headers declare, with C linkage
and, for the reference API, also with the reference's C++ linkage."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "gpu_deconvolution_b200", "lib", "libNativeSPIMReconstructionCuda.so")

# C++-mangled names of the reference build (nm -D of the upstream library
# compiled from its sources): the C++ linkage exports must match them.
REFERENCE_MANGLED = [
    "_Z15setErrorHandlerPFvPvPKcES_",
    "_Z6iDivUpii",
    "_Z18__getLastCudaErrorPKcS0_i",
    "_Z11__gpuAssertjPKci",
    "_Z17getNumCUDADevicesv",
    "_Z17getCudaDeviceNameiPc",
    "_Z13setCudaDevicei",
    "_Z11fmvd_mallocm",
    "_Z9fmvd_freePv",
    "_Z23fmvd_initialize_cuda_16iiPKPKfPPfii13fmvd_psf_typeiiPFiPPtiEPFvS6_E",
    "_Z22fmvd_initialize_cuda_8iiPKPKfPPfii13fmvd_psf_typeiiPFiPPhiEPFvS6_E",
    "_Z30fmvd_deconvolve_planes_cuda_16PK17fmvd_plan_cuda_16i",
    "_Z29fmvd_deconvolve_planes_cuda_8PK16fmvd_plan_cuda_8i",
    "_Z20fmvd_destroy_cuda_16P17fmvd_plan_cuda_16",
    "_Z19fmvd_destroy_cuda_8P16fmvd_plan_cuda_8",
    "_Z29fmvd_deconvolve_files_cuda_16PP8_IO_FILES0_iiiPPfS3_ii13fmvd_psf_typeii",
    "_Z28fmvd_deconvolve_files_cuda_8PP8_IO_FILES0_iiiPPfS3_ii13fmvd_psf_typeii",
    "_Z16transform_cuda_8PPhiiiiiiPfPKciifS3_",
    "_Z17transform_cuda_16PPtiiiiiiPfPKciifS3_",
]


def declared_functions():
    names = set()
    for f in os.listdir(INCLUDE):
        if not f.endswith(".h") or f.startswith("fastspim"):
            continue
        text = open(os.path.join(INCLUDE, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = re.sub(r"#[^\n]*", "", text)
        text = re.sub(r"typedef[^;]*;", "", text)
        for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof"):
                continue
            names.add(name)
    return names


@pytest.fixture(scope="module")
def exported():
    if not os.path.exists(LIB):
        pytest.fail("native library not built (gpu_deconvolution_b200/build.py)")
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_every_declared_function_is_exported(exported):
    names = declared_functions()
    assert len(names) > 40
    missing = sorted(n for n in names if n not in exported)
    assert not missing, missing


def test_reference_cxx_linkage_exported(exported):
    missing = [n for n in REFERENCE_MANGLED if n not in exported]
    assert not missing, missing


def test_library_loads_without_gpu():
    from gpu_deconvolution_b200 import native
    lib = native.load()
    assert lib.iDivUp(10, 3) == 4
    assert lib.iDivUp(9, 3) == 3
    assert lib.fmvd_b200_source_pitch(16, 28) == 32
    assert lib.fmvd_b200_source_pitch(8, 28) == 32


def test_error_handler_convention():
    """__gpuAssert with a failing code reports through the installed handler
    (the Python binding raises instead of exiting)."""
    from gpu_deconvolution_b200 import native
    lib = native.load()
    native.clear_errors()
    lib.__gpuAssert(2, b"file.cu", 7)
    with pytest.raises(native.FmvdError, match=r"Cuda error 2: .* in file.cu \(line 7\)"):
        native.check()
    lib.__gpuAssert(0, b"file.cu", 8)
    native.check()


def test_headers_compile_as_c_and_cpp(tmp_path):
    src = tmp_path / "t.c"
    src.write_text("#include <fmvd_deconvolve.h>\n#include <fmvd_transform.h>\n#include <fmvd_cuda_utils.h>\n"
                   "#include <fmvd_b200.h>\nint main(void){fmvd_psf_type t = efficient_bayesian; return (int)t - 1;}\n")
    for comp, name in (("gcc", "t.c"), ("g++", "t.cpp")):
        target = tmp_path / name
        if name != "t.c":
            target.write_text(src.read_text())
        r = subprocess.run([comp, "-fsyntax-only", "-I" + INCLUDE, str(target)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_reference_style_cxx_caller_links(tmp_path):
    """A C++ caller compiled against reference-style C++ declarations (no
    extern "C") links against the library."""
    src = tmp_path / "caller.cpp"
    src.write_text(
        "#include <stdio.h>\n"
        "enum fmvd_psf_type { independent, efficient_bayesian, optimization_1, optimization_2 };\n"
        "struct fmvd_plan_cuda_16;\n"
        "typedef int (*datasource_16_t)(unsigned short **buffer, int offset);\n"
        "typedef void (*datasink_16_t)(unsigned short *buffer);\n"
        "fmvd_plan_cuda_16 *fmvd_initialize_cuda_16(int, int, float const *const *, float **, int, int,"
        " fmvd_psf_type, int, int, datasource_16_t, datasink_16_t);\n"
        "void fmvd_destroy_cuda_16(fmvd_plan_cuda_16 *);\n"
        "int iDivUp(int a, int b);\n"
        "int main(){ return iDivUp(7, 2) == 4 ? 0 : 1; }\n"
        "void unused(){ fmvd_destroy_cuda_16(fmvd_initialize_cuda_16(1,1,0,0,1,1,independent,1,1,0,0)); }\n")
    exe = tmp_path / "caller"
    r = subprocess.run(["g++", str(src), "-o", str(exe), LIB, "-Wl,-rpath," + os.path.dirname(LIB)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_host_feed_library_loads_without_gpu():
    """The C caller of the streaming API (lib/libfmvd_host_feed.so) loads and
    resolves its calls into the main library."""
    from gpu_deconvolution_b200 import native
    feed = native.load_host_feed()
    assert feed.fmvd_feed_deconvolve_16 is not None
