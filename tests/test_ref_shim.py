"""The drop-in boundary against the reference's own declarations.

gpu-spectral-channel-dns_b200/shim/ref_shim.cu defines the reference's
hot-path entry points (initFFT, transform_3d_one, transform, cuda_transpose,
cheby_s2p/p2s, getUVW, computeLambVector, rhsNonlinear, solveEq,
initAuxMatrix, nextStep, initFlow, output_velocity, write/read_recover_data,
launch_subthread, synchronizeGPUsolver) over the C ABI.  Compiled here
against the reference's include/ directory, every definition must match the
reference's declaration, and linked against libdnsb200.so with no undefined
symbol, every ABI call must resolve.  Skipped where the reference's headers
are absent (REF_INCLUDE overrides their location).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_INCLUDE = os.environ.get("REF_INCLUDE", "/root/reference/include")
SHIM = os.path.join(ROOT, "gpu-spectral-channel-dns_b200", "shim", "ref_shim.cu")
LIBDIR = os.path.join(ROOT, "gpu-spectral-channel-dns_b200")


def test_shim_compiles_against_reference_headers_and_links(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.isdir(REF_INCLUDE) or not os.path.exists(nvcc):
        pytest.skip("reference headers or nvcc not available")
    if not os.path.exists(os.path.join(LIBDIR, "libdnsb200.so")):
        pytest.skip("libdnsb200.so not built")
    obj = str(tmp_path / "ref_shim.o")
    r = subprocess.run([nvcc, "-std=c++17", "-Xcompiler", "-fPIC", "-diag-suppress", "2464",
                        "-gencode", "arch=compute_100a,code=sm_100a", "-c", SHIM,
                        "-I", REF_INCLUDE, "-I", os.path.join(ROOT, "include"), "-o", obj],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    cudalib = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "lib64")
    r = subprocess.run(["g++", "-shared", "-o", str(tmp_path / "libshim.so"), obj, "-L", LIBDIR,
                        "-ldnsb200", "-L", cudalib, "-lcudart", "-Wl,--no-undefined"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
