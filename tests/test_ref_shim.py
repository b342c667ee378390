"""The drop-in boundary against the reference's own driver and declarations.

gpu-spectral-channel-dns_b200/shim/ref_shim.cu defines the reference's
hot-path entry points and the set-up calls of its driver over the C ABI.
gpu-spectral-channel-dns_b200/shim/build_ref_main.py compiles it against the
reference's include/ directory (every definition must match the reference's
declaration) and links it with the reference's unchanged main_loop.cpp,
operation.cpp, data.cpp and transform_multi_gpu.cpp and with libdnsb200.so into
two executables, with --no-undefined: every symbol the reference's driver
needs resolves, and none is defined twice.  Skipped where the reference's
sources are absent (REFERENCE_DIR names their location).
"""
import importlib.util
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-spectral-channel-dns_b200")


def _recipe():
    spec = importlib.util.spec_from_file_location("build_ref_main",
                                                  os.path.join(PKG, "shim", "build_ref_main.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_reference_driver_links_against_the_shim(tmp_path):
    m = _recipe()
    if m.reference_dir() is None:
        pytest.skip("the reference's sources are not present")
    if not os.path.exists(os.path.join(PKG, "libdnsb200.so")):
        pytest.skip("libdnsb200.so not built")
    exes = m.build(str(tmp_path))
    assert exes and all(os.access(e, os.X_OK) for e in exes)
    # the executables name the reference's and the library's entry points
    syms = subprocess.run(["nm", "-C", exes[0]], capture_output=True, text=True).stdout
    for name in ("run_simulation()", "RPCF_Paras::read_para", "nextStep(problem&)", "initFlow(problem&)",
                 "get_rhs_v(problem&)", "solveEq(", "allocHostMemory(problem&)", "allocDeviceMem(problem&)"):
        assert name in syms, name
    assert "U dns_step" in syms.replace("                 U", " U")
