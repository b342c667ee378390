"""Build the reference's own driver over libdnsb200: two executables.

``ref_main``      the reference's unchanged source/main_loop.cpp
                  (run_simulation) with operation.cpp, data.cpp and
                  transform_multi_gpu.cpp, compiled from where they lie in the
                  reference checkout, linked with ref_shim.cu (fused nextStep)
                  and -ldnsb200, with --no-undefined: every symbol the
                  reference's driver needs resolves, none twice;
``ref_main_fbf``  the same with ref_shim.cu compiled with
                  -DDNS_SHIM_FUNCTION_BY_FUNCTION (the reference's nextStep
                  sequence through the per-function drop-ins).

The reference checkout is taken from REFERENCE_DIR, else the location it has
in the build container (/root/reference).  The executables land next to this
file; the GPU tests run them from there.  ``python build_ref_main.py`` or
``build()``; returns the two paths, or None where the reference's sources are
absent.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libdnsb200.so")
REF_SOURCES = ("main_loop.cpp", "operation.cpp", "data.cpp", "transform_multi_gpu.cpp")
OUTPUTS = {"ref_main": [], "ref_main_fbf": ["-DDNS_SHIM_FUNCTION_BY_FUNCTION"]}


def reference_dir():
    d = os.environ.get("REFERENCE_DIR", "/root/reference")
    return d if os.path.isfile(os.path.join(d, "source", "main_loop.cpp")) else None


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)}\n{r.stderr[-4000:]}")
    return r


def build(out_dir: str | None = None):
    ref = reference_dir()
    if ref is None:
        return None
    out_dir = out_dir or HERE
    nvcc = _nvcc()
    cuda = os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))
    cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
    obj_dir = os.path.join(out_dir, "_build_ref_main")
    os.makedirs(obj_dir, exist_ok=True)
    inc = ["-I", os.path.join(ref, "include"), "-I", os.path.join(cuda, "include")]
    ref_objs = []
    for src in REF_SOURCES:
        obj = os.path.join(obj_dir, src + ".o")
        _run([cxx, "-std=c++17", "-O2", "-w", *inc, "-c", os.path.join(ref, "source", src), "-o", obj])
        ref_objs.append(obj)
    paths = []
    for name, defs in OUTPUTS.items():
        shim_obj = os.path.join(obj_dir, name + "_shim.o")
        _run([nvcc, "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-diag-suppress", "2464,1650",
              "-gencode", "arch=compute_100a,code=sm_100a", *defs, "-c",
              os.path.join(HERE, "ref_shim.cu"), "-I", os.path.join(ref, "include"),
              "-I", os.path.join(ROOT, "include"), "-o", shim_obj])
        exe = os.path.join(out_dir, name)
        rpath = os.path.relpath(PKG, out_dir)
        _run([cxx, "-o", exe, *ref_objs, shim_obj, "-L", PKG, "-ldnsb200",
              "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,--no-undefined",
              f"-Wl,-rpath,$ORIGIN/{rpath}"])
        paths.append(exe)
    return paths


if __name__ == "__main__":
    if not os.path.exists(LIB):
        sys.exit("libdnsb200.so is not built")
    print(build())
