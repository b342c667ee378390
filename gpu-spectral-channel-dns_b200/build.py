"""Build libdnsb200.so in-tree for sm_100a with nvcc.

``python build.py`` (or ``build()`` from Python) compiles every CUDA and C++
source under ``csrc/`` into ``libdnsb200.so`` next to this file.  The CUDA runtime
is linked statically, so the library needs only the driver at run time.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdnsb200.so")
DRIVER_SRC = os.path.join(HERE, "driver", "dns_run.cpp")
DRIVER = os.path.join(HERE, "dns_run")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "dns_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build_driver(force: bool = False) -> str:
    """The parameter.txt driver executable, linked against the library."""
    if not force and os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= max(
            os.path.getmtime(DRIVER_SRC), os.path.getmtime(LIB)):
        return DRIVER
    cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-o", DRIVER + ".tmp", DRIVER_SRC, "-L", HERE, "-ldnsb200",
           "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{r.stderr}")
    os.replace(DRIVER + ".tmp", DRIVER)
    return DRIVER


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        build_driver()
        return LIB
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    objs = []

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        cmd = [nvcc, *FLAGS, *ARCH, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    build_driver(force=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
