"""Build the reference program from its own sources into oracle/_ref/ref_program.

Test infrastructure: the whole reference (Riveryh/gpu-spectral-channel-DNS)
as its CMake build would link it -- every file of its source/ directory,
compiled from where it lies, with its GPU half on cuFFT and its CPU half on
OpenMP -- except source/matrix_op.cpp, which needs Eigen (absent here) and
is replaced by oracle/ref_build/matrix_op_lu.cpp (the same two routines,
own code).  Nothing else is changed: the reference's own limits stay
(MAX_NZ = 100, so Ny <= 100; the plane Couette base flow), and its main reads
../input/parameter.txt.  The reference checkout is taken from REFERENCE_DIR,
else the location it has in the build container (/root/reference); where it
is absent this does nothing (a GPU host runs the built file).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(os.path.dirname(HERE), "_ref")
EXE = os.path.join(OUT_DIR, "ref_program")


def reference_dir():
    d = os.environ.get("REFERENCE_DIR", "/root/reference")
    return d if os.path.isfile(os.path.join(d, "source", "main_loop.cpp")) else None


def _nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def build():
    ref = reference_dir()
    if ref is None:
        return None
    nvcc = _nvcc()
    obj_dir = os.path.join(OUT_DIR, "ref_program_obj")
    os.makedirs(obj_dir, exist_ok=True)
    src = os.path.join(ref, "source")
    files = sorted(f for f in os.listdir(src) if f.endswith((".cu", ".cpp")) and f != "matrix_op.cpp")
    common = ["-std=c++14", "-O2", "-DNDEBUG", "-w", "-gencode", "arch=compute_100a,code=sm_100a",
              "-Xcompiler", "-fopenmp", "-I", os.path.join(ref, "include")]
    objs = []
    for f in files + [os.path.join(HERE, "matrix_op_lu.cpp")]:
        path = f if os.path.isabs(f) else os.path.join(src, f)
        obj = os.path.join(obj_dir, os.path.basename(path) + ".o")
        lang = ["-x", "cu", "-rdc=true"] if path.endswith(".cu") else ["-x", "c++"]
        r = subprocess.run([nvcc, *common, *lang, "-c", path, "-o", obj], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{path}:\n{r.stderr[-3000:]}")
        objs.append(obj)
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", "-o", EXE, *objs,
                        "-lcufft", "-lcublas", "-Xcompiler", "-fopenmp", "-lpthread"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-3000:])
    return EXE


if __name__ == "__main__":
    print(build())
