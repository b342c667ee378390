"""The library's FFT engines run on the host (CPU, no GPU).

The butterfly and index arithmetic of the three FFTs the kernels use is
shared host/device code; tests/native/*_check.cpp run it pass by pass on the
CPU exactly as a block or warp does (all loads of a pass, then all stores):

* fft.cuh   runtime-length radix-4/2/3 FFT (the fallback for other lengths),
* fft2.cuh  compile-time-length Stockham FFT shared by a thread block,
* wfft.cuh  warp-synchronous Stockham FFT of one to three lines per warp.

Tolerances: FP64 2e-15, FP32 5e-7 of the largest output magnitude.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NATIVE = os.path.join(ROOT, "tests", "native")
CUDA_INC = "/usr/local/cuda/include"


def build(tmp_path_factory, name):
    out = str(tmp_path_factory.mktemp(name) / name)
    src = os.path.join(NATIVE, name + ".cpp")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-I", CUDA_INC, "-x", "c++", src, "-o", out],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(f"g++ {name} failed:\n{r.stderr}")
    return out


@pytest.fixture(scope="module")
def bins(tmp_path_factory):
    return {n: build(tmp_path_factory, n) for n in ("fft_check", "fft2_check", "wfft_check")}


def sample_vector(L):
    j = np.arange(L)
    return np.sin(0.37 * j * j + 1.0) + 1j * (np.cos(1.3 * j) - 0.25)


def run_line(exe, L, inv, prec):
    out = subprocess.run([exe, str(L), str(int(inv)), prec], capture_output=True, text=True,
                         check=True).stdout.split()
    v = np.array(out, dtype=float).reshape(-1, 2)
    return v[:, 0] + 1j * v[:, 1]


@pytest.mark.parametrize("L", [24, 36, 48, 64, 96, 128, 192, 256, 384, 512, 768])
@pytest.mark.parametrize("prec", ["d", "f"])
def test_runtime_fft(bins, L, prec):
    x = sample_vector(L)
    for inv in (False, True):
        got = run_line(bins["fft_check"], L, inv, prec)
        ref = np.fft.ifft(x) * L if inv else np.fft.fft(x)
        tol = 2e-15 if prec == "d" else 5e-7
        assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref)) * 4


@pytest.mark.parametrize("L", [48, 64, 96, 128, 144, 192, 256, 288, 384, 512, 576, 768])
@pytest.mark.parametrize("prec", ["d", "f"])
def test_block_fft(bins, L, prec):
    x = sample_vector(L)
    if prec == "f":
        x = x.astype(np.complex64).astype(np.complex128)
    for inv in (False, True):
        got = run_line(bins["fft2_check"], L, inv, prec)
        ref = np.fft.ifft(x) * L if inv else np.fft.fft(x)
        tol = 2e-15 if prec == "d" else 5e-7
        assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref)) * 4


def test_warp_fft(bins):
    out = subprocess.run([bins["wfft_check"]], capture_output=True, text=True, check=True).stdout
    rows = [ln.split() for ln in out.strip().splitlines()]
    assert len(rows) >= 20
    for prec, L, NL, ef, eb in rows:
        tol = 2e-15 if prec == "double2" else 5e-7
        assert float(ef) < tol and float(eb) < tol, (prec, L, NL, ef, eb)
