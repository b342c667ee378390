"""Host half of the banded wall-normal solve against the oracle (CPU).

The library's step solves the reference's collocation systems
(source/coefficient.cu:7-86) in an integrated, banded form whose operators
and factors are built on the host (csrc/wallsolve_host.cpp).  That host code
is compiled here with g++ (tests/native/wallsolve_check.cpp) and its solutions
are compared with np.linalg.solve on the oracle's dense collocation matrices,
which equal the reference's bit for bit (test_oracle_vs_reference.py).

Tolerance: the collocation v system is ill-conditioned (cond ~ 1e5 at
N = 32 to ~1e9 at N = 192); its dense solution carries relative errors of
that size times machine epsilon, and the explicit inverse the reference
multiplies by differs from a direct solve by as much.  The banded solution
must agree with the dense one to 2e-13 (omega, mean) and to 5e-11 at N <= 192
(v) in the relative 2-norm (measured at N = 192: 1.2e-11 and 1.1e-13).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import rpcf_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = [os.path.join(ROOT, "gpu-spectral-channel-dns_b200", "csrc", "wallsolve_host.cpp"),
       os.path.join(ROOT, "tests", "native", "wallsolve_check.cpp")]
EQ_V, EQ_OMEGA, EQ_MEAN = 0, 1, 2


@pytest.fixture(scope="module")
def ws(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("ws") / "libwscheck.so")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", *SRC, "-o", out],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail("g++ failed:\n" + r.stderr)
    return C.CDLL(out)


def dp(a):
    return a.ctypes.data_as(C.c_void_p)


def delta_of(U3):
    return 2 if U3[2] else (1 if U3[1] else 0)


def band(ws, eq, N, delta):
    out = np.zeros(5, dtype=np.int32)
    ws.ws_band(C.c_int(eq), C.c_int(N), C.c_int(delta), dp(out))
    return out


@pytest.mark.parametrize("N", [8, 32, 128])
@pytest.mark.parametrize("delta", [0, 1, 2])
def test_band_widths(ws, N, delta):
    """v: kl = delta + 4, ku = 2 delta + 8 (two dense columns); omega:
    kl = delta + 2, ku = 2 delta + 4; mean modes: kl 2, ku 4."""
    n, nb, nd, kl, ku = band(ws, EQ_V, N, delta)
    assert (n, nb, nd) == (N + delta + 1, N - 3, 2)
    assert kl == delta + 4 and ku <= 2 * delta + 8
    n, nb, nd, kl, ku = band(ws, EQ_OMEGA, N, delta)
    assert (n, nb, nd) == (N + delta + 1, N - 1, 0)
    assert kl == delta + 2 and ku <= 2 * delta + 4
    n, nb, nd, kl, ku = band(ws, EQ_MEAN, N, delta)
    assert (n, nb, nd, kl) == (N + 1, N - 1, 0, 2) and ku <= 4


def dense_system(eq, N, U3, Re, dt, kmn, al):
    T0, T2, T4 = O.get_T_matrix(N)
    U, dU, ddU = O.base_profile(np.cos(np.arange(N + 1) / N * O.PI), U3)
    if eq == EQ_V:
        return O.coef_v(N, U, ddU, T0, T2, T4, Re, dt, kmn, al), 4
    if eq == EQ_OMEGA:
        return O.coef_omega(N, U, T0, T2, Re, dt, kmn, al), 2
    return O.coef_u0(N, T0, T2, Re, dt), 2


def run_solve(ws, eq, shape_eq, N, U3, Re, dt, kmn, al, r):
    a = np.zeros(N + 1, dtype=np.complex128)
    rr = np.ascontiguousarray(r, dtype=np.complex128)
    st = ws.ws_solve(C.c_int(eq), C.c_int(shape_eq), C.c_int(N), C.c_int(delta_of(U3)),
                     C.c_double(Re), C.c_double(dt), C.c_double(kmn), C.c_double(al),
                     C.c_double(U3[0]), C.c_double(U3[1]), C.c_double(U3[2]), dp(rr), dp(a))
    assert st == 0
    return a


CASES = [(8, (0.5, 0.5, 0.0), 1300.0, 0.005), (32, (0.5, 0.5, 0.0), 1300.0, 0.005),
         (32, (1.0, 0.0, -1.0), 8400.0, 0.002), (64, (0.0, 0.0, 0.0), 2600.0, 0.005),
         (128, (0.5, 0.5, 0.0), 3000.0, 0.001), (128, (0.2, 0.3, 0.4), 3000.0, 0.001),
         (192, (0.5, 0.5, 0.0), 3000.0, 0.001)]  # Ny = 193: the 384x193x384 solve-only case
MODES = [(1.25, 0.5), (300.0, 10.0), (20000.0, 64.0), (0.25, 0.0), (16.0, 0.0)]


@pytest.mark.parametrize("N,U3,Re,dt", CASES)
def test_solutions_match_dense_collocation(ws, N, U3, Re, dt):
    rng = np.random.default_rng(N)
    for kmn, al in MODES:
        for eq, tol in ((EQ_V, 5e-11), (EQ_OMEGA, 2e-13)):
            A, nbc = dense_system(eq, N, U3, Re, dt, kmn, al)
            r = rng.standard_normal(N + 1) + 1j * rng.standard_normal(N + 1)
            r[:nbc] = 0
            ref = np.linalg.solve(A, r)
            got = run_solve(ws, eq, eq, N, U3, Re, dt, kmn, al, r)
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err < tol, (eq, kmn, al, err)


@pytest.mark.parametrize("N,U3,Re,dt", CASES)
def test_mean_modes_embedded(ws, N, U3, Re, dt):
    """The (0,0) mode's system (coef_u0) stored in the v and omega shapes,
    as the device packing stores it, gives the dense solution."""
    rng = np.random.default_rng(7)
    A, _ = dense_system(EQ_MEAN, N, U3, Re, dt, 0.0, 0.0)
    for shape_eq in (EQ_V, EQ_OMEGA, EQ_MEAN):
        r = rng.standard_normal(N + 1) + 1j * rng.standard_normal(N + 1)
        r[:2] = 0
        ref = np.linalg.solve(A, r)
        got = run_solve(ws, EQ_MEAN, shape_eq, N, U3, Re, dt, 0.0, 0.0, r)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-13


def bk_rows(ws, K, N, n, vals):
    g = np.zeros(n, dtype=np.complex128)
    v = np.ascontiguousarray(vals, dtype=np.complex128)
    ws.ws_integrate_values(C.c_int(K), C.c_int(N), C.c_int(n), dp(v), dp(g))
    return g


@pytest.mark.parametrize("N,U3", [(8, (0.5, 0.5, 0.0)), (32, (1.0, 0.0, -1.0)), (64, (0.2, 0.3, 0.4))])
def test_tilting_table(ws, N, U3):
    """Q w equals rows 2.. of B^2 applied to the interpolant of U'(y_m) w(y_m)
    at the interior points (zero at the walls) when w vanishes at the walls,
    as v^{n+1} does."""
    rng = np.random.default_rng(11)
    n = N + delta_of(U3) + 1
    b = rng.standard_normal(N - 1) + 1j * rng.standard_normal(N - 1)
    w = np.zeros(N + 1, dtype=np.complex128)
    w[:N - 1] -= b
    w[2:] += b  # Dirichlet basis: w(+-1) = 0
    y = np.cos(np.arange(N + 1) * np.pi / N)
    wv = np.polynomial.chebyshev.chebval(y, w)
    vals = (U3[1] + 2 * U3[2] * y) * wv
    vals[0] = vals[-1] = 0
    ref = bk_rows(ws, 2, N, n, vals)
    out = np.zeros(n, dtype=np.complex128)
    assert ws.ws_tilt(C.c_int(N), C.c_int(n), C.c_double(U3[1]), C.c_double(U3[2]), dp(w), dp(out)) == 0
    assert np.max(np.abs(out - ref)) <= 1e-13 * max(np.max(np.abs(ref)), 1e-300) + 1e-15


@pytest.mark.parametrize("N,n", [(8, 10), (32, 34), (128, 130), (192, 195)])
def test_integration_stencils(ws, N, n):
    """The banded stencils the y1 kernel applies equal the K-fold integration."""
    ws.ws_stencil_err.restype = C.c_double
    assert ws.ws_stencil_err(C.c_int(N), C.c_int(n)) < 1e-15
