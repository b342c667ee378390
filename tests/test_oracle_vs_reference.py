"""Pin the oracle to the reference's own code.

oracle/ref_build builds the reference's CPU operator and right-hand-side
functions (source/coefficient.cu, source/linear.cpp) from its sources into
oracle/_ref/libref_cpu.so.  The oracle's Chebyshev tables, base flow and
collocation operators must equal the reference's bit for bit; its explicit
CN right-hand sides (matrix products in NumPy, loops in the reference) to
rounding.  Skipped when the library was not built (no reference sources).
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import rpcf_oracle as O

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libref_cpu.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libref_cpu.so not built")
    lib = C.CDLL(LIB)
    return lib


def dp(a):
    return a.ctypes.data_as(C.c_void_p)


def ref_tables(ref, N):
    n1 = N + 1
    T0, T2, T4 = (np.zeros((n1, n1)) for _ in range(3))
    ref.ref_get_T_matrix(C.c_int(N), dp(T0), dp(T2), dp(T4))
    U, dU, ddU = (np.zeros(n1) for _ in range(3))
    ref.ref_get_U(C.c_int(n1), dp(U), dp(dU), dp(ddU))
    return T0, T2, T4, U, dU, ddU


@pytest.mark.parametrize("N", [32, 64, 128, 192])
def test_tables_bit_exact(ref, N):
    T0, T2, T4, U, dU, ddU = ref_tables(ref, N)
    o0, o2, o4 = O.get_T_matrix(N)
    assert np.array_equal(T0, o0) and np.array_equal(T2, o2) and np.array_equal(T4, o4)
    u, du, ddu = O.get_U(N + 1)
    assert np.array_equal(U, u) and np.array_equal(dU, du) and np.array_equal(ddU, ddu)


@pytest.mark.parametrize("N,Re,dt", [(32, 1300.0, 0.005), (64, 8400.0, 0.002), (128, 3000.0, 0.001)])
def test_operators_bit_exact(ref, N, Re, dt):
    T0, T2, T4, U, dU, ddU = ref_tables(ref, N)
    n1 = N + 1
    for kmn, al in [(1.25, 0.5), (4096.0 + 16384.0, 64.0), (0.25, 0.0)]:
        m = np.zeros((n1, n1), dtype=np.complex128)
        ref.ref_coef_v(dp(m), C.c_int(N), dp(U), dp(ddU), dp(T0), dp(T2), dp(T4), C.c_double(Re),
                       C.c_double(dt), C.c_double(kmn), C.c_double(al))
        assert np.array_equal(m, O.coef_v(N, U, ddU, T0, T2, T4, Re, dt, kmn, al))
        m = np.zeros((n1, n1), dtype=np.complex128)
        ref.ref_coef_omega(dp(m), C.c_int(N), dp(U), dp(T0), dp(T2), dp(T4), C.c_double(Re),
                           C.c_double(dt), C.c_double(kmn), C.c_double(al))
        assert np.array_equal(m, O.coef_omega(N, U, T0, T2, Re, dt, kmn, al))
    m = np.zeros((n1, n1), dtype=np.complex128)
    ref.ref_coef_u0(dp(m), C.c_int(N), dp(T0), dp(T2), C.c_double(Re), C.c_double(dt))
    assert np.array_equal(m, O.coef_u0(N, T0, T2, Re, dt))


@pytest.mark.parametrize("N,Re,dt", [(32, 1300.0, 0.005), (128, 3000.0, 0.001)])
def test_linear_rhs_matches_reference(ref, N, Re, dt):
    """_get_linear_v / _get_linear_omega_y / _get_linear_u0 on random
    pencils against the oracle's Problem.linear_* (relative 1e-13)."""
    T0, T2, T4, U, dU, ddU = ref_tables(ref, N)
    n1 = N + 1
    rng = np.random.default_rng(5)

    def crand():
        return rng.standard_normal(n1) + 1j * rng.standard_normal(n1)

    p = O.Params(4 * N, 12, 4 * N, Re=Re, dt=dt)  # Ny = N + 1
    pb = O.Problem(p)
    for kmn, al, be in [(1.25, 0.5, 1.0), (300.0, 10.0, -14.0)]:
        v, vold, vnew, om, nv, nvp, no, nop = (crand() for _ in range(8))
        # reference: rhs_v holds v^n on entry, rhs on exit; rhs_v_p receives v^n
        rv = v.copy()
        rvp = np.zeros(n1, dtype=complex)
        ref.ref_linear_v(dp(rv), dp(nv), dp(nvp), dp(rvp), C.c_int(N), dp(U), dp(ddU), dp(T0),
                         dp(T2), dp(T4), C.c_double(Re), C.c_double(dt), C.c_double(kmn),
                         C.c_double(al))
        pb.kmn = np.array([[kmn]])
        pb.ia = np.array([[al]])
        pb.ib = np.array([[be]])
        ov = pb.linear_v(v[None, None])[0, 0]
        assert np.array_equal(rvp, v)
        assert np.max(np.abs(rv - ov)) <= 1e-13 * np.max(np.abs(rv))
        ro = om.copy()
        ref.ref_linear_omega_y(dp(ro), dp(no), dp(nop), dp(vnew), dp(vold), C.c_int(N), dp(U),
                               dp(dU), dp(T0), dp(T2), C.c_double(Re), C.c_double(dt),
                               C.c_double(kmn), C.c_double(al), C.c_double(be))
        oo = pb.linear_omega(om[None, None], vnew[None, None], vold[None, None])[0, 0]
        i = np.arange(2, n1)
        oo[2:] += (no[i - 1] * 1.5 - nop[i - 1] * 0.5) * dt
        assert np.max(np.abs(ro - oo)) <= 1e-13 * np.max(np.abs(ro))
    u0, l0, l0p = crand(), crand(), crand()
    ru = u0.copy()
    ref.ref_linear_u0(dp(ru), dp(l0), dp(l0p), C.c_int(N), dp(T0), dp(T2), C.c_double(Re),
                      C.c_double(dt))
    ou = pb.linear_u0(u0, l0, l0p)
    assert np.max(np.abs(ru - ou)) <= 1e-13 * np.max(np.abs(ru))
