"""Pin the oracle to the reference's own CPU code through committed fixtures.

tests/golden/ref_cpu_N32.npz holds outputs of the reference's Chebyshev
tables, base flow, collocation operators (source/coefficient.cu) and CN
right-hand sides (source/linear.cpp) compiled from its sources
(tests/golden/make_golden.py).  Unlike test_oracle_vs_reference.py this
needs no reference sources: tables and operators must match bit for bit,
the right-hand sides (loops in the reference, matrix products here) to
1e-13 relative.  The v entry is _get_linear_v (the explicit CN operator), the
omega_y entry _get_linear_omega_y with its AB2 and tilting terms.
"""
import os

import numpy as np
import pytest

from oracle import rpcf_oracle as O

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cpu_N32.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(G)


def test_tables_and_base_flow(g):
    N = int(g["N"])
    T0, T2, T4 = O.get_T_matrix(N)
    assert np.array_equal(T0, g["T0"]) and np.array_equal(T2, g["T2"]) and np.array_equal(T4, g["T4"])
    U, dU, ddU = O.get_U(N + 1)
    assert np.array_equal(U, g["U"]) and np.array_equal(dU, g["dU"]) and np.array_equal(ddU, g["ddU"])


def test_collocation_operators(g):
    N, Re, dt = int(g["N"]), float(g["Re"]), float(g["dt"])
    T0, T2, T4, U, ddU = g["T0"], g["T2"], g["T4"], g["U"], g["ddU"]
    for i, (kmn, al, _) in enumerate(g["modes"]):
        assert np.array_equal(O.coef_v(N, U, ddU, T0, T2, T4, Re, dt, kmn, al), g[f"coef_v_{i}"])
        assert np.array_equal(O.coef_omega(N, U, T0, T2, Re, dt, kmn, al), g[f"coef_omega_{i}"])
    assert np.array_equal(O.coef_u0(N, T0, T2, Re, dt), g["coef_u0"])


def test_cn_right_hand_sides(g):
    N, Re, dt = int(g["N"]), float(g["Re"]), float(g["dt"])
    pb = O.Problem(O.Params(4 * N, 12, 4 * N, Re=Re, dt=dt))  # Ny = N + 1
    n1 = N + 1
    for i, (kmn, al, be) in enumerate(g["modes"]):
        pb.kmn = np.array([[kmn]])
        pb.ia = np.array([[al]])
        pb.ib = np.array([[be]])
        v = g[f"in_v_{i}"]
        rv = pb.linear_v(v[None, None])[0, 0]  # _get_linear_v: the CN operator part only
        ref = g[f"linear_v_{i}"]
        assert np.max(np.abs(rv - ref)) <= 1e-13 * np.max(np.abs(ref))
        ro = pb.linear_omega(g[f"in_om_{i}"][None, None], g[f"in_vnew_{i}"][None, None],
                             g[f"in_vold_{i}"][None, None])[0, 0]
        j = np.arange(2, n1)
        ro[2:] += (g[f"in_no_{i}"][j - 1] * 1.5 - g[f"in_nop_{i}"][j - 1] * 0.5) * dt
        ref = g[f"linear_omega_{i}"]
        assert np.max(np.abs(ro - ref)) <= 1e-13 * np.max(np.abs(ref))
    ru = pb.linear_u0(g["in_u0"], g["in_l0"], g["in_l0p"])
    assert np.max(np.abs(ru - g["linear_u0"])) <= 1e-13 * np.max(np.abs(g["linear_u0"]))
