"""Write ref_cpu_N32.npz: outputs of the reference's own CPU operator and
right-hand-side code (source/coefficient.cu, source/linear.cpp, compiled
from the reference's sources into oracle/_ref/libref_cpu.so by
oracle/ref_build) on fixed inputs, so that the oracle stays pinned to the
reference where its sources are not available (tests/test_oracle_golden.py).

Run from the repository root after oracle/ref_build has built the library:
    python tests/golden/make_golden.py
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_cpu_N32.npz")

N, RE, DT = 32, 1300.0, 0.005
MODES = [(1.25, 0.5, 1.0), (20480.0, 64.0, -128.0)]  # (k^2, alpha, beta)


def dp(a):
    return a.ctypes.data_as(C.c_void_p)


def main():
    ref = C.CDLL(LIB)
    n1 = N + 1
    T0, T2, T4 = (np.zeros((n1, n1)) for _ in range(3))
    ref.ref_get_T_matrix(C.c_int(N), dp(T0), dp(T2), dp(T4))
    U, dU, ddU = (np.zeros(n1) for _ in range(3))
    ref.ref_get_U(C.c_int(n1), dp(U), dp(dU), dp(ddU))
    out = dict(N=N, Re=RE, dt=DT, modes=np.array(MODES), T0=T0, T2=T2, T4=T4, U=U, dU=dU, ddU=ddU)
    rng = np.random.default_rng(5)

    def crand():
        return rng.standard_normal(n1) + 1j * rng.standard_normal(n1)

    for i, (kmn, al, be) in enumerate(MODES):
        m = np.zeros((n1, n1), dtype=np.complex128)
        ref.ref_coef_v(dp(m), C.c_int(N), dp(U), dp(ddU), dp(T0), dp(T2), dp(T4), C.c_double(RE),
                       C.c_double(DT), C.c_double(kmn), C.c_double(al))
        out[f"coef_v_{i}"] = m
        m = np.zeros((n1, n1), dtype=np.complex128)
        ref.ref_coef_omega(dp(m), C.c_int(N), dp(U), dp(T0), dp(T2), dp(T4), C.c_double(RE),
                           C.c_double(DT), C.c_double(kmn), C.c_double(al))
        out[f"coef_omega_{i}"] = m
        v, vold, vnew, om, nv, nvp, no, nop = (crand() for _ in range(8))
        rv = v.copy()
        rvp = np.zeros(n1, dtype=complex)
        ref.ref_linear_v(dp(rv), dp(nv), dp(nvp), dp(rvp), C.c_int(N), dp(U), dp(ddU), dp(T0),
                         dp(T2), dp(T4), C.c_double(RE), C.c_double(DT), C.c_double(kmn),
                         C.c_double(al))
        ro = om.copy()
        ref.ref_linear_omega_y(dp(ro), dp(no), dp(nop), dp(vnew), dp(vold), C.c_int(N), dp(U),
                               dp(dU), dp(T0), dp(T2), C.c_double(RE), C.c_double(DT),
                               C.c_double(kmn), C.c_double(al), C.c_double(be))
        out.update({f"in_v_{i}": v, f"in_nv_{i}": nv, f"in_nvp_{i}": nvp, f"in_om_{i}": om,
                    f"in_no_{i}": no, f"in_nop_{i}": nop, f"in_vnew_{i}": vnew,
                    f"in_vold_{i}": vold, f"linear_v_{i}": rv, f"linear_omega_{i}": ro})
    m = np.zeros((n1, n1), dtype=np.complex128)
    ref.ref_coef_u0(dp(m), C.c_int(N), dp(T0), dp(T2), C.c_double(RE), C.c_double(DT))
    out["coef_u0"] = m
    u0, l0, l0p = crand(), crand(), crand()
    ru = u0.copy()
    ref.ref_linear_u0(dp(ru), dp(l0), dp(l0p), C.c_int(N), dp(T0), dp(T2), C.c_double(RE),
                      C.c_double(DT))
    out.update(in_u0=u0, in_l0=l0, in_l0p=l0p, linear_u0=ru)
    np.savez_compressed(OUT, **out)
    print(OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
