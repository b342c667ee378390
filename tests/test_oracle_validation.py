"""Physical validation of the oracle (the reference's algorithm): laminar
flow stays laminar, mean modes decay by the Crank-Nicolson factor, and the
Orr-Sommerfeld mode of plane Poiseuille flow grows at its eigenvalue's rate
(cases in validation_cases.py).  The device step matches the oracle to
1e-11 per step (test_gpu_parity.py); test_gpu_validation.py runs the same
cases on the device."""
import numpy as np
import pytest

from oracle import rpcf_oracle as O
import validation_cases as VC


@pytest.mark.parametrize("prof,Ro", [((0.5, 0.5, 0.0), 0.1), (VC.POISEUILLE, 0.0)])
def test_laminar_stays_laminar(prof, Ro):
    pb = O.Problem(O.Params(48, 48, 128, Re=1300.0, Ro=Ro, dt=0.005, prof=prof))
    sz = pb.sz
    Z = np.zeros((sz.ny, sz.hnx, sz.nz), dtype=np.complex128)
    pb.set_state(Z, Z.copy())
    pb.bootstrap()
    for _ in range(10):
        pb.step()
    assert np.max(np.abs(pb.V)) <= 1e-14 and np.max(np.abs(pb.O)) <= 1e-14


def test_mean_modes_decay_by_the_cn_factor():
    pb = O.Problem(O.Params(48, 48, 4 * VC.MEAN_N, Re=VC.MEAN_RE, Ro=0.1, dt=VC.MEAN_DT))
    V0, O0 = VC.mean_state(pb.sz)
    pb.set_state(V0, O0)
    pb.bootstrap()
    for _ in range(VC.MEAN_STEPS):
        pb.step()
    eu, ew = VC.mean_decay_errors(V0, O0, pb.V, pb.O)
    assert eu < 1e-12 and ew < 1e-12, (eu, ew)
    others = pb.V.reshape(-1, pb.sz.nz)[1:]
    assert np.max(np.abs(others)) <= 1e-14


def test_orr_sommerfeld_solver_matches_orszag():
    c, _ = VC.os_mode()
    assert abs(c.real - VC.ORSZAG_C.real) < 2e-8 and abs(c.imag - VC.ORSZAG_C.imag) < 2e-8, c


def test_orr_sommerfeld_growth_rate():
    c, a = VC.os_mode()
    mx, my, mz = VC.OS_GRID
    pb = O.Problem(O.Params(mx, my, mz, n_pi_x=2.0, n_pi_y=2.0, Re=VC.OS_RE, Ro=0.0, dt=VC.OS_DT,
                            prof=VC.POISEUILLE))
    V0, O0 = VC.os_state(pb.sz, a)
    pb.set_state(V0, O0)
    pb.bootstrap()
    for _ in range(VC.OS_STEPS):
        pb.step()
    lam = VC.os_rate(pb.V, a)
    # growth rate alpha c_i to 4 digits of the published eigenvalue
    assert abs(lam.real - VC.ORSZAG_C.imag) < 3.7e-7, lam
    # and the discrete Crank-Nicolson rate of the computed eigenvalue, closely
    assert abs(lam - VC.cn_rate(c)) < 1e-9, (lam, VC.cn_rate(c))
