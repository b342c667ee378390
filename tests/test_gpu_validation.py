"""Physical validation of the device step (cases in validation_cases.py):
laminar flow stays laminar, mean modes decay by the Crank-Nicolson factor,
and the Orr-Sommerfeld mode of plane Poiseuille flow (Re 10^4, alpha = 1)
grows at the published eigenvalue's rate to 4 digits, in both forms."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import rpcf_oracle as O  # noqa: E402
import validation_cases as VC  # noqa: E402


@pytest.fixture(autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _run(pkg, mx, my, mz, V0, O0, steps, **kw):
    ctx = pkg.Context(pkg.make_params(mx, my, mz, **kw))
    ctx.set_state(V0, O0)
    ctx.bootstrap()
    ctx.step(steps)
    ctx.synchronize()
    V, Om = ctx.get_state()
    ctx.close()
    return V, Om


@pytest.mark.parametrize("U,Ro", [((0.5, 0.5, 0.0), 0.1), (VC.POISEUILLE, 0.0)])
def test_laminar_stays_laminar(pkg, U, Ro):
    sz = O.Sizes(48, 48, 128)
    Z = np.zeros((sz.ny, sz.hnx, sz.nz), dtype=np.complex128)
    V, Om = _run(pkg, 48, 48, 128, Z, Z, 10, Re=1300.0, Ro=Ro, dt=0.005, U=U)
    assert np.max(np.abs(V)) <= 1e-12 and np.max(np.abs(Om)) <= 1e-12


def test_mean_modes_decay_by_the_cn_factor(pkg):
    mz = 4 * VC.MEAN_N
    sz = O.Sizes(48, 48, mz)
    V0, O0 = VC.mean_state(sz)
    V, Om = _run(pkg, 48, 48, mz, V0, O0, VC.MEAN_STEPS, Re=VC.MEAN_RE, Ro=0.1, dt=VC.MEAN_DT)
    eu, ew = VC.mean_decay_errors(V0, O0, V, Om)
    assert eu < 1e-11 and ew < 1e-11, (eu, ew)


@pytest.mark.parametrize("mixed", [False, True])
def test_orr_sommerfeld_growth_rate(pkg, mixed):
    c, a = VC.os_mode()
    mx, my, mz = VC.OS_GRID
    sz = O.Sizes(mx, my, mz)
    V0, O0 = VC.os_state(sz, a)
    prec = pkg.PREC_MIXED if mixed else pkg.PREC_FP64
    V, _ = _run(pkg, mx, my, mz, V0, O0, VC.OS_STEPS, n_pi_x=2.0, n_pi_y=2.0, Re=VC.OS_RE, Ro=0.0,
                dt=VC.OS_DT, U=VC.POISEUILLE, precision=prec)
    lam = VC.os_rate(V, a)
    assert abs(lam.real - VC.ORSZAG_C.imag) < 3.7e-7, lam
    assert abs(lam - VC.cn_rate(c)) < (1e-7 if mixed else 1e-9), (lam, VC.cn_rate(c))
