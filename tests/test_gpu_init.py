"""GPU: the reference's analytic initial condition (dns_init_flow).

initFlow (source/RPCFKernels.cu:358-431) on the device against the oracle's
restatement (itself checked against the closed form in
test_oracle_init.py): state to 1e-13 of its largest coefficient (the two
evaluations differ only in the rounding of sin/cos and of the transforms).
Then the reference's fresh start (source/main_loop.cpp:30-52: initFlow, the
extra previous step, steps) against the oracle's at 1e-11 relative L2 after
10 steps, FP64 form.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import rpcf_oracle as O  # noqa: E402


@pytest.fixture(autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


CASES = [
    dict(mx=24, my=24, mz=32, n_pi_x=4.0, n_pi_y=2.0, Re=500.0, Ro=0.0, dt=0.01),
    dict(mx=48, my=36, mz=64, n_pi_x=2.0, n_pi_y=3.0, Re=1300.0, Ro=0.1, dt=0.005),
]


def relL2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("case", CASES)
def test_init_flow_matches_oracle(pkg, case):
    ctx = pkg.Context(pkg.make_params(**case))
    ctx.init_flow()
    V, Om = ctx.get_state()
    sz = O.Sizes(case["mx"], case["my"], case["mz"])
    rV, rO = O.init_state(sz, case["n_pi_x"] / 2, case["n_pi_y"] / 2)
    assert np.max(np.abs(V - rV)) < 1e-13 * np.max(np.abs(rV))
    assert np.max(np.abs(Om - rO)) < 1e-13 * np.max(np.abs(rO))
    ctx.close()


@pytest.mark.parametrize("case", CASES)
def test_fresh_start_sequence(pkg, case):
    ctx = pkg.Context(pkg.make_params(**case))
    ctx.init_flow()
    ctx.bootstrap()
    ctx.step(10)
    ctx.synchronize()
    V, Om = ctx.get_state()
    sz = O.Sizes(case["mx"], case["my"], case["mz"])
    pb = O.Problem(O.Params(**case))
    pb.set_state(*O.init_state(sz, pb.aphi, pb.beta))
    pb.bootstrap()
    for _ in range(10):
        pb.step()
    assert relL2(V, pb.V) < 1e-11 and relL2(Om, pb.O) < 1e-11
    ctx.close()
