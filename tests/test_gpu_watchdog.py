"""Failure detection on the device without a device fault: a NaN or an Inf
injected into the host-staged state is reported by dns_check_state
(DNS_ERR_NONFINITE), a clean state passes, and the check resets between
calls."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_check_state_reports_nonfinite_values(pkg, precision):
    prec = pkg.PREC_MIXED if precision == "mixed" else pkg.PREC_FP64
    ctx = pkg.Context(pkg.make_params(24, 24, 32, Re=500.0, Ro=0.0, dt=0.01, precision=prec))
    V0, O0 = pkg.seeded_state(16, 9, 16, 4.0, 2.0, 0.05, 0)
    ctx.set_state(V0, O0)
    ctx.check_state()
    for bad_v, bad_o in ((np.nan, None), (None, np.inf), (complex(0.0, -np.inf), None)):
        V, Om = V0.copy(), O0.copy()
        if bad_v is not None:
            V[3, 2, 4] = bad_v
        if bad_o is not None:
            Om[15, 8, 8] = bad_o
        ctx.set_state(V, Om)
        with pytest.raises(pkg.DnsError, match="NaN or Inf"):
            ctx.check_state()
    ctx.set_state(V0, O0)
    ctx.check_state()
    ctx.bootstrap()
    ctx.step(3)
    ctx.synchronize()
    ctx.check_state()
    ctx.close()
