"""Failure detection on the device without a device fault: a NaN or an Inf
injected into the host-staged state or AB2 history is reported by
dns_check_state (DNS_ERR_NONFINITE), a clean state passes, and the check
resets between calls."""
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
    # a non-finite AB2 history (written to recovery files) is reported too
    Nv, No = ctx.get_history()
    for bad in ((np.nan, 0), (0, np.inf)):
        Nv1, No1 = Nv.copy(), No.copy()
        Nv1[2, 1, 3] += bad[0]
        No1[7, 5, 2] += bad[1]
        ctx.set_history(Nv1, No1)
        with pytest.raises(pkg.DnsError, match="NaN or Inf"):
            ctx.check_state()
    ctx.set_history(Nv, No)
    ctx.check_state()
    ctx.step(3)
    ctx.synchronize()
    ctx.check_state()
    ctx.close()


def test_bounded_wait_times_out_and_the_context_recovers(pkg):
    """A staging wait that runs out (limit < 0: give up at once) makes the
    step report DNS_ERR_TIMEOUT without faulting; with the default limit back
    and the state set again, the context steps exactly as a fresh one."""
    mk = lambda: pkg.Context(pkg.make_params(48, 48, 128, Re=1300.0, Ro=0.1, dt=0.005,  # noqa: E731
                                             precision=pkg.PREC_MIXED))
    V0, O0 = pkg.seeded_state(32, 33, 32, 4.0, 2.0, 0.05, 0)
    ctx = mk()
    ctx.set_state(V0, O0)
    ctx.bootstrap()
    ctx.step(1)
    ctx.synchronize()
    ctx.set_wait_limit(-1)
    ctx.step(1)
    with pytest.raises(pkg.DnsError) as err:
        ctx.synchronize()
    assert err.value.status == 4  # DNS_ERR_TIMEOUT
    ctx.synchronize()  # reported once
    ctx.set_wait_limit()
    ctx.set_state(V0, O0)
    ctx.bootstrap()
    ctx.step(3)
    V, Om = ctx.get_state()
    ref = mk()
    ref.set_state(V0, O0)
    ref.bootstrap()
    ref.step(3)
    Vr, Or = ref.get_state()
    assert np.array_equal(V, Vr) and np.array_equal(Om, Or)
    ctx.close()
    ref.close()
