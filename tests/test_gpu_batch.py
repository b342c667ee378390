"""GPU: batches of runs (dns_create_batch, one launch per pass for all runs
of one grid) against the same runs as separate contexts.  Every kernel sees
the same lines, pencils and slots of each run as in a context of its own,
with that run's Re, Ro and dt, so a batched run equals its separate run to
rounding at most (asserted 1e-13 relative; measured 0).  Three runs with
different Re, Ro, dt, bootstrap and 3 steps from seeded states, both
precisions, on a grid with warp plans in every direction (384x384x128) and
on a small one (48x48x128, block forms)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


RUNS = [dict(Re=1300.0, Ro=0.1, dt=0.005), dict(Re=800.0, Ro=0.0, dt=0.002), dict(Re=2500.0, Ro=0.25, dt=0.004)]


@pytest.mark.parametrize("grid", [(384, 384, 128), (48, 48, 128)])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_matches_separate_runs(pkg, grid, prec, parity_log):
    P = pkg.PREC_FP64 if prec == "fp64" else pkg.PREC_MIXED
    mx, my, mz = grid
    plist = [pkg.make_params(mx, my, mz, precision=P, **r) for r in RUNS]
    b = pkg.BatchContext(plist)
    states = [pkg.seeded_state(b.Nx, b.Ny, b.Nz, amplitude=0.1, seed=7 + i) for i in range(len(RUNS))]
    b.set_state(np.stack([s[0] for s in states]), np.stack([s[1] for s in states]))
    b.bootstrap()
    b.step(3)
    Vb, Ob = b.get_state()
    Nvb, Nob = b.get_history()
    b.close()
    worst = 0.0
    for i, (p, (V0, O0)) in enumerate(zip(plist, states)):
        c = pkg.Context(p)
        c.set_state(V0, O0)
        c.bootstrap()
        c.step(3)
        V, O = c.get_state()
        Nv, No = c.get_history()
        c.close()
        for a, r in ((Vb[i], V), (Ob[i], O), (Nvb[i], Nv), (Nob[i], No)):
            worst = max(worst, float(np.linalg.norm(a - r) / np.linalg.norm(r)))
    parity_log.append(f"batch of {len(RUNS)} runs {mx}x{my}x{mz} {prec} vs separate contexts, "
                      f"bootstrap + 3 steps, state and history: {worst:.1e}")
    assert worst < 1e-13, worst


def test_batch_refuses_single_run_entries(pkg):
    b = pkg.BatchContext([pkg.make_params(48, 48, 128, **r) for r in RUNS])
    with pytest.raises(pkg.DnsError):
        b.init_flow()
    with pytest.raises(pkg.DnsError):
        pkg.BatchContext([pkg.make_params(48, 48, 128), pkg.make_params(96, 96, 128)])
    b.close()
