"""GPU: the slab-decomposed step (dns_slab_create / dns_slab_part) with all
ranks on one device, the exchanges as device copies between their buffers
(gpu-spectral-channel-dns_b200/slab.py, step_local), against the
undecomposed step of the same grid: bootstrap and 3 steps from the seeded
state, every rank's pencils gathered into the whole-grid arrays.  Each
kernel runs on the same lines, pencils and slots as in the whole-grid step,
so the two agree to rounding at most (asserted: 1e-13 relative; measured 0).
Grids: 48x48x128 (block-FFT forms, 2 and 3 ranks, FP64), 192x192x128 (warp
and tensor-copy forms, 2 ranks, both precisions)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("grid,R,prec", [
    ((48, 48, 128), 2, "fp64"), ((48, 48, 128), 3, "fp64"),
    ((192, 192, 128), 2, "fp64"), ((192, 192, 128), 2, "mixed")])
def test_slab_step_matches_whole_grid(pkg, grid, R, prec, parity_log):
    from importlib import import_module
    slab = import_module(pkg.__name__ + ".slab")
    P = pkg.PREC_FP64 if prec == "fp64" else pkg.PREC_MIXED
    mx, my, mz = grid
    params = pkg.make_params(mx, my, mz, Re=1300.0, Ro=0.1, dt=0.005, precision=P)
    full = pkg.Context(params)
    V0, O0 = pkg.seeded_state(full.Nx, full.Ny, full.Nz, amplitude=0.1, seed=0)
    full.set_state(V0, O0)
    full.bootstrap()
    full.step(3)
    Vf, Of = full.get_state()
    full.close()

    ctxs = [pkg.SlabContext(params, R, r) for r in range(R)]
    # every pencil owned once; the exchange sizes agree at both ends
    allp = np.sort(np.concatenate([c.pencils for c in ctxs]))
    assert np.array_equal(allp, np.arange(ctxs[0].H))
    for x in (0, 1):
        for r in range(R):
            for s in range(R):
                assert ctxs[r].exchange_bytes(x)[0][s] == ctxs[s].exchange_bytes(x)[1][r]
    for c in ctxs:
        c.scatter_state(V0, O0)
    bufs = slab.step_local(ctxs, boot=True)
    slab.step_local(ctxs, 3, bufs=bufs)
    Vs = np.zeros_like(Vf)
    Os = np.zeros_like(Of)
    for c in ctxs:
        c.gather_state(Vs, Os)
        c.close()
    ev, eo = _rel(Vs, Vf), _rel(Os, Of)
    parity_log.append(f"slab step {mx}x{my}x{mz} {prec}, {R} ranks on one device vs whole grid, "
                      f"bootstrap + 3 steps: v {ev:.1e} omega {eo:.1e}")
    assert ev < 1e-13 and eo < 1e-13, (ev, eo)


def test_slab_context_refuses_whole_grid_calls(pkg):
    c = pkg.SlabContext(pkg.make_params(48, 48, 128, Re=1300.0, Ro=0.1, dt=0.005), 2, 0)
    with pytest.raises(pkg.DnsError):
        c.step(1)
    with pytest.raises(pkg.DnsError):
        c.part(pkg.SLAB_Y3, 0, 0)  # no send buffer
    c.close()
