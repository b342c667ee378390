"""GPU: every compiled variant of every tunable pass (wall-normal backward and
forward passes, spanwise inverse and forward passes, the streamwise pass,
the block shapes of the banded solve) gives the step of the
default variants: in FP64 to 1e-12 relative (the parity bar; measured
differences are rounding, ~1e-15), in the mixed form to 1e-6 against the
FP64 step.  384x384x128 (256x33x256 modes): lengths with warp plans in both
precisions (Px = Pz = 384, M = 128), so every variant is available,
192x192x128 (its streamwise warp form), and the ensemble grids 48x48x128,
96x96x192 and 144x144x256 (warp plans whose passes leave lanes idle in
their last round); 3 steps after the bootstrap from the seeded state,
Re 1300, Ro 0.1, dt 0.005."""
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


GRID = (384, 384, 128)


def _run(pkg, prec, variants=None, steps=3, grid=GRID):
    c = pkg.Context(pkg.make_params(*grid, Re=1300.0, Ro=0.1, dt=0.005, precision=prec))
    for p, v in (variants or {}).items():
        c.set_variant(p, v)
    c.set_state(*pkg.seeded_state(c.Nx, c.Ny, c.Nz, amplitude=0.1, seed=0))
    c.bootstrap()
    c.step(steps)
    V, O = c.get_state()
    got = {p: c.get_variant(p) for p in range(pkg.NUM_PASSES)}
    c.close()
    return V, O, got


def _available(pkg, prec, grid=GRID):
    c = pkg.Context(pkg.make_params(*grid, Re=1300.0, Ro=0.1, dt=0.005, precision=prec))
    out = {}
    for p in range(pkg.NUM_PASSES):
        out[p] = []
        for v in range(pkg.MAX_VARIANTS):
            try:
                c.set_variant(p, v)
                out[p].append(v)
            except pkg.DnsError:
                pass
    c.close()
    return out


def test_available_variants(pkg):
    a64 = _available(pkg, pkg.PREC_FP64)
    amx = _available(pkg, pkg.PREC_MIXED)
    rings = [pkg.Y2_RING3_12K, pkg.Y2_RING3_12K_EF, pkg.Y2_RING2_8K_EF, pkg.Y2_RING3_8K_EF]
    assert a64 == {pkg.PASS_Y3: [pkg.Y3_FFT, pkg.Y3_BLOCK], pkg.PASS_Y1: [pkg.Y1_WARP, pkg.Y1_BLOCK],
                   pkg.PASS_ZB: [pkg.Z_WARP, pkg.Z_BLOCK], pkg.PASS_ZF: [pkg.Z_WARP, pkg.Z_BLOCK],
                   pkg.PASS_Y2: rings, pkg.PASS_X: [pkg.X_WARP3, pkg.X_WARP6, pkg.X_BLOCK]}
    assert amx[pkg.PASS_X] == [pkg.X_WARP3, pkg.X_WARP6, pkg.X_BLOCK]
    assert amx[pkg.PASS_Y2] == rings
    assert amx[pkg.PASS_ZB] == [pkg.Z_TENSOR_COPY, pkg.Z_WARP, pkg.Z_BLOCK]
    assert amx[pkg.PASS_ZF] == [pkg.Z_TENSOR_COPY, pkg.Z_WARP, pkg.Z_BLOCK]
    assert amx[pkg.PASS_Y1] == [pkg.Y1_WARP, pkg.Y1_BLOCK]
    assert amx[pkg.PASS_Y3] == [pkg.Y3_FFT, pkg.Y3_BLOCK]  # the tensor form needs Ny = 129


ENSEMBLE_GRIDS = [(48, 48, 128), (96, 96, 192), (144, 144, 256)]


@pytest.mark.parametrize("grid", ENSEMBLE_GRIDS)
def test_ensemble_grids_have_warp_forms(pkg, grid):
    for prec in (pkg.PREC_FP64, pkg.PREC_MIXED):
        a = _available(pkg, prec, grid)
        assert a[pkg.PASS_X] == [pkg.X_WARP3, pkg.X_WARP6, pkg.X_BLOCK], (grid, prec)
        assert pkg.Z_WARP in a[pkg.PASS_ZB] and pkg.Z_WARP in a[pkg.PASS_ZF], (grid, prec)
        assert a[pkg.PASS_Y1] == [pkg.Y1_WARP, pkg.Y1_BLOCK], (grid, prec)
        assert a[pkg.PASS_Y3][0] == pkg.Y3_FFT, (grid, prec)


@pytest.mark.parametrize("grid", [GRID, (192, 192, 128)] + ENSEMBLE_GRIDS)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_every_variant_same_step(pkg, prec, grid, parity_log):
    P = pkg.PREC_FP64 if prec == "fp64" else pkg.PREC_MIXED
    V64, O64, _ = _run(pkg, pkg.PREC_FP64, grid=grid)
    base = (V64, O64)
    tol = 1e-12 if prec == "fp64" else 1e-6
    avail = _available(pkg, P, grid)
    worst = {}
    for p, vs in avail.items():
        for v in vs:
            V, O, got = _run(pkg, P, {p: v}, grid=grid)
            assert got[p] == v
            e = max(_rel(V, base[0]), _rel(O, base[1]))
            worst[f"{pkg.PASS_NAMES[p]}:{pkg.VARIANT_NAMES[p][v]}"] = e
            assert e < tol, (prec, pkg.PASS_NAMES[p], pkg.VARIANT_NAMES[p][v], e)
    parity_log.append(f"variants, {prec}, 3 steps at {grid[0]}x{grid[1]}x{grid[2]} vs the FP64 default step: " +
                      ", ".join(f"{k} {e:.1e}" for k, e in worst.items()))
