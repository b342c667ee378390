"""GPU parity: every entry point of libdnsb200.so against the CPU oracle.

The oracle (oracle/rpcf_oracle.py) restates the reference in FP64 NumPy and
is pinned to the reference's own known-answer tests.  Transform-type ops are
compared element-wise (relative to the field's max) at 1e-13; the full
FP64 step at 1e-11 relative L2 after 20 steps (the explicit-inverse solves
carry cond(A) * eps of rounding, measured here); the mixed-precision step
(FP32 transforms and Lamb vector, FP64 solves and state) at 1e-6.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import rpcf_oracle as O  # noqa: E402

SMALL = [(48, 48, 128), (24, 24, 32), (36, 48, 64)]


def cuda_ok():
    return torch.cuda.is_available()


@pytest.fixture(autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.skip("no CUDA device")


def ctx_for(pkg, mx, my, mz, **kw):
    defaults = dict(n_pi_x=4.0, n_pi_y=2.0, Re=1300.0, Ro=0.1, dt=0.005)
    defaults.update(kw)
    return pkg.Context(pkg.make_params(mx, my, mz, **defaults))


def spec_tensor(arr, sz):
    """(ny, hnx, L) complex -> device tensor of pitch mz complex."""
    t = torch.zeros((sz.ny, sz.hnx, sz.mz), dtype=torch.complex128)
    t[:, :, :arr.shape[-1]] = torch.from_numpy(np.ascontiguousarray(arr))
    return t.cuda()


def phys_tensor(arr, sz):
    """(pz, my, mx) real -> device tensor of row pitch mx+2 doubles."""
    t = torch.zeros((sz.pz, sz.my, sz.mx + 2), dtype=torch.float64)
    t[:, :, :sz.mx] = torch.from_numpy(np.ascontiguousarray(arr))
    return t.cuda()


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def relL2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run(ctx):
    torch.cuda.synchronize()
    return ctx


def rng_spec(sz, seed, L):
    r = np.random.default_rng(seed)
    return r.standard_normal((sz.ny, sz.hnx, L)) + 1j * r.standard_normal((sz.ny, sz.hnx, L))


@pytest.mark.parametrize("mx,my,mz", SMALL)
@pytest.mark.parametrize("pad", [0, 1])
def test_cheby_s2p_p2s(pkg, mx, my, mz, pad):
    sz = O.Sizes(mx, my, mz)
    ctx = ctx_for(pkg, mx, my, mz)
    S = rng_spec(sz, 1, sz.mz)
    # s2p
    t = spec_tensor(S, sz)
    torch.cuda.synchronize()
    ctx.cheby_s2p(t.data_ptr(), sz.mz * 16, pad)
    ctx.synchronize()
    ref = O.cheby_s2p(S, sz.mz, pad=(pad == 0))
    L = sz.mz if pad == 0 else sz.mz // 2
    assert rel(t.cpu().numpy()[..., :L], ref[..., :L]) < 1e-13
    # p2s
    t = spec_tensor(S, sz)
    torch.cuda.synchronize()
    ctx.cheby_p2s(t.data_ptr(), sz.mz * 16, pad)
    ctx.synchronize()
    ref = O.cheby_p2s(S, sz.mz, pad=(pad == 0))
    assert rel(t.cpu().numpy()[..., :L], ref[..., :L]) < 1e-13
    ctx.close()


@pytest.mark.parametrize("mx,my,mz", SMALL)
def test_transpose(pkg, mx, my, mz):
    sz = O.Sizes(mx, my, mz)
    ctx = ctx_for(pkg, mx, my, mz)
    r = np.random.default_rng(2)
    Cx = r.standard_normal((sz.pz, sz.my, sz.mx // 2 + 1)) + 1j * r.standard_normal((sz.pz, sz.my, sz.mx // 2 + 1))
    tx = torch.from_numpy(Cx).cuda()
    ts = torch.zeros((sz.ny, sz.hnx, sz.mz), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    ctx.cuda_transpose(pkg.FORWARD, tx.data_ptr(), (sz.mx // 2 + 1) * 16, ts.data_ptr(), sz.mz * 16)
    ctx.synchronize()
    ref = O.transpose_forward(Cx, sz)
    assert np.array_equal(ts.cpu().numpy()[..., :sz.pz], ref[..., :sz.pz])
    tx2 = torch.zeros_like(tx)
    torch.cuda.synchronize()
    ctx.cuda_transpose(pkg.BACKWARD, tx2.data_ptr(), (sz.mx // 2 + 1) * 16, ts.data_ptr(), sz.mz * 16)
    ctx.synchronize()
    back = O.transpose_backward(ref, sz, np.zeros_like(Cx))
    assert np.array_equal(tx2.cpu().numpy(), back)
    ctx.close()


@pytest.mark.parametrize("mx,my,mz", SMALL)
@pytest.mark.parametrize("pad", [0, 1])
def test_transform_3d_one(pkg, mx, my, mz, pad):
    sz = O.Sizes(mx, my, mz)
    ctx = ctx_for(pkg, mx, my, mz)
    S = rng_spec(sz, 3, sz.nz)
    ts = spec_tensor(S, sz)
    tp = torch.zeros((sz.pz, sz.my, sz.mx + 2), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.transform_3d_one(pkg.BACKWARD, tp.data_ptr(), (sz.mx + 2) * 8, ts.data_ptr(), sz.mz * 16, pad)
    ctx.synchronize()
    Sfull = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=complex)
    Sfull[..., :sz.nz] = S
    ref = O.transform_backward(Sfull, sz, pad=(pad == 0))
    got = tp.cpu().numpy()[..., :sz.mx]
    npl = sz.pz if pad == 0 else sz.nz
    assert rel(got[:npl], ref[:npl]) < 1e-13
    # forward on a smooth physical field built from the result
    P = ref.copy()
    if pad == 1:
        P = O.transform_backward(Sfull, sz, pad=True)
    tp2 = phys_tensor(P, sz)
    ts2 = torch.zeros((sz.ny, sz.hnx, sz.mz), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    ctx.transform_3d_one(pkg.FORWARD, tp2.data_ptr(), (sz.mx + 2) * 8, ts2.data_ptr(), sz.mz * 16, pad)
    ctx.synchronize()
    refS = O.transform_forward(P, sz, pad=(pad == 0))
    ncoef = sz.pz if pad == 0 else sz.nz
    assert rel(ts2.cpu().numpy()[..., :ncoef], refS[..., :ncoef]) < 1e-13
    ctx.close()


@pytest.mark.parametrize("mx,my,mz", SMALL)
def test_get_uvw(pkg, mx, my, mz):
    sz = O.Sizes(mx, my, mz)
    ctx = ctx_for(pkg, mx, my, mz)
    W = rng_spec(sz, 4, sz.nz)
    OZ = rng_spec(sz, 5, sz.nz)
    ts = [torch.zeros((sz.ny, sz.hnx, sz.mz), dtype=torch.complex128, device="cuda") for _ in range(6)]
    ts[2] = spec_tensor(W, sz)
    ts[5] = spec_tensor(OZ, sz)
    torch.cuda.synchronize()
    ctx.get_uvw([t.data_ptr() for t in ts], sz.mz * 16)
    ctx.synchronize()
    tw = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=complex)
    toz = np.zeros_like(tw)
    tw[..., :sz.nz] = W
    toz[..., :sz.nz] = OZ
    ref = O.get_uvw(tw, toz, sz, 2.0, 1.0)
    for i, (t, r) in enumerate(zip(ts, ref)):
        assert rel(t.cpu().numpy()[..., :sz.nz], r) < 1e-12, i


@pytest.mark.parametrize("mx,my,mz", SMALL[:2])
def test_compute_lamb(pkg, mx, my, mz):
    sz = O.Sizes(mx, my, mz)
    ctx = ctx_for(pkg, mx, my, mz, Ro=0.3)
    r = np.random.default_rng(6)
    F = [r.standard_normal((sz.pz, sz.my, sz.mx)) for _ in range(6)]
    ts = [phys_tensor(f, sz) for f in F]
    torch.cuda.synchronize()
    ctx.compute_lamb([t.data_ptr() for t in ts], [t.data_ptr() for t in ts[:3]], (sz.mx + 2) * 8)
    ctx.synchronize()
    ref = O.lamb(*F, sz, 0.3)
    for t, rr in zip(ts[:3], ref):
        assert rel(t.cpu().numpy()[..., :sz.mx], rr) < 1e-15


@pytest.mark.parametrize("mx,my,mz", SMALL)
def test_rhs_nonlinear(pkg, mx, my, mz):
    sz = O.Sizes(mx, my, mz)
    ctx = ctx_for(pkg, mx, my, mz)
    L = [rng_spec(sz, 7 + i, sz.nz) for i in range(3)]
    ts = [spec_tensor(x, sz) for x in L]
    torch.cuda.synchronize()
    ctx.rhs_nonlinear(ts[0].data_ptr(), ts[1].data_ptr(), ts[2].data_ptr(), sz.mz * 16)
    ctx.synchronize()
    full = []
    for x in L:
        f = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=complex)
        f[..., :sz.nz] = x
        full.append(f)
    hv, ho = O.rhs_nonlinear(full[0], full[1], full[2], sz, 2.0, 1.0)
    assert rel(ts[0].cpu().numpy()[..., :sz.nz], hv) < 1e-12
    assert rel(ts[1].cpu().numpy()[..., :sz.nz], ho) < 1e-12


@pytest.mark.parametrize("mx,my,mz", SMALL[:2])
def test_init_aux_matrix_and_solve(pkg, mx, my, mz):
    sz = O.Sizes(mx, my, mz)
    p = O.Params(mx, my, mz, Re=1300.0, Ro=0.1, dt=0.005)
    ctx = ctx_for(pkg, mx, my, mz)
    pb = O.Problem(p)
    nn = sz.nz * sz.nz
    iv = torch.zeros((sz.ny, sz.hnx, sz.nz, sz.nz), dtype=torch.complex128, device="cuda")
    io = torch.zeros_like(iv)
    torch.cuda.synchronize()
    ctx.init_aux_matrix(iv.data_ptr(), io.data_ptr())
    ctx.synchronize()
    gv = iv.cpu().numpy()
    go = io.cpu().numpy()
    # forward error of an explicit inverse is ~cond(A) eps; check A * inv = I
    pb.build_inverses()
    eye = np.eye(sz.nz)
    rv_ = np.max(np.abs(np.einsum("yxij,yxjk->yxik", pb.A_v, gv) - eye))
    ro_ = np.max(np.abs(np.einsum("yxij,yxjk->yxik", pb.A_o, go) - eye))
    assert rv_ < 1e-8 and ro_ < 1e-10, (rv_, ro_)
    # solveEq with those inverses
    R = rng_spec(sz, 11, sz.nz)
    t = spec_tensor(R, sz)
    torch.cuda.synchronize()
    ctx.solve_eq(iv.data_ptr(), t.data_ptr(), sz.nz, sz.mz * 16)  # device buffers
    ctx.synchronize()
    ref = np.einsum("yxij,yxj->yxi", gv, R)
    assert rel(t.cpu().numpy()[..., :sz.nz], ref) < 1e-13


def oracle_run(mx, my, mz, nsteps, amp=0.05, seed=0, **kw):
    from conftest import load_package
    pkg = load_package()
    p = O.Params(mx, my, mz, **kw)
    pb = O.Problem(p)
    sz = pb.sz
    V, Om = pkg.seeded_state(sz.nx, sz.nz, sz.ny, p.n_pi_x, p.n_pi_y, amp, seed)
    pb.set_state(V, Om)
    pb.bootstrap()
    hist = []
    for _ in range(nsteps):
        pb.step()
        hist.append((pb.V.copy(), pb.O.copy()))
    return (V, Om), hist, pb


STEP_CASES = [
    dict(mx=48, my=48, mz=128, Re=1300.0, Ro=0.1, dt=0.005),
    dict(mx=24, my=24, mz=32, Re=500.0, Ro=0.0, dt=0.01),
    dict(mx=36, my=48, mz=64, Re=2000.0, Ro=0.2, dt=0.002, U=(0.0, 1.0, 0.0)),
    dict(mx=48, my=36, mz=64, Re=8400.0, Ro=0.0, dt=0.002, U=(1.0, 0.0, -1.0)),
    # wall-normal lengths of the 256x129x256 workload (padded DCT on 512 points)
    dict(mx=48, my=48, mz=512, Re=3000.0, Ro=0.02, dt=0.001),
    # streamwise / spanwise lengths of that workload (384-point lines)
    dict(mx=384, my=384, mz=32, Re=3000.0, Ro=0.02, dt=0.001),
]


@pytest.mark.parametrize("case", STEP_CASES)
def test_step_fp64_matches_oracle(pkg, case):
    case = dict(case)
    U = case.pop("U", (0.5, 0.5, 0.0))
    nsteps = 20
    (V0, O0), hist, pb = oracle_run(case["mx"], case["my"], case["mz"], nsteps,
                                    Re=case["Re"], Ro=case["Ro"], dt=case["dt"], prof=U)
    ctx = pkg.Context(pkg.make_params(case["mx"], case["my"], case["mz"], Re=case["Re"],
                                      Ro=case["Ro"], dt=case["dt"], U=U))
    ctx.set_state(V0, O0)
    ctx.bootstrap()
    nvp, nop = ctx.get_history()
    Nv, No = O.Problem.nonlinear(_fresh(pb, V0, O0))
    assert relL2(nvp, Nv) < 1e-12 and relL2(nop, No) < 1e-12
    for k in range(nsteps):
        ctx.step(1)
        ctx.synchronize()
        if k in (0, 1, nsteps - 1):
            V, Om = ctx.get_state()
            eV = relL2(V, hist[k][0])
            eO = relL2(Om, hist[k][1])
            assert eV < 1e-11 and eO < 1e-11, (k, eV, eO)
    ctx.close()


def _fresh(pb, V, Om):
    q = O.Problem(pb.p)
    q.set_state(V, Om)
    return q


# the tensor-staged spanwise passes at 192 points and the wall-normal warp
# passes at 256 points in one step (the 384-point x, zb, zf kernels and the
# 512-point y kernels are covered by the cases above), 5 steps: the oracle
# takes ~6 s a step here
MIXED_CASES = STEP_CASES[:2] + STEP_CASES[4:] + [
    dict(mx=192, my=192, mz=256, Re=3000.0, Ro=0.02, dt=0.001, steps=5),
]


@pytest.mark.parametrize("case", MIXED_CASES)
def test_step_mixed_close_to_fp64(pkg, case):
    case = dict(case)
    U = case.pop("U", (0.5, 0.5, 0.0))
    nsteps = case.pop("steps", 20)
    (V0, O0), hist, _ = oracle_run(case["mx"], case["my"], case["mz"], nsteps,
                                   Re=case["Re"], Ro=case["Ro"], dt=case["dt"], prof=U)
    ctx = pkg.Context(pkg.make_params(case["mx"], case["my"], case["mz"], Re=case["Re"],
                                      Ro=case["Ro"], dt=case["dt"], U=U,
                                      precision=pkg.PREC_MIXED))
    ctx.set_state(V0, O0)
    ctx.bootstrap()
    ctx.step(nsteps)
    ctx.synchronize()
    V, Om = ctx.get_state()
    assert relL2(V, hist[-1][0]) < 1e-6
    assert relL2(Om, hist[-1][1]) < 1e-6
    ctx.close()


# The 48-run ensemble (12 runs each of 32x33x32, 64x49x64, 96x65x96 and
# 128x97x128 modes; Re ~ U[500, 3000], Ro ~ U[0, 0.3], dt 0.002, seeded field
# of amplitude 0.1, seeds 1000 + m; the runs are independent replicas): the
# first member of each size, FP64 step against the oracle at every step and
# the mixed form at the last.  Few steps: the oracle takes ~20 s a step at
# 128x97x128.
ENSEMBLE_SIZES = [(48, 48, 128), (96, 96, 192), (144, 144, 256), (192, 192, 384)]
_ensemble_cache = {}


def ensemble_member(m):
    mx, my, mz = ENSEMBLE_SIZES[m // 12]
    r = np.random.default_rng(1000 + m)
    return dict(mx=mx, my=my, mz=mz, Re=float(r.uniform(500.0, 3000.0)),
                Ro=float(r.uniform(0.0, 0.3)), dt=0.002, seed=1000 + m,
                steps=2 if m // 12 == 3 else 3)


def ensemble_oracle(m):
    if m not in _ensemble_cache:
        c = ensemble_member(m)
        _ensemble_cache[m] = oracle_run(c["mx"], c["my"], c["mz"], c["steps"], amp=0.1,
                                        seed=c["seed"], Re=c["Re"], Ro=c["Ro"], dt=c["dt"])
    return _ensemble_cache[m]


@pytest.mark.parametrize("m", [0, 12, 24, 36])
def test_ensemble_member_fp64(pkg, m):
    c = ensemble_member(m)
    (V0, O0), hist, _ = ensemble_oracle(m)
    ctx = pkg.Context(pkg.make_params(c["mx"], c["my"], c["mz"], Re=c["Re"], Ro=c["Ro"], dt=c["dt"]))
    ctx.set_state(V0, O0)
    ctx.bootstrap()
    for k in range(c["steps"]):
        ctx.step(1)
        ctx.synchronize()
        V, Om = ctx.get_state()
        eV, eO = relL2(V, hist[k][0]), relL2(Om, hist[k][1])
        assert eV < 1e-11 and eO < 1e-11, (m, k, eV, eO)
    ctx.close()


@pytest.mark.parametrize("m", [12, 24, 36])
def test_ensemble_member_mixed(pkg, m):
    c = ensemble_member(m)
    (V0, O0), hist, _ = ensemble_oracle(m)
    ctx = pkg.Context(pkg.make_params(c["mx"], c["my"], c["mz"], Re=c["Re"], Ro=c["Ro"], dt=c["dt"],
                                      precision=pkg.PREC_MIXED))
    ctx.set_state(V0, O0)
    ctx.bootstrap()
    ctx.step(c["steps"])
    ctx.synchronize()
    V, Om = ctx.get_state()
    assert relL2(V, hist[-1][0]) < 1e-6 and relL2(Om, hist[-1][1]) < 1e-6, m
    ctx.close()


def test_step_many_equals_one_by_one(pkg):
    """Concurrent stepping of independent runs (one stream each) gives every
    run exactly the state it reaches alone: one member of each ensemble size,
    both precisions."""
    runs = []
    for m in (0, 12, 24, 36):
        c = ensemble_member(m)
        for prec in (pkg.PREC_MIXED, pkg.PREC_FP64):
            Nx, Nz, Ny = c["mx"] // 3 * 2, c["my"] // 3 * 2, c["mz"] // 4 + 1
            V0, O0 = pkg.seeded_state(Nx, Ny, Nz, 4.0, 2.0, 0.1, c["seed"])
            runs.append((c, prec, V0, O0))

    def make(c, prec, V0, O0):
        ctx = pkg.Context(pkg.make_params(c["mx"], c["my"], c["mz"], Re=c["Re"], Ro=c["Ro"],
                                          dt=c["dt"], precision=prec))
        ctx.set_state(V0, O0)
        ctx.bootstrap()
        return ctx

    alone = []
    for r in runs:
        ctx = make(*r)
        ctx.step(4)
        ctx.synchronize()
        alone.append(ctx.get_state())
        ctx.close()
    ctxs = [make(*r) for r in runs]
    pkg.step_many(ctxs, 4)
    for ctx, (Va, Oa) in zip(ctxs, alone):
        ctx.synchronize()
        V, Om = ctx.get_state()
        assert np.array_equal(V, Va) and np.array_equal(Om, Oa)
        ctx.close()
    dup = make(*runs[0])
    with pytest.raises(pkg.DnsError):
        pkg.step_many([dup, dup], 1)
    dup.close()
