"""The step function by function: the reference-layout drop-ins for
getNonlinear (+ the worker's no-pad s2p), get_rhs_v, get_rhs_omega, the mean
modes, solveEq on host buffers and the operators of initAuxMatrix, each
against the oracle; then the reference's whole nextStep sequence
(source/solver.cpp:35-101) run through these entry points on host buffers,
against the oracle's step."""
import numpy as np
import pytest
import torch

from oracle import rpcf_oracle as O

pytestmark = pytest.mark.gpu

GRIDS = [(48, 48, 128), (36, 48, 64)]


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def problem(mx, my, mz, U=(0.5, 0.5, 0.0), Re=1300.0, Ro=0.1, dt=0.005):
    return O.Problem(O.Params(mx, my, mz, Re=Re, Ro=Ro, dt=dt, prof=U))


def context(pkg, mx, my, mz, U=(0.5, 0.5, 0.0), Re=1300.0, Ro=0.1, dt=0.005):
    return pkg.Context(pkg.make_params(mx, my, mz, Re=Re, Ro=Ro, dt=dt, U=U))


def rand(sz, seed, decay=0.8):
    r = np.random.default_rng(seed)
    n = np.arange(sz.nz)
    a = (r.standard_normal((sz.ny, sz.hnx, sz.nz)) + 1j * r.standard_normal((sz.ny, sz.hnx, sz.nz)))
    return a * decay ** n


def dev(a, mz):
    """(ny, hnx, nz) complex -> device pencils of pitch mz*16 bytes."""
    t = torch.zeros(a.shape[:2] + (mz,), dtype=torch.complex128, device="cuda")
    t[..., :a.shape[2]] = torch.from_numpy(a).cuda()
    torch.cuda.synchronize()
    return t


@pytest.mark.parametrize("mx,my,mz", GRIDS)
@pytest.mark.parametrize("where", ["host", "device"])
def test_nonlinear_matches_oracle(pkg, mx, my, mz, where):
    pb = problem(mx, my, mz)
    sz = pb.sz
    V, Om = pkg.seeded_state(sz.nx, sz.nz, sz.ny, amplitude=0.1, seed=3)
    pb.set_state(V, Om)
    Nv, No = pb.nonlinear()
    ctx = context(pkg, mx, my, mz)
    if where == "host":
        nv = np.zeros_like(V)
        no = np.zeros_like(V)
        ctx.nonlinear(V.ctypes.data, Om.ctypes.data, nv.ctypes.data, no.ctypes.data, sz.nz * 16, pkg.HOST)
    else:
        tv, to = dev(V, sz.mz), dev(Om, sz.mz)
        tn, tm = dev(np.zeros_like(V), sz.mz), dev(np.zeros_like(V), sz.mz)
        ctx.nonlinear(tv.data_ptr(), to.data_ptr(), tn.data_ptr(), tm.data_ptr(), sz.mz * 16)
        ctx.synchronize()
        nv, no = tn.cpu().numpy()[..., :sz.nz], tm.cpu().numpy()[..., :sz.nz]
    assert rel(nv, Nv) < 1e-12 and rel(no, No) < 1e-12, (rel(nv, Nv), rel(no, No))
    # the context's own state is untouched: a step from its state still works
    with pytest.raises(pkg.DnsError):
        ctx.step(1)  # no state was set
    ctx.close()


@pytest.mark.parametrize("U", [(0.5, 0.5, 0.0), (1.0, 0.0, -1.0)])
@pytest.mark.parametrize("where", ["host", "device"])
def test_rhs_v_and_omega_match_oracle(pkg, U, where):
    mx, my, mz = 48, 48, 128
    pb = problem(mx, my, mz, U=U)
    sz = pb.sz
    V, Vn, Om = rand(sz, 1), rand(sz, 2), rand(sz, 3)
    Nv, Nvp, No, Nop = (rand(sz, s, 1.0) for s in (4, 5, 6, 7))
    # oracle: get_rhs_v (rhs.cpp:185-219) without the mean modes
    ev = pb.linear_v(V)
    k = np.arange(4, sz.nz)
    ev[..., 4:] += (Nv[..., k - 2] * 1.5 - Nvp[..., k - 2] * 0.5) * pb.p.dt
    ev[0, 0] = V[0, 0]
    eo = pb.linear_omega(Om, Vn, V)
    i = np.arange(2, sz.nz)
    eo[..., 2:] += (No[..., i - 1] * 1.5 - Nop[..., i - 1] * 0.5) * pb.p.dt
    eo[0, 0] = Om[0, 0]
    ctx = context(pkg, mx, my, mz, U=U)
    vp0 = rand(sz, 9)
    if where == "host":
        rv, rvp, ro = V.copy(), vp0.copy(), Om.copy()
        p = sz.nz * 16
        ctx.rhs_v(rv.ctypes.data, rvp.ctypes.data, Nv.ctypes.data, Nvp.ctypes.data, p, pkg.HOST)
        ctx.rhs_omega(ro.ctypes.data, No.ctypes.data, Nop.ctypes.data, Vn.ctypes.data, V.ctypes.data,
                      p, pkg.HOST)
    else:
        t = {n: dev(a, sz.mz) for n, a in dict(rv=V, rvp=vp0, nv=Nv, nvp=Nvp, ro=Om, no=No, nop=Nop,
                                                vn=Vn, v=V).items()}
        p = sz.mz * 16
        ctx.rhs_v(t["rv"].data_ptr(), t["rvp"].data_ptr(), t["nv"].data_ptr(), t["nvp"].data_ptr(), p)
        ctx.rhs_omega(t["ro"].data_ptr(), t["no"].data_ptr(), t["nop"].data_ptr(), t["vn"].data_ptr(),
                      t["v"].data_ptr(), p)
        ctx.synchronize()
        rv, rvp, ro = (t[n].cpu().numpy()[..., :sz.nz] for n in ("rv", "rvp", "ro"))
    assert rel(rv, ev) < 1e-13, rel(rv, ev)
    assert rel(ro, eo) < 1e-13, rel(ro, eo)
    # rhs_v_p <- v^n on every pencil but (0,0), which keeps its old value
    exp_p = V.copy()
    exp_p[0, 0] = vp0[0, 0]
    assert np.array_equal(rvp, exp_p)
    ctx.close()


def test_rhs_mean_matches_oracle(pkg):
    mx, my, mz = 48, 48, 128
    pb = problem(mx, my, mz)
    sz = pb.sz
    r = np.random.default_rng(11)
    vec = [np.ascontiguousarray(r.standard_normal(sz.nz) + 1j * r.standard_normal(sz.nz))
           for _ in range(6)]
    eu = pb.linear_u0(vec[0], vec[1], vec[2])
    ew = pb.linear_u0(vec[3], vec[4], vec[5])
    ctx = context(pkg, mx, my, mz)
    u0, w0 = vec[0].copy(), vec[3].copy()
    ctx.rhs_mean(u0.ctypes.data, vec[1].ctypes.data, vec[2].ctypes.data, w0.ctypes.data,
                 vec[4].ctypes.data, vec[5].ctypes.data, pkg.HOST)
    assert rel(u0, eu) < 1e-13 and rel(w0, ew) < 1e-13
    ctx.close()


@pytest.mark.parametrize("mx,my,mz", GRIDS)
def test_operators_and_tables_match_oracle(pkg, mx, my, mz):
    pb = problem(mx, my, mz)
    sz = pb.sz
    pb.build_inverses()
    ctx = context(pkg, mx, my, mz)
    T0, T2, T4, U, dU, ddU = ctx.operator_tables()
    for a, b in ((T0, pb.T0), (T2, pb.T2), (T4, pb.T4), (U, pb.U), (dU, pb.dU), (ddU, pb.ddU)):
        assert np.array_equal(a, b)
    Av = np.zeros((sz.ny, sz.hnx, sz.nz, sz.nz), dtype=np.complex128)
    Ao = np.zeros_like(Av)
    ctx.operator_matrices(Av.ctypes.data, Ao.ctypes.data, pkg.HOST)
    # entries as the reference rounds them; the oracle's NumPy evaluation
    # order may differ in the last bit
    assert np.max(np.abs(Av - pb.A_v)) <= 1e-15 * np.max(np.abs(pb.A_v))
    assert np.max(np.abs(Ao - pb.A_o)) <= 1e-15 * np.max(np.abs(pb.A_o))
    ctx.close()


def test_solve_eq_on_host_buffers(pkg):
    mx, my, mz = 36, 48, 64
    sz = O.Sizes(mx, my, mz)
    r = np.random.default_rng(5)
    inv = (r.standard_normal((sz.ny, sz.hnx, sz.nz, sz.nz)) +
           1j * r.standard_normal((sz.ny, sz.hnx, sz.nz, sz.nz)))
    b = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=np.complex128)  # the reference's pitch: mz complex
    b[..., :sz.nz] = rand(sz, 6)
    exp = np.einsum("yxij,yxj->yxi", inv, b[..., :sz.nz])
    ctx = context(pkg, mx, my, mz)
    pad = b[..., sz.nz:].copy()
    ctx.solve_eq(inv.ctypes.data, b.ctypes.data, sz.nz, sz.mz * 16, pkg.HOST)
    assert rel(b[..., :sz.nz], exp) < 1e-14
    assert np.array_equal(b[..., sz.nz:], pad)  # beyond N: untouched
    ctx.close()


@pytest.mark.parametrize("U,Ro", [((0.5, 0.5, 0.0), 0.1), ((1.0, 0.0, -1.0), 0.0)])
def test_reference_step_sequence_on_host_buffers(pkg, U, Ro):
    """nextStep as the reference runs it (source/solver.cpp:35-101) with
    every piece on the GPU through the C ABI and every buffer on the host:
    nonlinear phase + history swap + mean-mode lambda (rhs.cpp:60-183),
    get_rhs_v, solveEq(v), get_rhs_omega, solveEq(omega), save_0_v_omega_y;
    the AB2 history starts as the oracle's bootstrap leaves it."""
    mx, my, mz = 48, 48, 128
    pb = problem(mx, my, mz, U=U, Ro=Ro)
    sz = pb.sz
    V0, O0 = pkg.seeded_state(sz.nx, sz.nz, sz.ny, amplitude=0.05, seed=0)
    pb.set_state(V0, O0)
    pb.bootstrap()
    ctx = context(pkg, mx, my, mz, U=U, Ro=Ro)
    nz, p = sz.nz, sz.nz * 16
    inv_v = np.zeros((sz.ny, sz.hnx, nz, nz), dtype=np.complex128)
    inv_o = np.zeros_like(inv_v)
    ctx.init_aux_matrix(inv_v, inv_o, pkg.HOST)
    rhs_v, rhs_o = V0.copy(), O0.copy()
    rhs_v_p = V0.copy()
    nl_v, nl_o = pb.Nv_p.copy(), pb.No_p.copy()
    nl_v_p, nl_o_p = np.zeros_like(nl_v), np.zeros_like(nl_o)
    lx0, lz0 = pb.lx0_p.copy(), pb.lz0_p.copy()
    tv0, to0 = V0[0, 0].copy(), O0[0, 0].copy()
    H = pkg.HOST
    for step in range(5):
        pb.step()
        # get_rhs_v: the nonlinear phase on the worker (rhs.cpp:83-127)
        nl_v, nl_v_p = nl_v_p, nl_v
        nl_o, nl_o_p = nl_o_p, nl_o
        ctx.nonlinear(rhs_v.ctypes.data, rhs_o.ctypes.data, nl_v.ctypes.data, nl_o.ctypes.data, p, H)
        lx0_p, lz0_p = lx0, lz0
        lx0, lz0 = nl_v[0, 0].copy(), nl_o[0, 0].copy()
        ctx.rhs_v(rhs_v.ctypes.data, rhs_v_p.ctypes.data, nl_v.ctypes.data, nl_v_p.ctypes.data, p, H)
        ctx.rhs_mean(tv0.ctypes.data, lx0.ctypes.data, lx0_p.ctypes.data, to0.ctypes.data,
                     lz0.ctypes.data, lz0_p.ctypes.data, H)
        rhs_v[0, 0] = tv0
        rhs_o[0, 0] = to0
        ctx.solve_eq(inv_v.ctypes.data, rhs_v.ctypes.data, nz, p, H)
        ctx.rhs_omega(rhs_o.ctypes.data, nl_o.ctypes.data, nl_o_p.ctypes.data, rhs_v.ctypes.data,
                      rhs_v_p.ctypes.data, p, H)
        ctx.solve_eq(inv_o.ctypes.data, rhs_o.ctypes.data, nz, p, H)
        tv0, to0 = rhs_v[0, 0].copy(), rhs_o[0, 0].copy()  # save_0_v_omega_y
        ev, eo = rel(rhs_v, pb.V), rel(rhs_o, pb.O)
        assert ev < 1e-12 and eo < 1e-12, (step, ev, eo)
    ctx.close()
