"""GPU: recovery files and physical field output in the reference's formats.

write_recover_data / read_recover_data (source/output.cpp:105-178): a run
restarted from a recovery file continues the run that wrote it.  The state
and the AB2 history cross the file as pencils of collocation values, which the
library converts to and from its Chebyshev-coefficient history; the restarted
run must agree with the uninterrupted one to 1e-12 relative L2 after further
steps (FP64 form).

output_velocity / write_velocity (source/output.cpp:19-103): the velocity and
vorticity files hold u, v, w (resp. omega_x, omega_y, omega_z) as pz planes of
my rows of mx doubles; compared with the oracle's backward transforms of
getUVW at 1e-12 of each field's maximum.
"""
import os

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
    dict(mx=24, my=24, mz=32, Re=500.0, Ro=0.0, dt=0.01),
    dict(mx=48, my=48, mz=128, Re=1300.0, Ro=0.1, dt=0.005),
]


def relL2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def make_ctx(pkg, case, precision=None):
    kw = dict(Re=case["Re"], Ro=case["Ro"], dt=case["dt"])
    if precision is not None:
        kw["precision"] = precision
    return pkg.Context(pkg.make_params(case["mx"], case["my"], case["mz"], **kw))


def seeded(pkg, case, amp=0.05, seed=3):
    sz = O.Sizes(case["mx"], case["my"], case["mz"])
    return pkg.seeded_state(sz.nx, sz.nz, sz.ny, 4.0, 2.0, amp, seed)


@pytest.mark.parametrize("case", CASES)
def test_recovery_restart_continues_run(pkg, case, tmp_path):
    V0, O0 = seeded(pkg, case)
    a = make_ctx(pkg, case)
    a.set_state(V0, O0)
    a.bootstrap()
    a.step(5)
    a.synchronize()
    path = str(tmp_path / "recover.dat")
    a.write_recovery(path)
    sz = O.Sizes(case["mx"], case["my"], case["mz"])
    # header (3 int, 2 size_t), six mean vectors, five pencil buffers
    with open(path, "rb") as f:
        dims = np.frombuffer(f.read(12), dtype=np.int32)
        psize, tsize = np.frombuffer(f.read(16), dtype=np.uint64)
    assert tuple(dims) == (case["mx"], case["my"], case["mz"])
    assert tsize % (sz.hnx * sz.ny) == 0 and tsize // (sz.hnx * sz.ny) >= sz.mz * 16
    assert psize >= (sz.mx // 2 + 1) * 16 * sz.my * sz.pz
    assert os.path.getsize(path) == 28 + 6 * sz.nz * 16 + 5 * int(tsize)

    b = make_ctx(pkg, case)
    b.read_recovery(path)
    Va, Oa = a.get_state()
    Vb, Ob = b.get_state()
    assert np.array_equal(Va, Vb) and np.array_equal(Oa, Ob)
    ha, hb = a.get_history(), b.get_history()
    assert relL2(hb[0], ha[0]) < 1e-13 and relL2(hb[1], ha[1]) < 1e-13
    a.step(5)
    b.step(5)
    a.synchronize()
    b.synchronize()
    Va, Oa = a.get_state()
    Vb, Ob = b.get_state()
    assert relL2(Vb, Va) < 1e-12 and relL2(Ob, Oa) < 1e-12
    a.close()
    b.close()


def test_recovery_rejects_other_grid(pkg, tmp_path):
    case = CASES[0]
    V0, O0 = seeded(pkg, case)
    a = make_ctx(pkg, case)
    a.set_state(V0, O0)
    a.bootstrap()
    path = str(tmp_path / "recover.dat")
    a.write_recovery(path)
    other = dict(CASES[1])
    b = make_ctx(pkg, other)
    with pytest.raises(pkg.DnsError):
        b.read_recovery(path)
    # a truncated file is an error, not a partial restore
    with open(path, "rb") as f:
        head = f.read(4096)
    short = str(tmp_path / "short.dat")
    with open(short, "wb") as f:
        f.write(head)
    with pytest.raises(pkg.DnsError):
        a.read_recovery(short)
    with pytest.raises(pkg.DnsError):
        a.read_recovery(str(tmp_path / "missing.dat"))
    a.close()
    b.close()


def read_field_file(path, sz):
    d = np.fromfile(path, dtype=np.float64)
    assert d.size == 3 * sz.pz * sz.my * sz.mx
    return d.reshape(3, sz.pz, sz.my, sz.mx)


@pytest.mark.parametrize("case", CASES)
def test_field_files_match_oracle(pkg, case, tmp_path):
    sz = O.Sizes(case["mx"], case["my"], case["mz"])
    V0, O0 = seeded(pkg, case)
    ctx = make_ctx(pkg, case)
    ctx.set_state(V0, O0)
    vel, vort = str(tmp_path / "run_velocity.0.dat"), str(tmp_path / "run_vortricity.0.dat")
    ctx.write_fields(vel, vort)
    pb = O.Problem(O.Params(case["mx"], case["my"], case["mz"], Re=case["Re"], Ro=case["Ro"],
                            dt=case["dt"]))
    pb.set_state(V0, O0)
    ref = pb.physical_fields()
    got = np.concatenate([read_field_file(vel, sz), read_field_file(vort, sz)])
    for i in range(6):
        err = np.max(np.abs(got[i] - ref[i])) / max(np.max(np.abs(ref[i])), 1e-300)
        assert err < 1e-12, (i, err)
    # the state is left as it was
    V, Om = ctx.get_state()
    assert np.array_equal(V, V0) and np.array_equal(Om, O0)
    ctx.close()


def test_field_files_mixed_precision(pkg, tmp_path):
    """The mixed-precision form keeps an FP64 state; its field files equal
    the FP64 form's on the same state."""
    case = CASES[1]
    sz = O.Sizes(case["mx"], case["my"], case["mz"])
    V0, O0 = seeded(pkg, case)
    out = []
    for prec in (None, pkg.PREC_MIXED):
        ctx = make_ctx(pkg, case, prec)
        ctx.set_state(V0, O0)
        p = str(tmp_path / f"vel{prec}.dat")
        ctx.write_fields(p, None)
        out.append(read_field_file(p, sz))
        ctx.close()
    assert np.max(np.abs(out[1] - out[0])) <= 1e-13 * np.max(np.abs(out[0]))
