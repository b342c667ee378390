"""The reference program itself (its cuFFT GPU half and OpenMP CPU half, built
from its own sources by oracle/ref_build/build_ref_program.py; only the Eigen
routines of source/matrix_op.cpp replaced by an own LU) against the library
and the oracle: a whole-step pin of the reference, its GPU transforms
included.

The reference's own limits hold: plane Couette base flow U = (1 + y)/2 and
Ny <= MAX_NZ = 100.  Same parameter.txt for the reference program and for the
library's driver dns_run (48 x 48 x 128: 32 x 33 x 32 modes, Re 1300, Ro 0.1,
dt 0.005, the analytic initFlow start, 12 steps after the bootstrap); both
write the reference's recovery file, which holds the state and the AB2
history.  Compared: the reference program against the oracle (the same
algorithm in FP64 NumPy, explicit inverses), and against the library.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import rpcf_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "ref_program")
DNS_RUN = os.path.join(ROOT, "gpu-spectral-channel-dns_b200", "dns_run")

pytestmark = pytest.mark.gpu

PARAMS = "48 48 128\n4.0 2.0\n1300 0.1 0.005\n0 0 10 100 10\nout/o\nout/r\n"


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _read(pkg, path):
    ctx = pkg.Context(pkg.make_params(48, 48, 128, Re=1300.0, Ro=0.1, dt=0.005))
    ctx.read_recovery(str(path))
    V, Om = ctx.get_state()
    Nv, No = ctx.get_history()
    ctx.close()
    return V, Om, Nv, No


def test_reference_program_matches_oracle_and_library(pkg, tmp_path, parity_log):
    if not os.path.exists(REF_EXE):
        pytest.skip("oracle/_ref/ref_program not built (needs the reference's sources)")
    (tmp_path / "input").mkdir()
    (tmp_path / "input" / "parameter.txt").write_text(PARAMS)
    runs = {}
    for name, exe in (("reference", REF_EXE), ("library", DNS_RUN)):
        d = tmp_path / name
        (d / "out").mkdir(parents=True)
        r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=600)
        ok = r.returncode == 0
        if name == "reference" and not ok:
            # the reference never joins its worker thread (std::thread
            # sub_thread, source/rhs.cpp:22): the thread's destructor calls
            # std::terminate at exit, after every step and file is done
            ok = (r.returncode == -6 and r.stderr.strip() == "terminate called without an active exception"
                  and "WRINTING RECOVERY FILES" in r.stdout)
        assert ok, (name, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
        assert r.stdout.count("STEP:") == 11, name
        if name == "reference":
            ms = [float(x.split(":")[1]) for x in r.stdout.splitlines() if x.startswith("Time cost of current step:")]
            parity_log.append(f"reference program step time at 48x48x128 (cuFFT + OpenMP solves), "
                              f"median of {len(ms)}: {1e3 * sorted(ms)[len(ms) // 2]:.3f} ms")
        runs[name] = d
    ref = _read(pkg, runs["reference"] / "recovery.dat")
    lib = _read(pkg, runs["library"] / "recovery.dat")
    # the oracle: initFlow's state, bootstrap, 12 steps
    p = O.Params(48, 48, 128, Re=1300.0, Ro=0.1, dt=0.005)
    pb = O.Problem(p)
    V0, O0 = O.init_state(pb.sz, pb.aphi, pb.beta)
    pb.set_state(V0, O0)
    pb.bootstrap()
    for _ in range(12):
        pb.step()
    e_ro = [_rel(ref[0], pb.V), _rel(ref[1], pb.O)]
    e_rl = [_rel(lib[i], ref[i]) for i in range(4)]
    parity_log.append("reference program (cuFFT + CPU solves), 12 steps at 48x48x128: vs oracle v %.1e omega %.1e; "
                      "library vs reference program v %.1e omega %.1e Nv %.1e Nomega %.1e" % (*e_ro, *e_rl))
    assert max(e_ro) < 1e-12, e_ro
    assert max(e_rl) < 1e-11, e_rl


def _run_prog(exe, root, params, recovery=None):
    """Run a reference-layout program (reference or dns_run) in root/run with
    root/input/parameter.txt; optionally start from a copy of `recovery`."""
    import shutil
    (root / "input").mkdir(parents=True, exist_ok=True)
    (root / "input" / "parameter.txt").write_text(params)
    d = root / "run"
    (d / "out").mkdir(parents=True, exist_ok=True)
    if recovery is not None:
        shutil.copy(recovery, d / "recovery.dat")
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=600)
    ok = r.returncode == 0 or (exe == REF_EXE and r.returncode == -6 and
                               r.stderr.strip() == "terminate called without an active exception")
    assert ok, (exe, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return d / "recovery.dat"


def test_reference_program_restarts_from_library_recovery(pkg, tmp_path, parity_log):
    """Byte compatibility of the recovery file in the library -> reference
    direction: the library's driver runs 10 steps and writes recovery.dat;
    the reference program restarts from that file (start_type 1, its own
    read_recover_data) and runs to step 15, as does the library's driver; the
    two files at step 15 (state and AB2 history) agree to the level of the
    two programs' rounding.  (The other direction, the library reading the
    reference program's file, is the test above.)"""
    if not os.path.exists(REF_EXE):
        pytest.skip("oracle/_ref/ref_program not built (needs the reference's sources)")
    base = "48 48 128\n4.0 2.0\n1300 0.1 0.005\n"
    rec10 = _run_prog(DNS_RUN, tmp_path / "lib10", base + "0 0 10 100 10\nout/o\nout/r\n")
    restart = base + "1 10 15 100 5\nout/o\nout/r\n"
    rec_ref = _run_prog(REF_EXE, tmp_path / "ref15", restart, rec10)
    rec_lib = _run_prog(DNS_RUN, tmp_path / "lib15", restart, rec10)
    ref = _read(pkg, rec_ref)
    lib = _read(pkg, rec_lib)
    e = [_rel(lib[i], ref[i]) for i in range(4)]
    parity_log.append("reference program restarted from the library's recovery file, steps 10..15 at "
                      "48x48x128, vs the library's own restart: v %.1e omega %.1e Nv %.1e Nomega %.1e" % tuple(e))
    assert max(e) < 1e-11, e
