"""The reference's unchanged driver (source/main_loop.cpp, run_simulation)
running on the library through the shim, against the library's own driver.

Three runs of the same parameter.txt (48x48x128, Re 1300, Ro 0.1, dt 0.005,
fresh start, 6 steps, fields and recovery every 3 steps), each in its own
directory:
  ref_main      the reference's driver, fused nextStep;
  ref_main_fbf  the reference's driver, nextStep as the reference's own
                sequence through the per-function drop-ins (explicit
                inverses on the host, as the reference multiplies);
  dns_run       the library's driver over the C ABI.
ref_main must reproduce dns_run bit for bit (recovery file and field files):
the shim's "extra previous step" and second initFlow reach the same state and
AB2 history as dns_run's bootstrap.  ref_main_fbf agrees with them to the
rounding of its different solve (explicit inverses against the banded
factors).  A restart from the recovery file (start_type 1) runs three more
steps under both drivers, again bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-spectral-channel-dns_b200")
EXES = {"ref_main": os.path.join(PKG, "shim", "ref_main"),
        "ref_main_fbf": os.path.join(PKG, "shim", "ref_main_fbf"),
        "dns_run": os.path.join(PKG, "dns_run")}

pytestmark = pytest.mark.gpu

PARAMS = "48 48 128\n4.0 2.0\n1300 0.1 0.005\n{st} {s0} {s1} 3 3\nout/o\nout/r\n"


def _state(pkg, path):
    ctx = pkg.Context(pkg.make_params(48, 48, 128, Re=1300.0, Ro=0.1, dt=0.005))
    ctx.read_recovery(str(path))
    V, O = ctx.get_state()
    Nv, No = ctx.get_history()
    ctx.close()
    return V, O, Nv, No


def _run(name, cwd):
    r = subprocess.run([EXES[name]], cwd=cwd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (name, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_reference_driver_on_the_library(pkg, tmp_path, parity_log):
    missing = [n for n, e in EXES.items() if not os.path.exists(e)]
    if missing:
        pytest.skip(f"not built: {missing} (the shim executables need the reference's sources)")
    (tmp_path / "input").mkdir()
    (tmp_path / "input" / "parameter.txt").write_text(PARAMS.format(st=0, s0=0, s1=6))
    runs = {}
    for name in EXES:
        d = tmp_path / name
        (d / "out").mkdir(parents=True)
        out = _run(name, d)
        assert out.count("STEP:") == 7, name
        runs[name] = d
    a = open(runs["ref_main"] / "recovery.dat", "rb").read()
    b = open(runs["dns_run"] / "recovery.dat", "rb").read()
    assert a == b, "fused shim and dns_run recovery files differ"
    for step in (0, 3, 6):
        for kind in ("velocity", "vortricity"):
            f = f"o_{kind}.{step}.dat"
            assert (open(runs["ref_main"] / "out" / f, "rb").read() ==
                    open(runs["dns_run"] / "out" / f, "rb").read()), f
    sf = _state(pkg, runs["ref_main_fbf"] / "recovery.dat")
    sn = _state(pkg, runs["dns_run"] / "recovery.dat")
    errs = [_rel(x, y) for x, y in zip(sf, sn)]
    parity_log.append("reference driver, function by function vs fused, after 6 steps: "
                      "v %.1e omega %.1e Nv %.1e Nomega %.1e" % tuple(errs))
    assert max(errs) < 1e-11, errs
    # restart: steps 7..9 from the step-6 recovery file
    (tmp_path / "input" / "parameter.txt").write_text(PARAMS.format(st=1, s0=7, s1=9))
    for name in ("ref_main", "dns_run"):
        out = _run(name, runs[name])
        assert out.count("STEP:") == 3, name
    assert (open(runs["ref_main"] / "recovery.dat", "rb").read() ==
            open(runs["dns_run"] / "recovery.dat", "rb").read())
