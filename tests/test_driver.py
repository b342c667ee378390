"""The parameter.txt driver (dns_run, the reference's run_simulation).

CPU: usage, a missing or malformed parameter file and a wrong start type are
errors with a message, before any device work.  GPU: a fresh start (initial
fields, three output steps, a recovery file) and a restart from that file
run to completion and write files of the reference's sizes.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "gpu-spectral-channel-dns_b200", "dns_run")


@pytest.fixture(scope="module")
def exe():
    if not os.path.exists(EXE):
        import importlib.util
        spec = importlib.util.spec_from_file_location(
            "dns_build", os.path.join(ROOT, "gpu-spectral-channel-dns_b200", "build.py"))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        m.build()
    return EXE


def _run(exe, args, cwd, timeout=600):
    return subprocess.run([exe, *args], cwd=cwd, capture_output=True, text=True, timeout=timeout)


def _gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


def test_usage_and_parameter_errors(exe, tmp_path):
    r = _run(exe, ["--help"], tmp_path)
    assert r.returncode == 0 and "usage" in r.stdout
    r = _run(exe, [str(tmp_path / "missing.txt")], tmp_path)
    assert r.returncode == 2 and "parameter file" in r.stderr
    bad = tmp_path / "short.txt"
    bad.write_text("48 48 128\n4.0 2.0\n")
    r = _run(exe, [str(bad)], tmp_path)
    assert r.returncode == 2 and "parameter file" in r.stderr
    r = _run(exe, ["--bogus"], tmp_path)
    assert r.returncode == 1


def test_without_a_device_the_context_fails_cleanly(exe, tmp_path):
    if _gpu():
        pytest.skip("a CUDA device is present")
    f = tmp_path / "parameter.txt"
    f.write_text("48 48 128\n4.0 2.0\n1300 0.1 0.005\n0 0 4 2 4\nout/o\nout/r\n")
    r = _run(exe, [str(f)], tmp_path)
    assert r.returncode == 2 and "create" in r.stderr


@pytest.mark.gpu
def test_fresh_start_and_restart(exe, tmp_path):
    if not _gpu():
        pytest.skip("no CUDA device")
    (tmp_path / "out").mkdir()
    f = tmp_path / "parameter.txt"
    f.write_text("48 48 128\n4.0 2.0\n1300 0.1 0.005\n0 0 4 2 4\nout/o\nout/r\n")
    r = _run(exe, [str(f)], tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.count("STEP:") == 5
    size = 3 * (128 // 2 + 1) * 48 * 48 * 8  # three components of pz x my x mx doubles
    for step in (0, 2, 4):
        for kind in ("velocity", "vortricity"):
            path = tmp_path / "out" / f"o_{kind}.{step}.dat"
            assert path.stat().st_size == size
            assert np.all(np.isfinite(np.fromfile(path, dtype=np.float64)))
    assert (tmp_path / "recovery.dat").exists()
    # restart from the recovery file written at step 4
    g = tmp_path / "restart.txt"
    g.write_text("48 48 128\n4.0 2.0\n1300 0.1 0.005\n1 5 6 2 100\nout/p\nout/r\n")
    r = _run(exe, [str(g)], tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    assert (tmp_path / "out" / "p_velocity.6.dat").stat().st_size == size
