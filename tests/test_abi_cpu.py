"""CPU checks of the C-ABI library: it loads without a GPU, exports every
symbol declared in include/dns_b200.h, and reports errors through status
codes (no compute calls are made here)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "dns_b200.h")).read()
    return sorted(set(re.findall(r"\b(dns_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_agree(pkg):
    assert declared_symbols() == sorted(pkg.EXPORTS)


def test_library_exports_every_symbol(pkg):
    lib = pkg.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.dns_abi_version() == 2


def test_status_strings(pkg):
    lib = pkg.load_library()
    for s in range(8):
        assert lib.dns_status_string(s)


def test_argument_errors_without_gpu(pkg):
    lib = pkg.load_library()
    assert lib.dns_create(None, None) == 1  # DNS_ERR_ARG
    p = pkg.make_params(48, 48, 126)  # mz not a multiple of 4
    h = ctypes.c_void_p()
    assert lib.dns_create(ctypes.byref(p), ctypes.byref(h)) == 1
    assert b"mz" in lib.dns_last_error()
    p = pkg.make_params(50, 48, 128)  # mx = 50 is not 2^a 3^b
    assert lib.dns_create(ctypes.byref(p), ctypes.byref(h)) == 1
    # solve-only and ensemble entries reject missing arguments before any device work
    assert lib.dns_solve_wall(None, None, None, 16, 0) == 1
    assert lib.dns_step_many(None, 0, 1) == 1
    assert b"no contexts" in lib.dns_last_error()
    assert lib.dns_check_state(None) == 1


def test_parameter_file(pkg, tmp_path):
    f = tmp_path / "parameter.txt"
    f.write_text("48 48 128\n4.0 2.0\n1300 0.1 0.005\n0 0 100 10 50\n../out/o\n../out/r\n")
    p, r = pkg.read_parameter_file(str(f))
    assert (p.mx, p.my, p.mz) == (48, 48, 128)
    assert (p.Re, p.Ro, p.dt) == (1300, 0.1, 0.005)
    assert (r.start_type, r.start_step, r.end_step, r.save_internal, r.save_recovery_internal) == (0, 0, 100, 10, 50)
    assert r.output_file_prefix == b"../out/o"
    bad = tmp_path / "short.txt"
    bad.write_text("48 48 128\n4.0 2.0\n")
    import pytest
    with pytest.raises(pkg.DnsError):
        pkg.read_parameter_file(str(bad))
    with pytest.raises(pkg.DnsError):
        pkg.read_parameter_file(str(tmp_path / "missing.txt"))
