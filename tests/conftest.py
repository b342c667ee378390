import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "gpu-spectral-channel-dns_b200")

if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_package():
    """Import the package directory (its name is not an identifier)."""
    if "dns_b200" in sys.modules:
        return sys.modules["dns_b200"]
    spec = importlib.util.spec_from_file_location(
        "dns_b200", os.path.join(PKG_DIR, "__init__.py"),
        submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dns_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    from oracle import rpcf_oracle
    return rpcf_oracle


# Measured parity errors, printed in the terminal summary (also with -q), so a
# run's log carries the numbers and not only pass/fail.
PARITY_LOG = []


@pytest.fixture
def parity_log():
    return PARITY_LOG


def pytest_terminal_summary(terminalreporter):
    if PARITY_LOG:
        terminalreporter.section("measured parity errors")
        for line in PARITY_LOG:
            terminalreporter.write_line(line)
