import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C-ABI")


def _ensure_built():
    """Build the oracle and the libraries if a fresh checkout lacks them (make is
    incremental; nothing is rebuilt when the files are current)."""
    if not os.path.exists(os.path.join(REPO, "oracle", "_build", "libsph_oracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "all"], check=True)
    lib = os.path.join(REPO, "cosmosphere_b200", "lib")
    need = ["libcosmoSPHere.so", "libcosmoSPHere_quintic.so", "libcosmo_inputs.so"]
    if not all(os.path.exists(os.path.join(lib, f)) for f in need):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(REPO, "cosmosphere_b200"), "all"], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def repo():
    return REPO
