"""Shared test setup: paths, the `gpu` marker, and the in-tree builds the tests load."""
import os
import subprocess
import sys

import pytest

RAIZ = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PACOTE = os.path.join(RAIZ, "tanque-de-agua_b200")
for p in (PACOTE, os.path.join(RAIZ, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    # The oracle (test infrastructure) is a few seconds of g++; build it when missing.
    so = os.path.join(RAIZ, "oracle", "liboracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(RAIZ, "oracle")], check=True, capture_output=True)


@pytest.fixture(scope="session")
def oraculo():
    from oraculo import carregar_oraculo
    return carregar_oraculo()


@pytest.fixture(scope="session")
def lib_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tanque import _abi
    return _abi.carregar()
