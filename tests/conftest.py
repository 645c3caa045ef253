import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def reference_root():
    """The reference source tree: $REF_ROOT, else the default that the oracle
    build recipe (oracle/Makefile, `REF_ROOT ?= ...`) compiles from."""
    if os.environ.get("REF_ROOT"):
        return os.environ["REF_ROOT"]
    with open(os.path.join(ROOT, "oracle", "Makefile")) as f:
        for line in f:
            if line.startswith("REF_ROOT") and "?=" in line:
                return line.split("?=", 1)[1].strip()
    return ""


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libfmmb.so")


@pytest.fixture(scope="session")
def oracle():
    """The CPU checker (restatement + reference build), compiled on demand."""
    from oracle import pyoracle
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        pyoracle.build()
    return pyoracle
