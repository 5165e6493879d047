"""Shared test setup: paths, the `gpu` marker, and in-tree builds."""
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "plp-gpu_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
# the reference tree, only present where it is mounted
REFERENCE = os.environ.get("PLP_REFERENCE", "/root/reference")
for p in (PKG, os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (parity tests of the CUDA path)")


def _make(path):
    subprocess.run(["make", "-s", "-C", path], check=True)


@pytest.fixture(scope="session", autouse=True)
def built():
    _make(os.path.join(REPO, "oracle"))
    _make(PKG)


def has_reference():
    return os.path.isdir(os.path.join(REFERENCE, "gpu"))
