"""Shared fixtures.  `-m "not gpu"` runs everywhere; `-m gpu` needs a B200."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.join(ROOT, "tests")
PKG = os.path.join(ROOT, "on-galaxy_b200")
GOLDEN = os.path.join(TESTS, "golden")
for p in (TESTS, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle_lib import ORACLE_SO, Oracle
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "libogx_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def load(name):
        if name not in cache:
            cache[name] = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
        return cache[name]
    return load


@pytest.fixture(scope="session")
def ogx():
    import ogx as m
    m.load()
    return m
