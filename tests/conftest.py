"""Test configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs on any machine: the oracle against the golden vectors of
the reference's own kernel, host logic, and the C ABI's exports.  `-m gpu`
runs the CUDA library on a B200 against the oracle.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the built CUDA library")


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(ROOT, "tests", "golden", "optkmatch_cases.npz")
    z = np.load(path)
    out = {}
    for n in z["names"]:
        n = str(n)
        out[n] = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(n + "/")}
    return out


@pytest.fixture(scope="session")
def ctx():
    from mirorr_b200 import build as mb_build
    mb_build.build()
    import mirorr_b200 as mb
    c = mb.Context(0)
    yield c
    c.close()
