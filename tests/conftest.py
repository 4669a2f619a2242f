"""Test configuration.

Mirrors the reference harness (tests/conftest.py:5-49 of Crinton/FastCTQW): the
``--matrix-sizes`` and ``--dtype`` options parametrise any test that takes ``N`` /
``dtype``.  Tests that need a B200 carry ``@pytest.mark.gpu``; everything else runs on CPU.
"""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_addoption(parser):
    parser.addoption("--matrix-sizes", action="store", default="1,2,3,16,33,64,128,257",
                     type=str, help="comma-separated matrix sizes, e.g. --matrix-sizes=500,1000")
    parser.addoption("--dtype", action="store", default="complex64", type=str,
                     help="complex64 or complex128")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_generate_tests(metafunc):
    dtype_map = {"complex64": np.complex64, "complex128": np.complex128}
    if "N" in metafunc.fixturenames:
        sizes = [int(s) for s in metafunc.config.getoption("--matrix-sizes").split(",") if s.strip()]
        metafunc.parametrize("N", sizes)
    if "dtype" in metafunc.fixturenames:
        d = metafunc.config.getoption("--dtype")
        if d in dtype_map:
            metafunc.parametrize("dtype", [dtype_map[d]])


GOLDEN = os.path.join(REPO, "tests", "golden", "golden_cases.npz")


def load_golden():
    """{case_name: {key: array}} from the committed fixture file."""
    z = np.load(GOLDEN)
    out = {}
    for k in z.files:
        name, key = k.split("::")
        out.setdefault(name, {})[key] = z[k]
    return out


@pytest.fixture(scope="session")
def golden():
    return load_golden()
