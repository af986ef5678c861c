"""Test configuration: the `gpu` marker, and shared helpers.

`-m "not gpu"` runs everything that needs no GPU (the oracle against the reference's known
answers, the host logic, the C-ABI exports, multi-process sharding over gloo); `-m gpu` runs
the parity tests, which call the CUDA path through the C ABI and check it against the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libclayfluid.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc

    orc.build()
    return orc


@pytest.fixture(scope="session")
def root():
    import clay_engine_b200 as ce

    r = ce.init(0)
    yield r
    r.destroy()
