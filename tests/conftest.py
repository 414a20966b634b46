"""Shared test setup.

* `-m "not gpu"` tests check the oracle (the CPU restatement of the
  reference) against the reference's own known-answer tests, the host-side
  logic, and that libvp8a.so loads and exports every ABI symbol.
* `-m gpu` tests are the parity tests proper: the CUDA path, called through
  the C ABI, must reproduce the oracle bit-exactly.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oxideav-vp8_b200"), os.path.join(ROOT, "oracle"), os.path.dirname(__file__)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    import oracle as o

    o.build()
    o.load()
    return o


@pytest.fixture(scope="session")
def ctx():
    import vp8a

    c = vp8a.Context(0)
    yield c
    c.close()
