"""Shared test setup: markers, library builds, oracle handles."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def ob():
    from octlb_b200 import build
    build.build()
    import octlb_b200
    return octlb_b200


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    if not os.path.exists(oracle.ORC_PATH):
        oracle.build(ref=False)
    return oracle.load("orc")


@pytest.fixture(scope="session")
def ref():
    from oracle import oracle
    L = oracle.load("ref")
    if L is None:
        pytest.skip("reference oracle (oracle/_ref) not built")
    return L


@pytest.fixture(scope="session")
def tlm():
    from oracle import oracle
    L = oracle.load("tlm")
    if L is None:
        pytest.skip("tangent-linear reference (oracle/_ref/liboctlb_ref_tlm.so) not built")
    return L
