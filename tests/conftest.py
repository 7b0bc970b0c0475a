import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)

N26 = os.path.join(TESTS, "golden", "n26")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def q():
    build = importlib.import_module("2degas_b200.build")
    build.build()
    return importlib.import_module("2degas_b200")


@pytest.fixture(scope="session")
def n26_dir():
    return N26


@pytest.fixture
def n26(q):
    return q.System.read(N26, "n26")


@pytest.fixture
def n26_configs(n26):
    return n26.read_configs(N26, ".0", 0, 64)


@pytest.fixture(scope="session")
def oracle_cls():
    from oracle_lib import Oracle, build

    build()
    return Oracle


@pytest.fixture(scope="session")
def has_gpu():
    import torch

    return torch.cuda.is_available()
