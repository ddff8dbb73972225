import os
import sys

import pytest
import torch

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the native kernels")


def pytest_collection_modifyitems(config, items):
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        p = os.path.join(GOLDEN, name)
        if not os.path.exists(p):
            pytest.skip(f"golden fixture {name} missing (run tests/golden/make_golden.py)")
        return dict(np.load(p))

    return load


@pytest.fixture(scope="session")
def orc():
    from oracle import orc as o

    o.build()
    return o


@pytest.fixture(scope="session")
def lib():
    from atom3d_b200 import _lib, build

    build.build()
    return _lib.load()
