import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and libknng.so")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import bindings

    bindings.build(with_reference=os.path.isdir(bindings.REFERENCE_SRC))
    return bindings


@pytest.fixture(scope="session")
def golden():
    import json

    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def knng_lib():
    """libknng.so, built if needed (nvcc cross-compiles without a GPU)."""
    from sigmod23ann_b200 import build, load_library

    build.build()
    return load_library()
