import json
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs through the C-ABI on cuda:0)")
    config.addinivalue_line("markers", "slow: long-running parity case")


def golden(name: str):
    return json.loads((GOLDEN / name).read_text())


@pytest.fixture(scope="session")
def lib():
    """The product library, built in-tree if needed."""
    import coding_reliability_b200 as dd
    from coding_reliability_b200.build import build
    if not dd.lib_path().exists():
        build()
    return dd.load()


@pytest.fixture(scope="session")
def ctx(lib):
    import coding_reliability_b200 as dd
    if dd.device_count() == 0:
        pytest.fail("GPU test without a CUDA device")
    c = dd.Context(0)
    yield c
    c.close()
