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


class Kernel(int):
    """A dd.KERNEL_* value that also names the tcgen05 epilogue it runs with."""
    epilogue = 0
    label = ""


def kernel_variant(name: str) -> Kernel:
    import coding_reliability_b200 as dd
    k = Kernel(dd.KERNEL_POPC if name == "popc" else dd.KERNEL_MMA)
    k.epilogue = {"popc": 0, "mma_paired": dd.MMA_EPILOGUE_PAIRED, "mma_single": dd.MMA_EPILOGUE_SINGLE}[name]
    k.label = name
    return k


@pytest.fixture(params=["popc", "mma_paired", "mma_single"])
def kernel(request, ctx):
    """Every histogram kernel variant, named explicitly: the popc kernel and the
    tcgen05 kernel with each of its two epilogues.  A parity test never depends
    on which variant the context's autotuner would pick for KERNEL_AUTO."""
    import coding_reliability_b200 as dd
    k = kernel_variant(request.param)
    ctx.set_mma_epilogue(k.epilogue if k.epilogue else dd.MMA_EPILOGUE_AUTO)
    yield k
    ctx.set_mma_epilogue(dd.MMA_EPILOGUE_AUTO)
