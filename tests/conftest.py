import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and calls the C ABI on it")


@pytest.fixture(scope="session", autouse=True)
def _built():
    import ybus_b200.build as b
    b.build()
    import oracle.oracle as o
    o.build()


@pytest.fixture(scope="session")
def gpu():
    from ybus_b200 import Gpu
    g = Gpu.new()
    if g is None:
        if os.environ.get("YBUS_REQUIRE_CUDA") == "1":
            pytest.fail("no CUDA device, and YBUS_REQUIRE_CUDA=1")
        pytest.skip("no CUDA device")
    return g
