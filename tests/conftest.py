import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (str(ROOT), str(ROOT / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib
    oracle_lib.build_oracle()
    return oracle_lib.lib()


@pytest.fixture(scope="session")
def engine_lib():
    from gemray_studio_b200 import build
    build.build()
    from gemray_studio_b200 import abi
    return abi.load_library()


@pytest.fixture(scope="session")
def renderer(engine_lib):
    from gemray_studio_b200 import GpuFrameRenderer
    r = GpuFrameRenderer()
    yield r
    r.close()
