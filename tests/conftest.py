import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")
    config.addinivalue_line("markers", "slow: long CPU run (opt-in with DG_SLOW_TESTS=1)")


@pytest.fixture(scope="session", autouse=True)
def built_library():
    """Build libdumses_gpu.so in-tree when a source is newer than it."""
    from dumses_hybrid_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, built in-tree if needed; fails loudly when absent."""
    from dumses_hybrid_b200 import build, load_library
    build.build()
    return load_library()
