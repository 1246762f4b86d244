import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
for p in (REPO, REPO / "bf-new_b200", REPO / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels in libbfx.so)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds libbfx.so and the oracle if stale (no-ops when current)."""
    subprocess.run([sys.executable, str(REPO / "bf-new_b200" / "build.py")], check=True,
                   stdout=subprocess.DEVNULL)
    subprocess.run(["make", "-s", "-C", str(REPO / "oracle"), "oracle"], check=True)
    yield


@pytest.fixture(scope="session")
def gpu():
    import bfx
    if bfx.device_count() == 0:
        pytest.fail("no CUDA device visible to libbfx")
    return 0
