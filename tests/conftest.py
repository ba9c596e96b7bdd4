import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long CPU/GPU case")


def _ensure_built():
    # the checker (oracle) and the library are built from the tree when absent
    if not (os.path.exists(os.path.join(ROOT, "oracle", "liboracle64.so"))
            and os.path.exists(os.path.join(ROOT, "oracle", "liboracle32.so"))):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    from kirch_datuming_b200 import build
    build.build()


_ensure_built()


@pytest.fixture(scope="session")
def golden():
    import _cases
    return _cases.Golden()
