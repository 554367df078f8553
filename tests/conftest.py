import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    # the C oracle is test infrastructure; (re)build it when its sources are
    # newer than this checkout's library
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "all"],
                   check=True, capture_output=True)


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.oracle_toolbox()


@pytest.fixture(scope="session")
def gpu_tb():
    from lsmlib_b200 import gpu
    return gpu.toolbox()
