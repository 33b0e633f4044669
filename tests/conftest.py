import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
# shared test protocols (fractal_case.py) import by name
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the B200 library)")
    # the checker and the library are built in-tree before any test imports them
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


@pytest.fixture(scope="session")
def gpu_lib():
    from partmc_b200 import build
    build.build()
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from partmc_b200 import _lib
    return _lib.lib()
