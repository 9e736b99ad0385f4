import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and librzk_cuda.so")


@pytest.fixture(scope="session")
def oracle_built():
    """Compile the CPU checkers (liboracle.so; the reference harness where the reference
    tree exists)."""
    import oracle
    oracle.build(ref=True)
    return True


@pytest.fixture(scope="session")
def gpu_lib():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test on a machine without a CUDA device")
    from renzoku_b200 import build as rbuild, rzk
    rbuild.build()
    return rzk.load()


@pytest.fixture(scope="session")
def ctx(gpu_lib):
    from renzoku_b200 import rzk
    c = rzk.Context(0)
    yield c
    c.close()
