import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "drape-2_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) and runs the CUDA library")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    if not os.path.exists(oracle.LIB):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def ref_available(oracle_mod):
    return oracle_mod.ref_available()


@pytest.fixture(scope="session")
def cuda_mod():
    from drape_b200 import cuda
    cuda.load()
    return cuda


@pytest.fixture(scope="session")
def gpu(cuda_mod):
    """The CUDA module, after checking that a usable device is present (fails loudly otherwise)."""
    if not cuda_mod.is_available():
        pytest.fail("no usable sm_100 CUDA device for a gpu-marked test")
    return cuda_mod
