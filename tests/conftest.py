import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _ensure_built():
    lib = os.path.join(ROOT, "cdocker_b200", "libcdock_b200.so")
    if not os.path.exists(lib):
        from cdocker_b200 import build
        build.build()
    orc = os.path.join(ROOT, "oracle", "libcdk_oracle.so")
    if not os.path.exists(orc):
        from oracle import oracle
        oracle.build()


_ensure_built()


@pytest.fixture(scope="session")
def has_gpu():
    import torch
    return torch.cuda.is_available()


@pytest.fixture(scope="session")
def grids_cache():
    return {}


@pytest.fixture(scope="session")
def c0(grids_cache):
    from cdocker_b200 import synth
    return synth.make_workload("c0_32", seed=0, grids_cache=grids_cache)
