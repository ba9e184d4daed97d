"""Shared fixtures.  GPU tests carry @pytest.mark.gpu and run on a B200; everything else
runs on the CPU (the solver library is only loaded, never stepped, without a GPU)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def solver_lib():
    from cmakepro_cuda_seissim_v2_b200 import build, capi

    build.build()
    return capi.load()


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return 0


@pytest.fixture(scope="session")
def solver2d_lib():
    from cmakepro_cuda_seissim_v2_b200 import build, capi2d

    build.build()
    return capi2d.load()
