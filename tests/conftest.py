import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def reflib():
    from oracle.oracle import RefLib, have_ref
    if not have_ref():
        pytest.fail("oracle/_ref reference build missing (run make -C oracle)")
    return RefLib()


@pytest.fixture(scope="session")
def restate():
    from oracle.oracle import Restate, have_restate
    if not have_restate():
        pytest.fail("oracle/_ref/librestate.so missing (run make -C oracle restate)")
    return Restate()


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    from mkfit_b200 import Context
    ctx = Context(0)
    yield ctx
    ctx.close()
