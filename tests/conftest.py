import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds the generator and the oracle (CPU) once per session."""
    from lamb_b200 import build as b
    b.build_gen()
    import oracle
    if not os.path.exists(oracle.LIB):
        oracle.build()
    yield


@pytest.fixture(scope="session")
def gpu_ctx():
    from lamb_b200 import build as b
    b.build_cuda()
    from lamb_b200.gpu import Context
    ctx = Context(0)
    yield ctx
    ctx.close()
