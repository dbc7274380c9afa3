import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def orc():
    """The CPU oracle (test infrastructure)."""
    import oracle
    return oracle.lib()


@pytest.fixture(scope="session")
def opsb_lib():
    """The OPS-B200 shared library, built in-tree if needed."""
    from ops_b200 import build as _build  # noqa: F401
    import ops_b200.build as b
    b.build()
    import ops_b200
    return ops_b200.lib()


@pytest.fixture(scope="session")
def gpu_runtime(opsb_lib):
    from ops_b200 import ops
    ops.ops_init(0, 0)
    yield opsb_lib
