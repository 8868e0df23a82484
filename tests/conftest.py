import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a library)")


@pytest.fixture(scope="session")
def ora():
    """The CPU oracle (this repo's C restatement), built on first use."""
    import oracle
    oracle.build_oracle(ref=False)
    return oracle


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library; a GPU test fails (not skips) when it is missing."""
    import polyspectrum_b200 as ps
    ps.lib()
    return ps
