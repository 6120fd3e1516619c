import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libgpe_b200.so")
    config.addinivalue_line("markers", "slow: longer CPU-oracle comparisons")


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    """Make sure the oracle libraries exist (build them from source if needed)."""
    from oracle import oracle as O

    if not os.path.exists(O.ORACLE_SO):
        O.build(ref=True)
    yield
