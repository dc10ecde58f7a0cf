import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds libgba.so and the oracle once per session (incremental)."""
    from cpu_gpu_coprocess_groupby_agg_b200 import build as B
    B.build()
    import cpu_oracle as O
    O.build()
    yield


@pytest.fixture(scope="session")
def ctx():
    from cpu_gpu_coprocess_groupby_agg_b200 import Context
    c = Context(0)
    yield c
    c.close()
