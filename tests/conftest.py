"""Shared test set-up: the `gpu` marker, import paths and the oracle build."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import vt_oracle
    vt_oracle.load()
    return vt_oracle


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from metal_vibe_tracer_b200 import Context
    c = Context(0)
    yield c
    c.close()
