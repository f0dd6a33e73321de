"""Shared test set-up: the `gpu` marker, import paths and the oracle build."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# CPU tests that check the table generators against the reference's data read it from the checkout
# the build recipe uses (VT_REFERENCE_ROOT); where it is absent they skip.
from __graft_entry__ import REFERENCE_DEFAULT  # noqa: E402

os.environ.setdefault("VT_REFERENCE_ROOT", REFERENCE_DEFAULT)


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
