import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine library")


@pytest.fixture(scope="session")
def golden_solve():
    return dict(np.load(GOLDEN / "solve_cases.npz"))


@pytest.fixture(scope="session")
def golden_invert():
    return dict(np.load(GOLDEN / "invert_cases.npz"))


@pytest.fixture(scope="session")
def golden_fixtures():
    return dict(np.load(GOLDEN / "reference_fixtures.npz"))


@pytest.fixture(scope="session")
def engine():
    """The engine's C ABI on a GPU; fails loudly if the library or device is missing."""
    import torch
    from python_b200 import build, engine as eng
    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    build.build_engine()
    lib = eng.load()
    assert lib.cusolver_create() == 0, eng.last_error()
    return eng
