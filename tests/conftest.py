"""Shared fixtures.  GPU tests are marked ``gpu`` and run only on a B200 box
(``pytest -m gpu``); everything else runs on CPU."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"
if str(GOLDEN) not in sys.path:
    sys.path.insert(0, str(GOLDEN))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, failing loudly when it is missing on a GPU box."""
    import torch  # noqa: F401  (initialises the CUDA driver like a user process would)
    from implexity_b200 import _abi

    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    return _abi.load()
