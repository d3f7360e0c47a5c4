import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def record_error(name: str, value: float) -> None:
    """Appends a measured parity error to $CTLAB_PARITY_LOG (JSON lines)."""
    path = os.environ.get("CTLAB_PARITY_LOG")
    if path:
        import json
        with open(path, "a") as f:
            f.write(json.dumps({"case": name, "rel_l2": value}) + "\n")
