import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")


def gpu_available() -> bool:
    try:
        import torch  # noqa: F401  (only to probe the device)
        return torch.cuda.is_available()
    except Exception:
        return False
