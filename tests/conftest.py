"""Test configuration.

Markers: ``gpu`` — needs a CUDA device (run with ``-m gpu`` on a B200).  Every
other test runs on CPU.  The oracle (``oracle/``) is the checker only.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O
    O.lib()  # builds _build/liboracle.so when missing
    return O


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
