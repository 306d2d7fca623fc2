"""pytest set-up: import paths and the `gpu` marker.

`-m "not gpu"` runs on any host (oracle known answers, golden fixtures,
C-ABI loading and host-side checks, gloo multi-process tests); `-m gpu`
runs the parity tests on a B200 through the C-ABI of libminecu_b200.so.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("mine.cu_b200", "oracle", "tests"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on a B200)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a host without CUDA")
    return torch.device("cuda", 0)
