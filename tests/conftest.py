import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: large CPU oracle runs")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build(with_ref=oracle.have_reference_tree())
    return oracle


@pytest.fixture(scope="session")
def bt():
    import blacktracer_b200
    from blacktracer_b200 import build
    build.build()
    return blacktracer_b200


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return torch
