import json
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")
    config.addinivalue_line("markers", "slow: longer CPU oracle runs")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference
    if not Reference.available():
        pytest.skip("oracle/_ref not built (no reference checkout when oracle/Makefile ran)")
    return Reference()


@pytest.fixture(scope="session")
def published():
    with open(os.path.join(GOLDEN, "published.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def reference_runs():
    with open(os.path.join(GOLDEN, "reference_runs.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def ccb():
    import cuda_graph_clustering_b200 as m
    m.lib()
    return m


@pytest.fixture(scope="session")
def cuda_device():
    """A CUDA device for the gpu-marked tests (the library uses the current device, 0)."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test without a CUDA device")
    torch.cuda.init()
    return 0
