"""Shared test set-up: marker registration and import paths.

`-m "not gpu"` runs here without a GPU (oracle vs golden vectors, host logic,
C-ABI loading and argument validation); `-m gpu` runs the parity tests on a
B200 through the C-ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "jacobi-svd-cuda_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")

# Golden cases too large to store their input: (rows, columns, SplitMix64 seed)
# of tests/golden/make_golden.py.
_SEEDED_GOLDEN_INPUTS = {
    "cfg1_512x512": (512, 512, 1),
    "g1024x256": (1024, 256, 28),
    "g2100x24_t256": (2100, 24, 23),
}


def golden_input(name, fixture):
    """Input matrix of a golden case: stored, or regenerated from its seed."""
    if "a" in fixture:
        return fixture["a"]
    import workloads

    m, n, seed = _SEEDED_GOLDEN_INPUTS[name]
    return workloads.gaussian_splitmix(m, n, seed)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    # temporary files of the tests stay inside the repository, in a folder
    # that git ignores and each session starts afresh
    if not config.option.basetemp:
        config.option.basetemp = os.path.join(ROOT, ".pytest_tmp")


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    torch.cuda.init()
    return torch.device("cuda:0")
