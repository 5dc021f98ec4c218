"""Shared test setup: import paths, the `gpu` marker and common fixtures.

CPU tests (`-m "not gpu"`) check the oracle against the reference's golden
vectors, the host-side logic, and that libcpx.so loads and exports every
symbol of include/cpx.h.  GPU tests (`-m gpu`) are the parity tests proper:
they call the CUDA path through the C ABI and compare it with the oracle and,
where oracle/_ref/libcpxref.so is present, with the reference's own kernels.
"""
import pathlib
import sys

import pytest

REPO = pathlib.Path(__file__).resolve().parents[1]
for sub in ("", "clear-plenoxels_b200", "oracle", "tests/golden"):
    p = str(REPO / sub)
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
