import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cheddar-fhe_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


# figures tests want shown in the run's summary (precision bits, rates)
REPORT = []


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_terminal_summary(terminalreporter):
    if REPORT:
        terminalreporter.write_line("figures reported by the tests:")
        for line in REPORT:
            terminalreporter.write_line("  " + line)


def param_path(name):
    return os.path.join(PKG, "params", name)


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
