import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "tests"), os.path.join(REPO, "fmm-fft_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU case")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


# Accuracy figures that GPU tests record (rel-L2, max error per case), printed at the end of the
# run so that they show under `pytest -q` too.
_ACCURACY_LINES = []


@pytest.fixture
def accuracy_report():
    def add(line):
        _ACCURACY_LINES.append(str(line))
    return add


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    if _ACCURACY_LINES:
        terminalreporter.write_sep("-", "accuracy per case")
        for line in _ACCURACY_LINES:
            terminalreporter.write_line(line)
