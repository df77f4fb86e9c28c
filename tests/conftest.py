import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

_REPORT: dict = {}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built native library")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")


def pytest_collection_modifyitems(config, items):
    import torch
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture
def report():
    """report(key, name=value, ...) records measured figures (errors, times) of a test; with OI_PARITY_REPORT
    set to a path, the session writes them there as JSON at its end."""
    def rec(key, **values):
        _REPORT.setdefault(key, {}).update({k: (float(v) if isinstance(v, (int, float)) or hasattr(v, 'item')
                                                else v) for k, v in values.items()})
    return rec


def pytest_sessionfinish(session, exitstatus):
    path = os.environ.get('OI_PARITY_REPORT')
    if path and _REPORT:
        with open(path, 'w') as fh:
            json.dump(_REPORT, fh, indent=1, sort_keys=True)
