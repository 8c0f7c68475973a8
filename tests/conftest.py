import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")
    config.addinivalue_line("markers", "slow: longer-running case, skipped unless --runslow or MPDX_RUNSLOW=1")


def pytest_addoption(parser):
    parser.addoption("--runslow", action="store_true", default=False, help="also run tests marked slow")


def pytest_collection_modifyitems(config, items):
    if config.getoption("--runslow") or os.environ.get("MPDX_RUNSLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow: pass --runslow (or MPDX_RUNSLOW=1) to run")
    for item in items:
        if "slow" in item.keywords:
            item.add_marker(skip)
