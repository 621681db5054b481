import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hvm-64_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long CPU runs (set HVM64_SLOW=1)")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("HVM64_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow; set HVM64_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)
