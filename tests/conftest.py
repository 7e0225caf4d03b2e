import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")
    config.addinivalue_line("markers", "slow: long CPU runs of the oracle (opt in with BOWSHOCK_SLOW=1)")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("BOWSHOCK_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow oracle run: set BOWSHOCK_SLOW=1")
    for item in items:
        if "slow" in item.keywords:
            item.add_marker(skip)
