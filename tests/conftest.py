import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs through the CUDA path of libltg.so)")


def pytest_collection_modifyitems(config, items):
    # GPU tests are skipped only when explicitly deselected; on a CPU-only
    # machine `-m gpu` would fail loudly, which is the intent.
    pass
