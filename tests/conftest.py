import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libtscgpu.so")


def pytest_collection_modifyitems(config, items):
    # gpu tests are only skipped when explicitly deselected by -m; nothing is silently emulated
    pass
