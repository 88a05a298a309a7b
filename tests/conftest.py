"""Shared test configuration.

``gpu`` marks tests that need a CUDA device and the built engine library; the
CPU suite runs with ``-m "not gpu"``.
"""

from __future__ import annotations

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and libbls_b200.so")
