"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device (a B200) and the built library; the
rest run on any CPU host.  The CPU oracle under ``oracle/`` is the parity
checker for both.
"""

from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and the built library")
    config.addinivalue_line("markers", "slow: long-running parity sweep")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
