"""Shared pytest configuration: the ``gpu`` marker and common fixtures."""

from __future__ import annotations

import os
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# the tests never read or write the user's autotuner cache: plans built here use the
# defaults unless a test tunes them into its own file
os.environ["GD_AUTOTUNE_CACHE"] = os.path.join(
    tempfile.mkdtemp(prefix="gd_autotune_tests_"), "autotune.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    """Golden vectors written by tests/golden/make_golden.py from the reference."""
    with np.load(os.path.join(ROOT, "tests", "golden", "golden.npz")) as data:
        return {k: data[k] for k in data.files}
