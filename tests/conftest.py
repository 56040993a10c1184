"""Shared pytest setup: import paths and the ``gpu`` marker.

Tests marked ``gpu`` need a CUDA device and the built extension; the rest run
on the CPU (oracle, host logic, ABI exports, multi-process gloo paths).
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "voxel-sim_b200"
for p in (ROOT, PKG, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libvxcorot.so")
    config.addinivalue_line("markers", "slow: longer CPU test")


def pytest_collection_modifyitems(config, items):
    # keep the no-allocation entry-point test file last so a -x run has already
    # run every other test when it starts
    items.sort(key=lambda it: ("test_zz_" in it.nodeid, 0))
