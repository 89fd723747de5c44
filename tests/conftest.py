"""Shared pytest configuration: the ``gpu`` marker and common fixtures."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden" / "jht_golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def relerr(a, b) -> float:
    """max|a - b| / max|b| -- the reference's comparison convention (test_healpix.py:84-86)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def parse_tag(tag: str):
    """'s2_n16_l24' -> (spin, nside, lmax)."""
    parts = tag.split("_")
    return int(parts[0][1:]), int(parts[1][1:]), int(parts[2][1:])


TRANSFORM_TAGS = [
    "s0_n1_l3", "s0_n4_l16", "s0_n8_l12", "s0_n16_l24", "s0_n64_l128", "s0_n12_l20",
    "s2_n2_l5", "s2_n4_l16", "s2_n8_l12", "s2_n16_l24", "s2_n32_l64", "s2_n12_l20",
]
