"""Shared test set-up: repo root on sys.path, the `gpu` marker, small helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built CUDA library")


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def random_field(shape, seed=0, amp=0.3, offset=1.0):
    rng = np.random.default_rng(seed)
    return offset + amp * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
