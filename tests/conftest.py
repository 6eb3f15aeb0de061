"""Shared test setup.

Markers: ``gpu`` tests need a CUDA device and exercise the native library's
kernels through the C ABI; everything else runs on the CPU (oracle against
the golden fixtures, host-side plan logic, library symbol checks).
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")

# Boxcar widths of the benchmark configurations (passed explicitly).
BENCH_WIDTHS = [1, 2, 3, 4, 6, 8, 12, 16]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built native library")


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def series(n: int, seed: int, v_jitter: float = 0.25):
    rng = np.random.default_rng(seed)
    ts_e = rng.standard_normal(n).astype(np.float32)
    ts_v = (1.0 + v_jitter * rng.random(n)).astype(np.float32)
    return ts_e, ts_v


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device (no CPU fallback exists)")
    return torch
