import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def relerr(x, ref, floor_frac=1e-12):
    """Per-bin relative error |x - ref| / max(|ref|, floor_frac * max_bins |ref|).
    floor_frac = 1e-12 only keeps exactly-zero bins finite; the FP32 checks use 1e-3, i.e.
    error relative to the statistic's own scale where shot-noise subtraction leaves a bin
    near zero."""
    x = np.asarray(x)
    ref = np.asarray(ref)
    floor = floor_frac * float(np.max(np.abs(ref)))
    return float(np.max(np.abs(x - ref) / np.maximum(np.abs(ref), floor)))


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name))


def binning_from(arr):
    from hitomi_b200.api import Binning
    return Binning(float(arr[0]), float(arr[1]), int(arr[2]), float(arr[3]), float(arr[4]), int(arr[5]))


@pytest.fixture
def golden():
    return load_golden
