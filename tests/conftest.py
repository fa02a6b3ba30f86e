import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name))


def unpack_list(flat, offsets, dtype):
    arr = np.ascontiguousarray(flat).view(dtype).reshape(-1)
    return [arr[offsets[i]:offsets[i + 1]] for i in range(len(offsets) - 1)]


def as_records(raw, dtype):
    return np.ascontiguousarray(raw).view(dtype).reshape(-1)


@pytest.fixture(scope="session")
def gpu_lib():
    import dials_metal_spotfinder_b200 as sf
    if not sf.available():
        pytest.fail("no CUDA device: the gpu tests must run on the B200 box")
    return sf
