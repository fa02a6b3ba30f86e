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


def same_spots(got, want):
    """Spot rows equal field by field, bit for bit. The 4 padding bytes of a
    Spot carry no value (the reference leaves them indeterminate), so rows
    are not compared as raw bytes."""
    assert len(got) == len(want), (len(got), len(want))
    for name in want.dtype.names:
        a, b = np.ascontiguousarray(got[name]), np.ascontiguousarray(want[name])
        if a.tobytes() != b.tobytes():
            k = int(np.nonzero((a.view(np.uint8).reshape(len(a), -1) !=
                                b.view(np.uint8).reshape(len(b), -1)).any(1))[0][0])
            raise AssertionError(f"spot {k} field {name}: {got[k]} vs {want[k]}")


@pytest.fixture(scope="session")
def gpu_lib():
    import dials_metal_spotfinder_b200 as sf
    if not sf.available():
        pytest.fail("no CUDA device: the gpu tests must run on the B200 box")
    return sf
