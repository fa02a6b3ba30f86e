"""sf_find_u16_noalloc, the threshold entry point for callers that may not
allocate device memory (plugins inside a host that owns the GPU's memory,
real-time loops that cannot afford cudaMalloc / cudaFree stalls), against
sf_find_u16 through the C ABI: the same signal pixels, byte for byte, on
consecutive calls of different shapes -- every call reuses the one static
scratch array, so a call that failed to clear what the previous one left
there would show up here. Collected last on purpose (the file name), and
written to pass alone in a fresh process as well as after the other tests."""

import ctypes

import numpy as np
import pytest

from conftest import as_records, load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def noalloc_status(lib, img):
    img = np.ascontiguousarray(img, dtype=np.uint16)
    h, w = img.shape
    cap = max(h * w * 2 // 16, 1)
    out = np.zeros(cap, O.SIGNAL_PIXEL)
    found = ctypes.c_size_t(0)
    status = lib.sf_find_u16_noalloc(img.ctypes.data, h, w, out.ctypes.data, cap,
                                     ctypes.byref(found), None)
    return status, out[: found.value].copy() if status == 0 else out[:0]


def test_matches_sf_find_on_consecutive_calls(gpu_lib):
    from dials_metal_spotfinder_b200 import synth
    from dials_metal_spotfinder_b200._lib import lib

    series = synth.eiger_4m(frames=2)
    small = load_golden("small_series.npz")["frames"]
    # 4M, then a small frame, then another 4M frame: each call's layout
    # overlaps what the one before left in the scratch
    frames = [series.frame(0), small[3], series.frame(1)]
    for k, img in enumerate(frames):
        want_status, want = gpu_lib.find_status(img)
        status, got = noalloc_status(lib, img)
        assert status == want_status == 0, f"call {k}: {status} vs {want_status}"
        assert len(got) == len(want) > 0, f"call {k}: {len(got)} vs {len(want)}"
        assert got.tobytes() == want.tobytes(), f"call {k}: signal pixels differ"


def test_reference_frame_set(gpu_lib):
    from dials_metal_spotfinder_b200._lib import lib

    g = load_golden("threshold_u16.npz")
    for i, name in enumerate(g["names"]):
        status, got = noalloc_status(lib, g[f"frame{i}"])
        assert status == 0, name
        want = as_records(g[f"signal{i}"], O.SIGNAL_PIXEL)
        assert got.tobytes() == want.tobytes(), name


@pytest.mark.parametrize("h,w", [(1, 7), (9, 1), (23, 233), (257, 511)])
def test_status_codes_match(gpu_lib, h, w):
    from dials_metal_spotfinder_b200._lib import lib

    rng = np.random.default_rng(h * 131 + w)
    img = rng.poisson(3.0, (h, w)).astype(np.uint16)
    img[rng.random((h, w)) < 0.02] += np.uint16(400)
    want_status, want = gpu_lib.find_status(img)
    status, got = noalloc_status(lib, img)
    assert status == want_status
    assert got.tobytes() == want.tobytes()


def test_rejects_frames_beyond_the_scratch(gpu_lib):
    from dials_metal_spotfinder_b200._lib import last_error, lib

    img = np.zeros((4362, 4148), np.uint16)  # an Eiger2 16M frame needs more than 64 MiB
    found = ctypes.c_size_t(7)
    out = np.zeros(1, O.SIGNAL_PIXEL)
    status = lib.sf_find_u16_noalloc(img.ctypes.data, 4362, 4148, out.ctypes.data, 1,
                                     ctypes.byref(found), None)
    assert status == -1 and found.value == 0
    assert "scratch" in last_error()
    # and the entry point still works afterwards
    frame = load_golden("small_series.npz")["frames"][0]
    status, got = noalloc_status(lib, frame)
    assert status == 0 and got.tobytes() == gpu_lib.find(frame).tobytes()
