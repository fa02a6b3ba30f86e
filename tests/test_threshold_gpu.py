"""The CUDA threshold against the oracle: every SignalPixel field equal, as the
reference's own device test demands (tests/test_dext_gpu.cc:155-199), on the
reference's frame set, the configurations' shapes and the edge cases.
Calls go through the C ABI (sf_find_u16 / sf_find_u32)."""

import numpy as np
import pytest

from conftest import as_records, load_golden, unpack_list
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def same(got, want, what=""):
    assert len(got) == len(want), f"{what}: {len(got)} vs {len(want)}"
    if got.tobytes() != want.tobytes():
        bad = np.nonzero(got.view(np.uint8).reshape(-1, 16).any(1) != 0)[0]
        for k in range(len(got)):
            if got[k].tobytes() != want[k].tobytes():
                raise AssertionError(f"{what}: entry {k} differs: {got[k]} vs {want[k]}")
        raise AssertionError(f"{what}: differ ({len(bad)})")


def test_reference_frame_set(gpu_lib):
    g = load_golden("threshold_u16.npz")
    for i, name in enumerate(g["names"]):
        same(gpu_lib.find(g[f"frame{i}"]), as_records(g[f"signal{i}"], O.SIGNAL_PIXEL), name)


def test_u32_frames(gpu_lib):
    g = load_golden("threshold_u32.npz")
    for i in range(2):
        same(gpu_lib.find(g[f"frame{i}"]), as_records(g[f"signal{i}"], O.SIGNAL_PIXEL), f"u32 {i}")


def test_small_series(gpu_lib):
    g = load_golden("small_series.npz")
    signals = unpack_list(g["signal"], g["signal_offsets"], O.SIGNAL_PIXEL)
    for z, img in enumerate(g["frames"]):
        same(gpu_lib.find(img), signals[z], f"frame {z}")


@pytest.mark.parametrize("h,w", [(1, 1), (1, 7), (9, 1), (2, 2), (5, 300), (300, 5),
                                 (21, 231), (22, 232), (23, 233), (40, 464), (41, 465),
                                 (19, 27), (257, 511), (600, 700), (1033, 1041)])
def test_ragged_shapes(gpu_lib, h, w):
    rng = np.random.default_rng(h * 10007 + w)
    img = rng.poisson(3.0, (h, w)).astype(np.uint16)
    n = max(1, h * w // 400)
    ys, xs = rng.integers(0, h, n), rng.integers(0, w, n)
    for y, x in zip(ys, xs):
        img[max(0, y - 1):y + 2, max(0, x - 1):x + 2] += np.uint16(rng.integers(30, 3000))
    img[rng.random((h, w)) < 0.01] = 0xFFFF
    img[rng.random((h, w)) < 0.01] = 0xFFFE
    want = O.dext(img)
    status, got = gpu_lib.find_status(img)
    # The device list holds height * width * 2 / 16 entries, as the
    # reference's does (src/dext_cuda.cu:611-616): a frame with more signal
    # than that is refused with -2, even a tiny one with a single pixel.
    if want[2] > h * w * 2 // 16:
        assert status == -2 and len(got) == 0
        return
    assert status == want[0]
    same(got, want[1], f"{h}x{w}")


@pytest.mark.parametrize("fill", [0, 1, 0xFFFE, 0xFFFF, 0xFFFD])
def test_uniform_frames(gpu_lib, fill):
    img = np.full((70, 300), fill, np.uint16)
    same(gpu_lib.find(img), O.dext(img)[1], f"fill {fill}")


def test_wrapping_sum_of_squares(gpu_lib):
    # Windows whose sum of squares passes 2^32: the wrapped value must match.
    rng = np.random.default_rng(3)
    img = rng.poisson(2.0, (120, 150)).astype(np.uint16)
    img[40:47, 40:47] = rng.integers(20000, 65533, (7, 7))
    img[80:83, 100:103] = 65533
    img[10:12, 10:60] = rng.integers(30000, 65000, (2, 50))
    same(gpu_lib.find(img), O.dext(img)[1], "wrap")


def test_u32_random_with_sentinels(gpu_lib):
    rng = np.random.default_rng(5)
    for h, w in ((50, 70), (233, 481)):
        img = rng.poisson(6.0, (h, w)).astype(np.uint32)
        k = rng.integers(0, h * w, h * w // 50)
        img.reshape(-1)[k] += rng.integers(1000, 3_000_000, len(k)).astype(np.uint32)
        img[rng.random((h, w)) < 0.01] = 0xFFFFFFFF
        img[rng.random((h, w)) < 0.01] = 0xFFFFFFFE
        same(gpu_lib.find(img), O.dext(img)[1], f"u32 {h}x{w}")


def test_bad_arguments(gpu_lib):
    assert gpu_lib.find_status(np.zeros((0, 10), np.uint16))[0] == -1
    assert gpu_lib.find_status(np.zeros((10, 0), np.uint16))[0] == -1
    assert gpu_lib.find_status(np.zeros((4, 4), np.int32))[0] == -1
    # height * width beyond INT32_MAX is refused before anything is allocated
    import ctypes
    from dials_metal_spotfinder_b200 import _lib
    found = ctypes.c_size_t(7)
    buf = np.zeros(4, np.uint16)
    assert _lib.lib.sf_find_u16(buf.ctypes.data, 70000, 40000, None, 0,
                                ctypes.byref(found)) == -1
    assert _lib.lib.sf_find_u16(None, 4, 4, None, 0, ctypes.byref(found)) == -1


def test_overflow_returns_minus_two(gpu_lib):
    # A frame denser in signal than the reference's list holds (1 in 8).
    rng = np.random.default_rng(17)
    img = None
    for trial in range(50):
        cand = rng.poisson(1.0, (48, 64)).astype(np.uint16)
        cand[rng.random(cand.shape) < 0.45] = rng.integers(200, 20000)
        st, _, n = O.dext(cand, capacity=48 * 64 * 2 // 16)
        if st == -2:
            img = cand
            break
    assert img is not None, "could not build an over-dense frame"
    status, got = gpu_lib.find_status(img)
    assert status == -2 and len(got) == 0


@pytest.mark.parametrize("which", ["4m", "16m"])
def test_configuration_frames(gpu_lib, which):
    from dials_metal_spotfinder_b200 import synth
    series = synth.eiger_4m(frames=4) if which == "4m" else synth.eiger_16m(frames=3)
    for f in (1, 2):
        img = series.frame(f)
        st, want, n = O.dext(img)
        assert st == 0
        same(gpu_lib.find(img), want, f"{which} frame {f}")


def test_u32_16m_variant_frame(gpu_lib):
    from dials_metal_spotfinder_b200 import synth
    series = synth.eiger_16m(frames=3, dtype=np.uint32)
    img = series.frame(1)
    st, want, n = O.dext(img)
    assert st == 0
    same(gpu_lib.find(img), want, "u32 16M")


def test_concurrent_threads(gpu_lib):
    from concurrent.futures import ThreadPoolExecutor
    g = load_golden("small_series.npz")
    signals = unpack_list(g["signal"], g["signal_offsets"], O.SIGNAL_PIXEL)
    frames = list(g["frames"])

    def run(z):
        return z, gpu_lib.find(frames[z])

    with ThreadPoolExecutor(6) as pool:
        for z, got in pool.map(run, list(range(len(frames))) * 3):
            same(got, signals[z], f"thread frame {z}")


def test_find_into_pinned_list(gpu_lib):
    """The list written into a caller's page-locked array is the same list,
    returned as a view of it; an array of the wrong record type is refused."""
    g = load_golden("threshold_u16.npz")
    img = g["frame0"]
    cap = img.shape[0] * img.shape[1] * 2 // 16
    buf = gpu_lib.HostBuffer((cap,), gpu_lib.SIGNAL_PIXEL)
    try:
        got = gpu_lib.find(img, out=buf.array)
        assert np.shares_memory(got, buf.array)
        same(got, as_records(g["signal0"], O.SIGNAL_PIXEL), "pinned")
        status, _ = gpu_lib.find_status(img, out=np.zeros(cap, np.uint64))
        assert status == -1
    finally:
        buf.close()
