"""Pins the oracle (oracle/sf_oracle.c) to the reference's own outputs.

The golden fixtures were written by the reference's compiled code
(tests/golden/make_golden.py). Where oracle/_ref/libref.so is present the
oracle is also compared with it directly on seeded frames. The hand-derived
cases at the bottom are the reference's own grouping tests
(tests/test_dials_spots.cc), with the expected numbers worked there.
CPU only."""

import math

import numpy as np
import pytest

from conftest import as_records, load_golden, same_spots, unpack_list
from oracle import oracle as O


def test_threshold_u16_matches_golden():
    g = load_golden("threshold_u16.npz")
    names = list(g["names"])
    for i, name in enumerate(names):
        img = g[f"frame{i}"]
        want = as_records(g[f"signal{i}"], O.SIGNAL_PIXEL)
        status, got, n = O.dext(img)
        assert status == 0, name
        assert got.tobytes() == want.tobytes(), name


def test_threshold_u32_matches_golden():
    g = load_golden("threshold_u32.npz")
    for i in range(2):
        img = g[f"frame{i}"]
        want = as_records(g[f"signal{i}"], O.SIGNAL_PIXEL)
        status, got, n = O.dext(img)
        assert status == 0 and n == len(want)
        assert got.tobytes() == want.tobytes()


@pytest.mark.parametrize("mode,two_d", [("3d", False), ("2d", True)])
def test_grouping_matches_golden(mode, two_d):
    g = load_golden("small_series.npz")
    signals = unpack_list(g["signal"], g["signal_offsets"], O.SIGNAL_PIXEL)
    # the threshold of every frame, too
    for z, img in enumerate(g["frames"]):
        assert O.dext(img)[1].tobytes() == signals[z].tobytes()
    res = O.group(signals, *g["frames"].shape[1:], two_d=two_d)
    same_spots(res.spots, as_records(g[f"spots_{mode}"], O.SPOT))
    assert res.pixels.tobytes() == as_records(g[f"pixels_{mode}"], O.PIXEL).tobytes()
    assert [res.counts[k] for k in O.COUNT_NAMES] == list(g[f"counts_{mode}"])


def test_capacity_and_bad_arguments():
    img = np.zeros((16, 16), np.uint16)
    assert O.dext(np.zeros((0, 5), np.uint16))[0] == -1
    g = load_golden("threshold_u16.npz")
    frame = g["frame2"]
    status, _, n = O.dext(frame, capacity=10)
    assert status == -2 and n == 531
    assert O.dext(img)[0] == 0


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
def test_oracle_equals_reference_on_seeded_frames():
    rng = np.random.default_rng(7)
    for trial in range(12):
        h, w = int(rng.integers(1, 90)), int(rng.integers(1, 90))
        dtype = np.uint16 if trial % 3 else np.uint32
        lam = float(rng.uniform(0.2, 40))
        img = rng.poisson(lam, (h, w)).astype(dtype)
        for _ in range(int(rng.integers(0, 6))):
            y, x = int(rng.integers(0, h)), int(rng.integers(0, w))
            img[max(0, y - 1):y + 2, max(0, x - 1):x + 2] += dtype(rng.integers(50, 60000))
        if trial % 4 == 0:
            img[rng.random((h, w)) < 0.05] = np.iinfo(dtype).max - int(rng.integers(0, 2))
        a = O.dext(img, use_ref=True)
        b = O.dext(img)
        assert a[0] == b[0] and a[2] == b[2]
        assert a[1].tobytes() == b[1].tobytes()


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
def test_oracle_grouping_equals_reference_with_gaps_and_long_streaks():
    rng = np.random.default_rng(11)
    h, w = 40, 50
    sigs, numbers = [], []
    z = 0
    for f in range(60):
        z += 1 if rng.random() > 0.1 else 2  # occasional missing frame
        idx = np.unique(rng.integers(0, h * w, int(rng.integers(0, 120))))
        idx = np.union1d(idx, [101, 102, 103])  # a streak through every frame
        sig = np.zeros(len(idx), O.SIGNAL_PIXEL)
        sig["index"] = idx
        sig["value"] = rng.integers(1, 5000, len(idx))
        sigs.append(sig)
        numbers.append(z)
    for two_d in (False, True):
        for sep in (2.0, 0.0):
            a = O.group(sigs, h, w, numbers, use_ref=True, two_d=two_d, max_separation=sep,
                        min_spot_size=1)
            b = O.group(sigs, h, w, numbers, two_d=two_d, max_separation=sep, min_spot_size=1)
            same_spots(b.spots, a.spots)
            assert a.pixels.tobytes() == b.pixels.tobytes()
            assert a.counts == b.counts


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("config", ["4m_u16", "16m_u32"])
def test_oracle_equals_reference_on_detector_frames(config):
    """Whole detector frames at the benchmark's density (module gaps,
    Poisson ring, reflections): the restatement and the reference's own
    dext<T> give the same list, byte for byte."""
    from dials_metal_spotfinder_b200 import synth
    if config == "4m_u16":
        img = synth.eiger_4m(frames=2).frame(1)
    else:
        img = synth.eiger_16m(frames=2, dtype=np.uint32).frame(1)
    a = O.dext(img, use_ref=True)
    b = O.dext(img)
    assert a[0] == b[0] == 0 and a[2] == b[2] > 1000
    assert a[1].tobytes() == b[1].tobytes()


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
def test_oracle_grouping_equals_reference_on_a_4m_series():
    """Eight consecutive 4M frames, thresholded by the reference, grouped in
    3D and in 2D with the default options by both."""
    from dials_metal_spotfinder_b200 import synth
    series = synth.eiger_4m(frames=8)
    frames = [series.frame(z) for z in range(8)]
    sigs = [O.dext(img, use_ref=True)[1] for img in frames]
    for two_d in (False, True):
        a = O.group(sigs, *frames[0].shape, use_ref=True, two_d=two_d)
        b = O.group(sigs, *frames[0].shape, two_d=two_d)
        assert a.counts == b.counts and a.counts["accepted"] > 100
        assert a.spots.tobytes() == b.spots.tobytes()
        assert a.pixels.tobytes() == b.pixels.tobytes()


# -- hand-derived cases from the reference's tests/test_dials_spots.cc -------

H, W = 8, 10


def flat(indices, value):
    sig = np.zeros(len(indices), O.SIGNAL_PIXEL)
    sig["index"] = indices
    sig["value"] = value
    return sig


def pairs(at):
    sig = np.zeros(len(at), O.SIGNAL_PIXEL)
    sig["index"] = [a for a, _ in at]
    sig["value"] = [v for _, v in at]
    return sig


def close(a, b):
    assert abs(a - b) < 1e-9, (a, b)


def test_three_pixels_in_a_row():
    res = O.group([pairs([(0, 1), (1, 2), (2, 1)])], H, W, max_separation=0.0)
    assert len(res.spots) == 1
    s = res.spots[0]
    assert s["n_signal"] == 3
    close(s["intensity"], 4.0)
    close(s["position"][0], 1.5)
    close(s["position"][1], 0.5)
    close(s["position"][2], 0.5)
    close(s["variance"][0], 0.8 / 4 + 1 / 12)
    close(s["variance"][1], 1 / 12)
    assert list(s["bbox"]) == [0, 3, 0, 1, 0, 1]


def test_streak_is_one_spot_in_3d_three_in_2d():
    sigs = [flat([0, 1, 2], 1)] * 3
    res = O.group(sigs, H, W, max_separation=0.0)
    assert len(res.spots) == 1 and res.spots[0]["n_signal"] == 9
    close(res.spots[0]["variance"][2], 0.75 / 9 + 1 / 12)
    res2 = O.group(sigs, H, W, max_separation=0.0, two_d=True)
    assert len(res2.spots) == 3
    close(res2.spots[1]["position"][2], 1.5)


def test_missing_frame_breaks_connection():
    sigs = [flat([0, 1, 2], 1)] * 4
    res = O.group(sigs, H, W, [0, 1, 3, 4], max_separation=0.0)
    assert [s["n_signal"] for s in res.spots] == [6, 6]
    assert res.spots[1]["bbox"][4] == 3


@pytest.mark.parametrize("idx,expect", [([9, 10], 2), ([0, 10], 1), ([0, 11], 2)])
def test_connectivity_edges(idx, expect):
    res = O.group([flat(idx, 1)], H, W, max_separation=0.0, min_spot_size=1)
    assert len(res.spots) == expect


def test_size_and_separation_filters():
    res = O.group([flat([0, 1], 1), flat([40, 41, 42], 1)], H, W, max_separation=0.0)
    assert len(res.spots) == 1 and res.counts["too_small"] == 1
    res = O.group([flat([0, 1, 2, 3, 4, 5], 1)], H, W, max_separation=0.0, max_spot_size=5)
    assert len(res.spots) == 0 and res.counts["too_large"] == 1
    at = [(0, 100), (1, 100), (2, 1), (3, 1), (4, 1), (5, 1), (6, 90), (7, 90)]
    res = O.group([pairs(at)], H, W, max_separation=2.0)
    assert len(res.spots) == 0 and res.counts["separated"] == 1


def test_single_pixel_fallback_variance():
    res = O.group([flat([35], 700)], H, W, max_separation=0.0, min_spot_size=1)
    s = res.spots[0]
    close(s["position"][0], 5.5)
    close(s["position"][1], 3.5)
    close(s["variance"][0], 1 / 12)


def test_refusals():
    lab = O.Labeller(H, W, max_separation=0.0)
    lab.add(5, flat([0, 1, 2], 1))
    for frame, sig in ((4, flat([0], 1)), (5, flat([0], 1))):
        with pytest.raises(RuntimeError):
            lab.add(frame, sig)
    lab = O.Labeller(H, W)
    with pytest.raises(RuntimeError):
        lab.add(0, flat([2, 1], 1))
    with pytest.raises(RuntimeError):
        lab.add(0, flat([H * W], 1))


def test_long_streak_compaction():
    sigs = [flat([44, 45, 46, 70, 71, 72], 3)] * 200
    res = O.group(sigs, H, W, max_separation=0.0)
    assert [s["n_signal"] for s in res.spots] == [600, 600]
    assert res.spots[0]["bbox"][5] - res.spots[0]["bbox"][4] == 200
    assert len(res.pixels) == 1200
