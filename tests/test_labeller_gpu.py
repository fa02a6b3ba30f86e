"""The device labeller (sf_labeller_*) against the oracle and the reference's
golden grouping: spots, pixels and counts byte-identical (centroids and
variances bit-equal -- tighter than the 1e-9 relative the parity rule
allows), in the same order. The hand-derived cases are the reference's own
tests/test_dials_spots.cc."""

import numpy as np
import pytest

from conftest import as_records, load_golden, same_spots, unpack_list
from oracle import oracle as O

pytestmark = pytest.mark.gpu

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


def device(signals, h, w, frames=None, **opt):
    from dials_metal_spotfinder_b200.labeller import group
    return group(signals, h, w, frames, **opt)


def assert_same(signals, h, w, frames=None, **opt):
    spots, pixels, counts = device(signals, h, w, frames, **opt)
    want = O.group(signals, h, w, frames, **opt)
    assert counts == want.counts
    same_spots(spots, want.spots)
    assert pixels.tobytes() == want.pixels.tobytes()
    return spots


def test_three_pixels_in_a_row(gpu_lib):
    s = assert_same([pairs([(0, 1), (1, 2), (2, 1)])], H, W, max_separation=0.0)
    assert len(s) == 1 and abs(s[0]["variance"][0] - (0.8 / 4 + 1 / 12)) < 1e-12


def test_streak_3d_and_2d(gpu_lib):
    sigs = [flat([0, 1, 2], 1)] * 3
    assert len(assert_same(sigs, H, W, max_separation=0.0)) == 1
    assert len(assert_same(sigs, H, W, max_separation=0.0, two_d=True)) == 3


def test_missing_frame_breaks_connection(gpu_lib):
    sigs = [flat([0, 1, 2], 1)] * 4
    s = assert_same(sigs, H, W, [0, 1, 3, 4], max_separation=0.0)
    assert [int(x["n_signal"]) for x in s] == [6, 6]


@pytest.mark.parametrize("idx", [[9, 10], [0, 10], [0, 11]])
def test_connectivity_edges(gpu_lib, idx):
    assert_same([flat(idx, 1)], H, W, max_separation=0.0, min_spot_size=1)


def test_diagonal_in_z_is_not_an_edge(gpu_lib):
    assert len(assert_same([flat([0], 1), flat([10], 1)], H, W, max_separation=0.0,
                           min_spot_size=1)) == 2


def test_filters(gpu_lib):
    assert_same([flat([0, 1], 1), flat([40, 41, 42], 1)], H, W, max_separation=0.0)
    assert_same([flat([0, 1, 2, 3, 4, 5], 1)], H, W, max_separation=0.0, max_spot_size=5)
    at = [(0, 100), (1, 100), (2, 1), (3, 1), (4, 1), (5, 1), (6, 90), (7, 90)]
    assert_same([pairs(at)], H, W, max_separation=2.0)
    tail = [(0, 1000)] + [(x, 1) for x in range(1, 10)]
    assert_same([pairs(tail)], H, W, max_separation=2.0)
    assert_same([flat([35], 700)], H, W, max_separation=0.0, min_spot_size=1)


def test_no_early_emit_and_live(gpu_lib):
    from dials_metal_spotfinder_b200.labeller import Labeller
    lab = Labeller(H, W, max_separation=0.0)
    lab.add(0, flat([0, 1, 2], 1))
    assert len(lab.spots()) == 0 and lab.live() == 3
    lab.add(1, flat([40, 41, 42], 1))
    assert len(lab.spots()) == 1 and lab.live() == 3
    lab.finish()
    assert len(lab.spots()) == 2 and lab.live() == 0


def test_refusals_leave_state_unchanged(gpu_lib):
    import dials_metal_spotfinder_b200 as sf
    from dials_metal_spotfinder_b200.labeller import Labeller
    lab = Labeller(H, W, max_separation=0.0)
    lab.add(5, flat([0, 1, 2], 1))
    for frame, sig in ((4, flat([0], 1)), (5, flat([0], 1)), (6, flat([2, 1], 1)),
                       (6, flat([H * W], 1))):
        with pytest.raises(sf.Refused):
            lab.add(frame, sig)
    lab.add(6, flat([0, 1, 2], 1))
    lab.finish()
    assert [int(s["n_signal"]) for s in lab.spots()] == [6]


def test_long_streak_compaction(gpu_lib):
    sigs = [flat([44, 45, 46, 70, 71, 72], 3)] * 200
    s = assert_same(sigs, H, W, max_separation=0.0)
    assert [int(x["n_signal"]) for x in s] == [600, 600]


@pytest.mark.parametrize("mode,two_d", [("3d", False), ("2d", True)])
def test_small_series_golden(gpu_lib, mode, two_d):
    g = load_golden("small_series.npz")
    signals = unpack_list(g["signal"], g["signal_offsets"], O.SIGNAL_PIXEL)
    spots, pixels, counts = device(signals, *g["frames"].shape[1:], two_d=two_d)
    same_spots(spots, as_records(g[f"spots_{mode}"], O.SPOT))
    assert pixels.tobytes() == as_records(g[f"pixels_{mode}"], O.PIXEL).tobytes()
    assert [counts[k] for k in O.COUNT_NAMES] == list(g[f"counts_{mode}"])


@pytest.mark.parametrize("two_d,sep", [(False, 2.0), (False, 0.0), (True, 2.0)])
def test_random_series_with_gaps(gpu_lib, two_d, sep):
    rng = np.random.default_rng(11 + int(two_d) + int(sep))
    h, w = 40, 50
    sigs, numbers, z = [], [], 0
    for f in range(80):
        z += 1 if rng.random() > 0.1 else 2
        idx = np.unique(rng.integers(0, h * w, int(rng.integers(0, 150))))
        idx = np.union1d(idx, [101, 102, 103, 151])
        sig = np.zeros(len(idx), O.SIGNAL_PIXEL)
        sig["index"] = idx
        sig["value"] = rng.integers(1, 60000, len(idx))
        sigs.append(sig)
        numbers.append(z)
    assert_same(sigs, h, w, numbers, two_d=two_d, max_separation=sep, min_spot_size=1)
    assert_same(sigs, h, w, numbers, two_d=two_d, max_separation=sep, min_spot_size=3,
                max_spot_size=40)


def test_empty_frames_and_empty_series(gpu_lib):
    e = np.zeros(0, O.SIGNAL_PIXEL)
    assert_same([e, flat([3, 4, 5], 2), e, e, flat([3, 4, 5], 2)], H, W)
    assert_same([e, e], H, W)
    from dials_metal_spotfinder_b200.labeller import Labeller
    lab = Labeller(H, W)
    lab.finish()
    assert len(lab.spots()) == 0


def test_threshold_then_group_4m(gpu_lib):
    """Frames of the 4M configuration through the device threshold and the
    device labeller, against the oracle on the same frames."""
    from dials_metal_spotfinder_b200 import synth
    series = synth.eiger_4m(frames=6)
    frames = [series.frame(f) for f in range(6)]
    sigs = [gpu_lib.find(img) for img in frames]
    for img, sig in zip(frames, sigs):
        assert sig.tobytes() == O.dext(img)[1].tobytes()
    assert_same(sigs, *frames[0].shape)


def test_components_of_every_size_class(gpu_lib):
    """Components handled by each path of the spot pass: up to 512 members,
    512 to 1024 (the large-buffer launch) and beyond 1024 (through global
    memory, reachable with max_spot_size above 1024), with uneven values so
    that the doubles depend on the member order, and bright enough that the
    first pass can not be summed in parallel exactly."""
    rng = np.random.default_rng(5)
    h, w = 120, 160
    sigs = []
    for z in range(4):
        idx = []
        for y0, x0, side in ((5, 5, 10), (30, 40, 15), (70, 20, 24), (60, 100, 30)):
            ys, xs = np.mgrid[y0:y0 + side, x0:x0 + side]
            idx.append((ys * w + xs).ravel())
        idx = np.unique(np.concatenate(idx))
        sig = np.zeros(len(idx), O.SIGNAL_PIXEL)
        sig["index"] = idx
        sig["value"] = rng.integers(1, 0xFFFE, len(idx))
        sig["value"][::97] = 4_000_000_000  # 32-bit values: inexact parallel sums
        sigs.append(sig)
    spots = assert_same(sigs, h, w, max_spot_size=100000, max_separation=0.0)
    sizes = sorted(int(s["n_signal"]) for s in spots)
    assert sizes == [400, 900, 2304, 3600]  # 4 frames of 10^2, 15^2, 24^2 and 30^2
    assert_same(sigs, h, w, max_spot_size=100000, max_separation=2.0)
