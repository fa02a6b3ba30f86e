"""The benchmarked configuration itself, checked against the oracle.

The bench's step is threshold + placement + 3D grouping of Eiger2-16M-shaped
frames (4362 x 4148) in batches of 16 frames, with components still open at
the end of a batch carried into the next. These tests run that exact form
through the C ABI on whole 16M series and compare every spot, pixel and count
with the oracle's dext + Labeller (src/dext.cc, src/dials_spots.cc:57-360):

* 48 uint16 frames, three batches of 16 (two batch boundaries), graph replay;
* a uint32 series with intensities up to 2e6 (the 16M uint32 variant), with
  bright planted blobs whose sums of squares pass 2^52, so the spot pass
  takes its sequential path (the exact parallel first pass is refused for
  them) beside the parallel one.
"""

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _threads():
    import os
    return max(1, min(32, os.cpu_count() or 1))


def _make(series, n):
    with ThreadPoolExecutor(_threads()) as pool:
        return list(pool.map(series.frame, range(n)))


def _oracle_lists(frames):
    with ThreadPoolExecutor(_threads()) as pool:
        out = list(pool.map(O.dext, frames))
    for status, _, _ in out:
        assert status == 0
    return [sig for _, sig, _ in out]


def _through_engine(frames, batch, graph):
    from dials_metal_spotfinder_b200.engine import Engine
    spots, pixels = [], []
    with Engine([frames[0].shape] * batch, frames[0].dtype, slots=2) as eng:
        eng.enable_grouping(first_frame=0)
        eng.use_graph(graph)
        for b in range(len(frames) // batch):
            slot = b % 2
            for f in range(batch):
                eng.upload(slot, f, frames[b * batch + f])
            eng.run(slot)
            # the per-frame lists of the last batch, for the threshold check
            lists = [eng.signal(slot, f) for f in range(batch)]
            spots.append(eng.spots())
            pixels.append(eng.pixels())
        eng.finish()
        spots.append(eng.spots())
        pixels.append(eng.pixels())
        counts, live = eng.group_counts()
    return np.concatenate(spots), np.concatenate(pixels), counts, live, lists


@pytest.fixture(scope="module")
def series_16m_u16():
    from dials_metal_spotfinder_b200 import synth
    frames = _make(synth.eiger_16m(frames=48), 48)
    return frames, _oracle_lists(frames)


def test_16m_u16_three_batches_of_16(gpu_lib, series_16m_u16):
    from conftest import same_spots
    frames, lists = series_16m_u16
    spots, pixels, counts, live, last = _through_engine(frames, 16, graph=True)
    for f in range(16):
        assert last[f].tobytes() == lists[32 + f].tobytes(), f
    want = O.group(lists, *frames[0].shape)
    assert counts == want.counts
    assert live == 0
    assert counts["accepted"] > 100_000  # the batches carry many open spots
    same_spots(spots, want.spots)
    assert pixels.tobytes() == want.pixels.tobytes()


def test_16m_u16_boundary_spots_cross_batches(gpu_lib, series_16m_u16):
    """Spots that span a batch boundary exist in this series and are
    emitted once, with every member: the oracle's partition."""
    frames, lists = series_16m_u16
    want = O.group(lists[:32], *frames[0].shape)
    z0, z1 = want.spots["bbox"][:, 4], want.spots["bbox"][:, 5]
    assert int(((z0 < 16) & (z1 > 16)).sum()) > 100


def _bright_u32_series(n):
    """The 16M uint32 variant (intensities log-uniform up to 2e6) with, on
    a few frames, blobs of 3 x 3 x 2 pixels between 2^27 and 2^28: a spot's
    sum of squares then passes 2^52 (while a 7 x 7 window's still fits the
    64-bit accumulator) and its doubles must come from a sequential pass in
    member order."""
    from dials_metal_spotfinder_b200 import synth
    series = synth.eiger_16m(frames=n, dtype=np.uint32)
    frames = _make(series, n)
    rng = np.random.default_rng(0x5EED)
    h, w = frames[0].shape
    for f in range(0, n - 1, 3):
        for _ in range(6):
            y, x = int(rng.integers(30, h - 30)), int(rng.integers(30, w - 30))
            for dz in (0, 1):
                blob = rng.integers(1 << 27, 1 << 28, (3, 3)).astype(np.uint32)
                frames[f + dz][y:y + 3, x:x + 3] = blob
    return frames


def test_16m_u32_series_sequential_and_parallel_spot_pass(gpu_lib):
    from conftest import same_spots
    frames = _bright_u32_series(10)
    lists = _oracle_lists(frames)
    spots, pixels, counts, live, last = _through_engine(frames, 5, graph=False)
    for f in range(5):
        assert last[f].tobytes() == lists[5 + f].tobytes(), f
    want = O.group(lists, *frames[0].shape)
    assert counts == want.counts
    same_spots(spots, want.spots)
    assert pixels.tobytes() == want.pixels.tobytes()
    # the planted blobs are spots whose first pass cannot be exact in
    # parallel: n * max_v^2 is far beyond 2^52
    big = want.spots["intensity"] > 2.0 ** 30
    assert int(big.sum()) >= 6
