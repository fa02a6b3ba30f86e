"""The batched engine through the C ABI: every frame of a batch -- equal or
uneven shapes, either pixel type, any slot, graph replay or not -- gives
exactly the per-frame threshold (and so the oracle's output)."""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def frames_for(shapes, seed, dtype=np.uint16):
    rng = np.random.default_rng(seed)
    out = []
    for h, w in shapes:
        img = rng.poisson(2.0, (h, w)).astype(dtype)
        n = max(1, h * w // 300)
        ys, xs = rng.integers(0, h, n), rng.integers(0, w, n)
        for y, x in zip(ys, xs):
            img[max(0, y - 2):y + 3, max(0, x - 2):x + 3] += dtype(rng.integers(20, 5000))
        img[rng.random((h, w)) < 0.003] = np.iinfo(dtype).max
        out.append(img)
    return out


@pytest.mark.parametrize("graph", [False, True])
def test_uneven_batch_two_slots(gpu_lib, graph):
    from dials_metal_spotfinder_b200.engine import Engine
    shapes = [(300, 500), (64, 90), (531, 233), (1062, 1028), (7, 3), (250, 700)]
    batches = [frames_for(shapes, 1), frames_for(shapes, 2)]
    with Engine(shapes, np.uint16, slots=2) as eng:
        eng.use_graph(graph)
        for s in range(2):
            for f, img in enumerate(batches[s]):
                eng.upload(s, f, img)
        for rep in range(2):
            for s in range(2):
                eng.run(s)
            eng.synchronize()
            for s in range(2):
                counts = eng.counts(s)
                for f, img in enumerate(batches[s]):
                    st, want, n = O.dext(img, capacity=img.size * 2 // 16)
                    status, got = eng.signal_status(s, f)
                    assert counts[f] == n
                    assert status == st
                    if st == 0:
                        assert got.tobytes() == want.tobytes(), (s, f)


def test_u32_batch(gpu_lib):
    from dials_metal_spotfinder_b200.engine import Engine
    shapes = [(120, 260), (200, 150)]
    frames = frames_for(shapes, 3, np.uint32)
    frames[0][10:14, 10:14] += np.uint32(1_500_000)
    with Engine(shapes, np.uint32) as eng:
        for f, img in enumerate(frames):
            eng.upload(0, f, img)
        eng.run(0)
        eng.synchronize()
        for f, img in enumerate(frames):
            assert eng.signal(0, f).tobytes() == O.dext(img)[1].tobytes()


@pytest.mark.parametrize("seg,wpc", [(16, 1), (37, 2), (500, 4), (0, 4)])
def test_tunings_agree(gpu_lib, seg, wpc):
    from dials_metal_spotfinder_b200.engine import Engine
    shapes = [(400, 700), (333, 941)]
    frames = frames_for(shapes, 4)
    with Engine(shapes, np.uint16, seg_rows=seg, warps_per_block=wpc) as eng:
        for f, img in enumerate(frames):
            eng.upload(0, f, img)
        eng.run(0)
        eng.synchronize()
        for f, img in enumerate(frames):
            assert eng.signal(0, f).tobytes() == O.dext(img)[1].tobytes()


def test_16m_batch_matches_oracle(gpu_lib):
    from dials_metal_spotfinder_b200 import synth
    from dials_metal_spotfinder_b200.engine import Engine
    series = synth.eiger_16m(frames=4)
    frames = [series.frame(f) for f in (0, 1)]
    with Engine([f.shape for f in frames], np.uint16) as eng:
        for f, img in enumerate(frames):
            eng.upload(0, f, img)
        eng.run(0)
        eng.synchronize()
        for f, img in enumerate(frames):
            assert eng.signal(0, f).tobytes() == O.dext(img)[1].tobytes()


def run_series_through_engine(frames, batch, graph, slots=2, two_d=False):
    """Every frame of a series through the engine with grouping, `batch`
    frames per run; returns all spots, pixels and the final counts."""
    from dials_metal_spotfinder_b200.engine import Engine
    shape = frames[0].shape
    spots, pixels = [], []
    with Engine([shape] * batch, frames[0].dtype, slots=slots) as eng:
        eng.enable_grouping(first_frame=0, two_d=two_d)
        eng.use_graph(graph)
        nb = len(frames) // batch
        for b in range(nb):
            slot = b % slots
            for f in range(batch):
                eng.upload(slot, f, frames[b * batch + f])
            eng.run(slot)
            spots.append(eng.spots())
            pixels.append(eng.pixels())
        eng.finish()
        spots.append(eng.spots())
        pixels.append(eng.pixels())
        counts, live = eng.group_counts()
    return np.concatenate(spots), np.concatenate(pixels), counts


@pytest.mark.parametrize("batch,graph,two_d", [(1, False, False), (3, False, False),
                                               (3, True, False), (2, True, True)])
def test_engine_grouping_matches_oracle(gpu_lib, batch, graph, two_d):
    from conftest import same_spots
    from dials_metal_spotfinder_b200 import synth
    series = synth.small()
    frames = [series.frame(f) for f in range(12)]
    spots, pixels, counts = run_series_through_engine(frames, batch, graph, two_d=two_d)
    want = O.group([O.dext(img)[1] for img in frames], *frames[0].shape, two_d=two_d)
    assert counts == want.counts
    same_spots(spots, want.spots)
    assert pixels.tobytes() == want.pixels.tobytes()


def test_engine_grouping_4m(gpu_lib):
    from conftest import same_spots
    from dials_metal_spotfinder_b200 import synth
    series = synth.eiger_4m(frames=8)
    frames = [series.frame(f) for f in range(8)]
    spots, pixels, counts = run_series_through_engine(frames, 4, True)
    want = O.group([O.dext(img)[1] for img in frames], *frames[0].shape)
    assert counts == want.counts
    same_spots(spots, want.spots)
    assert pixels.tobytes() == want.pixels.tobytes()


def test_results_into_pinned_arrays(gpu_lib):
    """spots()/pixels() into caller arrays (page-locked here) give the same
    records as the allocating form, while the next run's frames upload; an
    array too short raises Overflow."""
    import dials_metal_spotfinder_b200 as sf
    from dials_metal_spotfinder_b200 import synth
    from dials_metal_spotfinder_b200.engine import Engine
    series = synth.small()
    frames = [series.frame(f) for f in range(6)]
    ref_spots, ref_pixels, _ = run_series_through_engine(frames, 2, False)
    sb = sf.HostBuffer((len(ref_spots) + 16,), sf.SPOT)
    pb = sf.HostBuffer((len(ref_pixels) + 16,), sf.PIXEL)
    spots, pixels = [], []
    try:
        with Engine([frames[0].shape] * 2, frames[0].dtype, slots=2) as eng:
            eng.enable_grouping(first_frame=0)
            for f in range(2):
                eng.upload(0, f, frames[f])
            eng.run(0)
            for b in (1, 2):
                for f in range(2):
                    eng.upload(b % 2, f, frames[2 * b + f])
                spots.append(eng.spots(out=sb.array).copy())
                pixels.append(eng.pixels(out=pb.array).copy())
                eng.run(b % 2)
            spots.append(eng.spots(out=sb.array).copy())
            pixels.append(eng.pixels(out=pb.array).copy())
            eng.finish()
            n = len(eng.pixels())
            if n:
                with pytest.raises(sf.Overflow):
                    eng.pixels(out=np.zeros(n - 1, sf.PIXEL))
            spots.append(eng.spots(out=sb.array).copy())
            pixels.append(eng.pixels(out=pb.array).copy())
    finally:
        sb.close()
        pb.close()
    assert np.concatenate(spots).tobytes() == ref_spots.tobytes()
    assert np.concatenate(pixels).tobytes() == ref_pixels.tobytes()


def test_batch_list_read_equals_per_frame_reads(gpu_lib):
    """signals(): every frame's list in one call, back to back, equal to the
    per-frame reads; a too-small array is refused with the counts filled."""
    import dials_metal_spotfinder_b200 as sf
    from dials_metal_spotfinder_b200.engine import Engine
    shapes = [(300, 500), (64, 90), (531, 233)]
    frames = frames_for(shapes, 9)
    with Engine(shapes, np.uint16) as eng:
        for f, img in enumerate(frames):
            eng.upload(0, f, img)
        eng.run(0)
        lists, counts = eng.signals(0)
        for f, img in enumerate(frames):
            assert lists[f].tobytes() == eng.signal(0, f).tobytes()
            assert lists[f].tobytes() == O.dext(img)[1].tobytes()
            assert counts[f] == len(lists[f])
        with pytest.raises(sf.Overflow):
            eng.signals(0, out=np.zeros(int(counts.sum()) - 1, sf.SIGNAL_PIXEL))
