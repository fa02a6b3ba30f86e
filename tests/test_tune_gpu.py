"""The autotuner (sf_tune) through the C ABI: a search returns a tuple inside
the asked range and stores it; the next call reads it back from the tuner
file without timing anything; an engine created without explicit tuning
picks it up; and the tuned plan's signal lists and 3D grouping are byte-
identical to other plans' (tuning changes the time, never the result)."""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _frames(n, shape=(700, 900), seed=5):
    from dials_metal_spotfinder_b200 import synth
    h, w = shape
    s = synth.Series(h, w, n + 4, seed, ring_r0=300.0, spots_per_frame=120.0)
    return [s.frame(f) for f in range(n)]


def _run(frames, batch, **kw):
    from dials_metal_spotfinder_b200.engine import Engine
    lists, spots, pixels = [], [], []
    with Engine([frames[0].shape] * batch, frames[0].dtype, slots=2, **kw) as eng:
        tuning = eng.tuning()
        eng.enable_grouping(first_frame=0)
        for b in range(len(frames) // batch):
            for f in range(batch):
                eng.upload(b % 2, f, frames[b * batch + f])
            eng.run(b % 2)
            lists += [eng.signal(b % 2, f) for f in range(batch)]
            spots.append(eng.spots())
            pixels.append(eng.pixels())
        eng.finish()
        spots.append(eng.spots())
        pixels.append(eng.pixels())
    return tuning, lists, np.concatenate(spots), np.concatenate(pixels)


def test_search_cache_and_engine_default(gpu_lib, tmp_path, monkeypatch):
    from conftest import same_spots
    from dials_metal_spotfinder_b200.tune import tune
    cache = str(tmp_path / "tune.txt")
    monkeypatch.setenv("SPOTFINDER_TUNE_CACHE", cache)
    sample = _frames(8)
    first = tune(sample, min_frames=4, max_frames=8, steps=2)
    assert not first["from_cache"] and first["candidates"] >= 4
    assert first["frames_per_launch"] in (4, 8)  # the candidates inside the range
    assert first["candidates"] >= 4
    assert first["warps_per_block"] in (1, 2, 4) and first["seg_rows"] >= 16
    assert first["us_per_frame"] > 0
    again = tune(sample, min_frames=4, max_frames=8)
    assert again["from_cache"] and again["candidates"] == 0
    assert first["blocks_per_sm"] >= 0
    for k in ("frames_per_launch", "warps_per_block", "seg_rows", "seg_ratio", "blocks_per_sm"):
        assert again[k] == first[k], k

    F = first["frames_per_launch"]
    frames = _frames(3 * F, seed=6)
    tuned = _run(frames, F)
    assert tuned[0]["from_cache"]
    assert tuned[0]["warps_per_block"] == first["warps_per_block"]
    assert tuned[0]["seg_rows"] == first["seg_rows"]
    assert tuned[0]["blocks_per_sm"] == first["blocks_per_sm"]
    other = _run(frames, F, seg_rows=17, warps_per_block=1)
    assert not other[0]["from_cache"] and other[0]["seg_rows"] == 17
    for a, b in zip(tuned[1], other[1]):
        assert a.tobytes() == b.tobytes()
    same_spots(tuned[2], other[2])
    assert tuned[3].tobytes() == other[3].tobytes()
    want = O.group([O.dext(img)[1] for img in frames], *frames[0].shape)
    same_spots(tuned[2], want.spots)
    assert tuned[3].tobytes() == want.pixels.tobytes()


def test_no_entry_means_the_cost_model(gpu_lib, tmp_path, monkeypatch):
    from dials_metal_spotfinder_b200.engine import Engine
    monkeypatch.setenv("SPOTFINDER_TUNE_CACHE", str(tmp_path / "empty.txt"))
    with Engine([(300, 400)] * 2, np.uint16) as eng:
        t = eng.tuning()
    assert not t["from_cache"] and t["warps_per_block"] == 2 and t["frames_per_launch"] == 2


def test_bad_arguments(gpu_lib):
    from dials_metal_spotfinder_b200 import BadArgument
    from dials_metal_spotfinder_b200.tune import tune
    with pytest.raises(ValueError):
        tune([])
    with pytest.raises(BadArgument):
        tune(_frames(2, (64, 64)), min_frames=16, max_frames=8)
