"""Uneven batches: several series of different frame shapes interleaved in
the same launches of the batched engine, each series grouped by its own
labeller in the same stream (the reference runs one Labeller per series,
src/find_spots.cc:460-636). Per frame the signal list equals the oracle's
dext (src/dext.cc), and per series the spots, pixels and counts equal the
oracle's Labeller fed that series alone (src/dials_spots.cc)."""

import numpy as np
import pytest

from conftest import same_spots
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# the four stills panels, slow x fast
STILLS = [(1062, 1028), (2162, 2068), (3269, 3110), (4362, 4148)]


def run_interleaved(series_list, per_run, runs, two_d, graph):
    """Batches of `per_run` frames of every series, interleaved series by
    series; returns per series (signal lists, spots, pixels, counts)."""
    from dials_metal_spotfinder_b200.engine import Engine
    shapes = []
    for _ in range(per_run):
        shapes += [(s.height, s.width) for s in series_list]
    eng = Engine(shapes, np.uint16, slots=2)
    eng.enable_grouping(first_frame=0, two_d=two_d)
    assert eng.nseries() == len(series_list)
    if graph:
        eng.use_graph(True)
    k = len(series_list)
    signals = [[] for _ in range(k)]
    spots = [[] for _ in range(k)]
    pixels = [[] for _ in range(k)]
    for r in range(runs):
        slot = r % 2
        frames = []
        for i in range(per_run):
            for j, s in enumerate(series_list):
                img = s.frame(r * per_run + i)
                frames.append(img)
                eng.upload(slot, len(frames) - 1, img)
        eng.run(slot)
        eng.synchronize()
        for f in range(len(frames)):
            signals[f % k].append(eng.signal(slot, f))
        for j in range(k):
            spots[j].append(eng.spots(j))
            pixels[j].append(eng.pixels(j))
    eng.finish()
    for j in range(k):
        spots[j].append(eng.spots(j))
        pixels[j].append(eng.pixels(j))
    counts = [eng.group_counts(j)[0] for j in range(k)]
    shapes_seen = [eng.series_shape(j) for j in range(k)]
    eng.close()
    assert shapes_seen == [(s.height, s.width) for s in series_list]
    return signals, [np.concatenate(x) for x in spots], [np.concatenate(x) for x in pixels], counts


def check_against_oracle(series_list, signals, spots, pixels, counts, two_d):
    for j, s in enumerate(series_list):
        for z, got in enumerate(signals[j]):
            want = O.dext(s.frame(z))[1]
            assert got.tobytes() == want.tobytes(), f"series {j} frame {z}"
        want = O.group(signals[j], s.height, s.width, two_d=two_d)
        assert counts[j] == want.counts, f"series {j}"
        same_spots(spots[j], want.spots)
        assert pixels[j].tobytes() == want.pixels.tobytes(), f"series {j}"


def test_uneven_stills_2d():
    from dials_metal_spotfinder_b200 import synth
    series_list = [synth.still(shape, frames=4) for shape in STILLS]
    out = run_interleaved(series_list, per_run=2, runs=2, two_d=True, graph=False)
    check_against_oracle(series_list, *out, two_d=True)


def test_two_rotation_series_3d_graph():
    from dials_metal_spotfinder_b200 import synth
    series_list = [synth.eiger_4m(frames=6), synth.small()]
    out = run_interleaved(series_list, per_run=2, runs=3, two_d=False, graph=True)
    check_against_oracle(series_list, *out, two_d=False)
