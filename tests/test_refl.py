"""The .refl writer (sf_refl_write; the reference's refl::write, src/refl.cc:
223-351) against the reference's own output: byte for byte on the golden
spot lists (tests/golden/refl_small*.refl, written by the reference from
the small configuration: 3D with shoeboxes, 2D with an empty identifier
map, 3D without shoeboxes under experiment id 3), and column by column on a
larger series grouped on the device. The shoebox column is built on the
device."""

import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, as_records, load_golden
from oracle import oracle as O
from refl_reader import read, shoeboxes

CASES = [("refl_small.refl", "3d", "golden", 0, True),
         ("refl_small_2d.refl", "2d", "", 0, True),
         ("refl_small_noshoebox.refl", "3d", "golden-3", 3, False)]
# The reference tree: $SPOTFINDER_REFERENCE, else a `reference` directory
# beside this repository. Absent on a machine without it (the test skips).
REFERENCE = os.environ.get("SPOTFINDER_REFERENCE") or os.path.join(
    os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))), "reference")
CHECK_REFL = os.path.join(REFERENCE, "tests", "check_refl.py")
COLUMNS = {"bbox": "int6", "flags": "std::size_t", "id": "int", "intensity.sum.value": "double",
           "intensity.sum.variance": "double", "n_signal": "int", "panel": "std::size_t",
           "shoebox": "Shoebox<>", "xyzobs.px.value": "vec3<double>",
           "xyzobs.px.variance": "vec3<double>"}


def check_table(path, spots, pixels, width, identifier, exp_id, with_shoeboxes):
    t = read(path)
    assert t["name"] == "dials::af::reflection_table" and t["version"] == 2
    assert t["nrows"] == len(spots)
    assert t["identifiers"] == ({exp_id: identifier} if identifier else {})
    want = dict(COLUMNS)
    if not with_shoeboxes:
        del want["shoebox"]
    assert {k: v[0] for k, v in t["columns"].items()} == want
    assert list(t["columns"]) == sorted(want)
    cols = t["columns"]
    n = len(spots)
    assert all(c[1] == n for c in cols.values())
    assert np.frombuffer(cols["bbox"][2], "<i4").reshape(n, 6).tolist() == spots["bbox"].tolist()
    assert (np.frombuffer(cols["flags"][2], "<u8") == 32).all()
    assert (np.frombuffer(cols["id"][2], "<i4") == exp_id).all()
    assert np.frombuffer(cols["intensity.sum.value"][2], "<f8").tobytes() == \
        np.ascontiguousarray(spots["intensity"]).tobytes()
    assert np.frombuffer(cols["n_signal"][2], "<i4").tolist() == spots["n_signal"].tolist()
    assert np.frombuffer(cols["xyzobs.px.value"][2], "<f8").tobytes() == \
        np.ascontiguousarray(spots["position"]).tobytes()
    assert np.frombuffer(cols["xyzobs.px.variance"][2], "<f8").tobytes() == \
        np.ascontiguousarray(spots["variance"]).tobytes()
    if with_shoeboxes:
        boxes = shoeboxes(cols["shoebox"][2], n)
        for s, (panel, bbox, data, mask, bg) in zip(spots, boxes):
            assert panel == 0 and list(bbox) == s["bbox"].tolist()
            px = pixels[int(s["first"]):int(s["first"]) + int(s["n_signal"])]
            x = px["index"] % width - bbox[0]
            y = px["index"] // width - bbox[2]
            z = px["frame"] - bbox[4]
            want_data = np.zeros_like(data)
            want_data[z, y, x] = px["value"].astype(np.float32)
            want_mask = np.zeros_like(mask)
            want_mask[z, y, x] = 5
            assert np.array_equal(data, want_data) and np.array_equal(mask, want_mask)
            assert not bg.any()


# -- the fixtures and the reader: no device needed ---------------------------

@pytest.mark.parametrize("name,mode,identifier,exp_id,with_shoeboxes", CASES)
def test_golden_tables_decode(name, mode, identifier, exp_id, with_shoeboxes):
    g = load_golden("small_series.npz")
    spots = as_records(g[f"spots_{mode}"], O.SPOT)
    pixels = as_records(g[f"pixels_{mode}"], O.PIXEL)
    check_table(os.path.join(GOLDEN, name), spots, pixels, g["frames"].shape[2], identifier,
                exp_id, with_shoeboxes)


@pytest.mark.skipif(not os.path.exists(CHECK_REFL), reason="the reference tree is not here")
@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_golden_tables_pass_check_refl(name):
    p = subprocess.run([sys.executable, CHECK_REFL, os.path.join(GOLDEN, name)],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stdout + p.stderr


# -- the writer, on the device ----------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("name,mode,identifier,exp_id,with_shoeboxes", CASES)
def test_byte_identical_to_the_reference(tmp_path, gpu_lib, name, mode, identifier, exp_id,
                                         with_shoeboxes):
    from dials_metal_spotfinder_b200 import refl
    g = load_golden("small_series.npz")
    spots = as_records(g[f"spots_{mode}"], O.SPOT)
    pixels = as_records(g[f"pixels_{mode}"], O.PIXEL)
    out = tmp_path / "strong.refl"
    refl.write(out, spots, pixels, g["frames"].shape[2], identifier=identifier,
               experiment_id=exp_id, shoeboxes=with_shoeboxes)
    assert out.read_bytes() == open(os.path.join(GOLDEN, name), "rb").read()


@pytest.mark.gpu
def test_series_grouped_on_the_device(tmp_path, gpu_lib):
    from dials_metal_spotfinder_b200 import refl, synth
    from dials_metal_spotfinder_b200.labeller import group
    series = synth.eiger_4m(frames=6)
    signals = [gpu_lib.find(series.frame(z)) for z in range(6)]
    h, w = series.height, series.width
    spots, pixels, counts = group(signals, h, w)
    assert len(spots) > 1000
    out = tmp_path / "strong.refl"
    refl.write(out, spots, pixels, w, identifier="series")
    check_table(out, spots, pixels, w, "series", 0, True)


@pytest.mark.gpu
def test_empty_table(tmp_path, gpu_lib):
    from dials_metal_spotfinder_b200 import refl
    out = tmp_path / "empty.refl"
    refl.write(out, np.zeros(0, O.SPOT), np.zeros(0, O.PIXEL), 100)
    t = read(out)
    assert t["nrows"] == 0 and all(c[1] == 0 and c[2] == b"" for c in t["columns"].values())


@pytest.mark.gpu
def test_refusals(tmp_path, gpu_lib):
    from dials_metal_spotfinder_b200 import refl
    from dials_metal_spotfinder_b200._lib import BadArgument, Refused
    g = load_golden("small_series.npz")
    spots = as_records(g["spots_3d"], O.SPOT).copy()
    pixels = as_records(g["pixels_3d"], O.PIXEL).copy()
    with pytest.raises(BadArgument):
        refl.write(tmp_path / "a.refl", spots, pixels, 0)
    bad = spots.copy()
    bad["first"][-1] = len(pixels)  # past the list
    with pytest.raises(Refused):
        refl.write(tmp_path / "b.refl", bad, pixels, 384)
    moved = pixels.copy()
    moved["frame"][int(spots["first"][0])] += 5  # outside its box
    with pytest.raises(Refused):
        refl.write(tmp_path / "c.refl", spots, moved, 384)
    with pytest.raises(Exception):
        refl.write(tmp_path / "no" / "such" / "dir.refl", spots, pixels, 384)
