"""The C++ drop-in for the reference's gpu:: interface (include/dext_gpu.hh,
shim/dext_gpu_b200.cc) and the templated Labeller facade
(include/spotfinder_b200.hpp), driven from C++ by tests/cpp/shim_check.cc the
way src/find_spots.cc drives the reference's: gpu::find<T> on host frames
(host_alloc'd), Labeller::add per frame, finish, spots/pixels/counts. The
results must equal the reference's golden outputs byte for byte, as in
tests/test_dext_gpu.cc:155-199 and tests/test_dials_spots.cc."""

import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, as_records, load_golden, same_spots
from oracle import oracle as O

CHECK = os.path.join(ROOT, "dials_metal_spotfinder_b200", "_build", "shim_check")


def run(*args, env=None, check=True):
    e = dict(os.environ)
    e.update(env or {})
    p = subprocess.run([CHECK, *map(str, args)], capture_output=True, text=True, env=e,
                       timeout=300)
    if check and p.returncode != 0:
        raise AssertionError(f"shim_check {args[0]} exited {p.returncode}: {p.stderr}")
    return p


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(CHECK):
        pytest.fail(f"{CHECK} is not built (make -C dials_metal_spotfinder_b200/csrc)")


# -- host logic: no device needed ------------------------------------------

def test_window_defaults_and_environment():
    p = run("info", env={"SPOTFINDER_GPU_STAGE0": "", "SPOTFINDER_GPU_STAGE2": ""})
    assert "stage0=direct stage2=tile" in p.stdout  # empty values warn, keep defaults
    p = run("info", env={"SPOTFINDER_GPU_STAGE0": "tile", "SPOTFINDER_GPU_STAGE2": "direct"})
    assert "stage0=tile stage2=direct" in p.stdout and p.stderr == ""
    p = run("info", env={"SPOTFINDER_GPU_STAGE2": "tiles"})
    assert "stage2=tile" in p.stdout
    assert "SPOTFINDER_GPU_STAGE2=tiles is not 'tile' or 'direct'" in p.stderr


def test_backend_names_cuda():
    assert "backend=CUDA" in run("info").stdout


# -- on the device ---------------------------------------------------------

def read_find(path):
    raw = open(path, "rb").read()
    status = int(np.frombuffer(raw[:4], np.int32)[0])
    n = int(np.frombuffer(raw[4:12], np.uint64)[0])
    return status, np.frombuffer(raw[12:12 + 16 * n], O.SIGNAL_PIXEL)


@pytest.mark.gpu
def test_available_on_the_device():
    assert "available=1" in run("info").stdout


@pytest.mark.gpu
def test_find_reference_frame_set(tmp_path):
    g = load_golden("threshold_u16.npz")
    for i, name in enumerate(g["names"]):
        img = g[f"frame{i}"]
        img.tofile(tmp_path / "in.raw")
        run("find16", img.shape[0], img.shape[1], tmp_path / "in.raw", tmp_path / "out.raw")
        status, got = read_find(tmp_path / "out.raw")
        assert status == 0, name
        assert got.tobytes() == as_records(g[f"signal{i}"], O.SIGNAL_PIXEL).tobytes(), name


@pytest.mark.gpu
def test_find_u32(tmp_path):
    g = load_golden("threshold_u32.npz")
    for i in range(2):
        img = g[f"frame{i}"]
        img.tofile(tmp_path / "in.raw")
        run("find32", img.shape[0], img.shape[1], tmp_path / "in.raw", tmp_path / "out.raw")
        status, got = read_find(tmp_path / "out.raw")
        assert status == 0
        assert got.tobytes() == as_records(g[f"signal{i}"], O.SIGNAL_PIXEL).tobytes()


@pytest.mark.gpu
def test_find_overflow_returns_minus_two_and_clears(tmp_path):
    img = np.full((8, 8), 0, np.uint16)
    img[3, 3] = 500  # one signal pixel; an 8 x 8 frame's list holds 8
    img.tofile(tmp_path / "in.raw")
    run("find16", 8, 8, tmp_path / "in.raw", tmp_path / "out.raw")
    status, got = read_find(tmp_path / "out.raw")
    assert status == 0 and len(got) == 1
    assert got.tobytes() == O.dext(img)[1].tobytes()
    img = np.zeros((8, 8), np.uint16)
    img[2:6, 2:6] = 3000  # 16 signal pixels: more than the list holds
    assert O.dext(img)[2] > 8
    img.tofile(tmp_path / "in.raw")
    run("find16", 8, 8, tmp_path / "in.raw", tmp_path / "out.raw")
    status, got = read_find(tmp_path / "out.raw")
    assert status == -2 and len(got) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("two_d", [False, True])
def test_series_through_the_facade(tmp_path, two_d):
    g = load_golden("small_series.npz")
    frames = g["frames"]
    nf, h, w = frames.shape
    frames.tofile(tmp_path / "frames.raw")
    run("series16", nf, h, w, 0, int(two_d), tmp_path / "frames.raw", tmp_path / "spots.raw",
        tmp_path / "pixels.raw", tmp_path / "counts.raw", tmp_path / "strong.refl")
    tag = "2d" if two_d else "3d"
    spots = np.fromfile(tmp_path / "spots.raw", O.SPOT)
    pixels = np.fromfile(tmp_path / "pixels.raw", O.PIXEL)
    counts = np.fromfile(tmp_path / "counts.raw", np.uint64)
    same_spots(spots, as_records(g[f"spots_{tag}"], O.SPOT))
    assert pixels.tobytes() == as_records(g[f"pixels_{tag}"], O.PIXEL).tobytes()
    assert list(counts[:6]) == list(g[f"counts_{tag}"])
    assert counts[6] == 0  # finish() leaves nothing live
    if not two_d:  # the reference's refl::write of the same spots, identifier "golden"
        assert (tmp_path / "strong.refl").read_bytes() == \
            open(os.path.join(ROOT, "tests", "golden", "refl_small.refl"), "rb").read()


@pytest.mark.gpu
def test_concurrent_workers(tmp_path):
    from dials_metal_spotfinder_b200 import synth
    img = synth.eiger_4m(frames=1).frame(0)
    img.tofile(tmp_path / "in.raw")
    p = run("threads16", img.shape[0], img.shape[1], 8, 3, tmp_path / "in.raw")
    assert "ok" in p.stdout


@pytest.mark.gpu
def test_out_of_order_frame_throws_and_changes_nothing():
    p = run("order", 16, 16)
    assert p.stdout.startswith("refused:")
