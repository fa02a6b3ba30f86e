"""The serving loop (sf_server_*): a series' results are the same alone and
in a mix with another series whose frames arrive while its own are on the
device, and both equal the oracle (src/dext.cc threshold per frame, then
src/dials_spots.cc grouping of the series alone); series are admitted by
device-memory budget; the latency report is consistent."""

import threading

import numpy as np
import pytest

from conftest import same_spots
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def encode_all(frames, algorithm="bslz4"):
    from dials_metal_spotfinder_b200 import chunk as C
    return [C.encode(f, algorithm) for f in frames]


def series_a():
    from dials_metal_spotfinder_b200 import synth
    s = synth.small()
    return s, [s.frame(z) for z in range(s.frames)], False


def series_b():
    from dials_metal_spotfinder_b200 import synth
    s = synth.still((1062, 1028), frames=6)
    return s, [s.frame(z) for z in range(s.frames)], True


def results(srv, sid):
    st = srv.stats(sid)
    return srv.spots(sid), srv.pixels(sid), st, srv.signal_counts(sid)


def check_oracle(frames, two_d, spots, pixels, st, counts):
    signals = [O.dext(f)[1] for f in frames]
    assert list(counts) == [len(s) for s in signals]
    want = O.group(signals, *frames[0].shape, two_d=two_d)
    assert {k: st[k] for k in want.counts} == want.counts
    same_spots(spots, want.spots)
    assert pixels.tobytes() == want.pixels.tobytes()


def test_alone_and_in_the_mix(gpu_lib):
    from dials_metal_spotfinder_b200.serve import Server
    sa, fa, two_d_a = series_a()
    sb, fb, two_d_b = series_b()
    ca, cb = encode_all(fa), encode_all(fb, "lz4")

    with Server() as srv:
        a = srv.open(fa[0].shape, two_d=two_d_a)
        for c in ca:
            assert srv.submit(a, c, timeout_s=30)
        srv.finish(a)
        alone = results(srv, a)
    check_oracle(fa, two_d_a, *alone)

    with Server(slots=2) as srv:
        a = srv.open(fa[0].shape, two_d=two_d_a)
        b = srv.open(fb[0].shape, two_d=two_d_b)

        def feed(sid, chunks, algorithm):
            for c in chunks:
                assert srv.submit(sid, c, algorithm, timeout_s=30)

        ta = threading.Thread(target=feed, args=(a, ca, "bslz4"))
        tb = threading.Thread(target=feed, args=(b, cb, "lz4"))
        ta.start()
        tb.start()
        ta.join()
        tb.join()
        srv.finish(a)
        srv.finish(b)
        mixed_a, mixed_b = results(srv, a), results(srv, b)
    assert mixed_a[0].tobytes() == alone[0].tobytes()
    assert mixed_a[1].tobytes() == alone[1].tobytes()
    assert list(mixed_a[3]) == list(alone[3])
    check_oracle(fb, two_d_b, *mixed_b)


def test_admission_by_device_memory(gpu_lib):
    from dials_metal_spotfinder_b200.serve import Busy, Server
    shape = (2162, 2068)
    with Server() as srv:
        sid = srv.open(shape)
        one = srv.stats(sid)["device_bytes"]
        srv.finish(sid)
    assert one > 0
    with Server(hbm_budget=int(one * 1.5)) as srv:
        a = srv.open(shape)
        with pytest.raises(Busy):
            srv.open(shape)
        srv.finish(a)  # its memory goes back to the budget
        b = srv.open(shape)
        srv.finish(b)


def test_latency_report(gpu_lib):
    from dials_metal_spotfinder_b200 import synth
    from dials_metal_spotfinder_b200.serve import Stream, drive
    s = synth.eiger_4m(frames=8)
    chunks = encode_all([s.frame(z) for z in range(8)])
    out = drive([Stream((s.height, s.width), chunks, rate_hz=200.0, frames=40)])
    r = out[0]
    assert r["frames_done"] + r["dropped"] == 40
    for key in ("frame_to_mask_ms", "frame_to_grouped_ms", "frame_to_spot_ms"):
        assert 0 < r[key]["p50"] <= r[key]["p99"] <= r[key]["max"]
    assert r["frame_to_mask_ms"]["p50"] <= r["frame_to_grouped_ms"]["p50"]


def test_pixel_mask_in_a_served_series(gpu_lib):
    from dials_metal_spotfinder_b200.serve import Server
    s, frames, two_d = series_a()
    mask = np.zeros(frames[0].shape, bool)
    mask[100:130, 200:260] = True
    mask[:, 17] = True
    with Server() as srv:
        sid = srv.open(frames[0].shape, two_d=two_d)
        srv.set_pixel_mask(sid, mask)
        for c in encode_all(frames):
            assert srv.submit(sid, c, timeout_s=30)
        srv.finish(sid)
        got = results(srv, sid)
    stamped = []
    for f in frames:
        f = f.copy()
        f[mask] = 0xFFFF
        stamped.append(f)
    check_oracle(stamped, two_d, *got)


def test_u32_series_served(gpu_lib):
    from dials_metal_spotfinder_b200 import synth
    from dials_metal_spotfinder_b200.serve import Server
    s = synth.Series(300, 420, 8, 0x5EED0042, dtype=np.uint32, gaps=False, ring_r0=150.0,
                     spots_per_frame=40.0, intensity=(50.0, 2.0e6))
    frames = [s.frame(z) for z in range(s.frames)]
    with Server() as srv:
        sid = srv.open(frames[0].shape, dtype=np.uint32)
        for c in encode_all(frames):
            assert srv.submit(sid, c, timeout_s=30)
        srv.finish(sid)
        got = results(srv, sid)
    check_oracle(frames, False, *got)


def test_take_as_results_arrive(gpu_lib):
    """take() while frames are still being submitted, and once more after
    the close: the pieces, in order, are the oracle's spots and pixels, and
    what the series still holds afterwards is nothing; a spot array too
    short for the first held run takes nothing (Overflow)."""
    import dials_metal_spotfinder_b200 as sf
    from dials_metal_spotfinder_b200.serve import Server
    s, frames, two_d = series_a()
    chunks = encode_all(frames)
    got_spots, got_pixels = [], []
    with Server() as srv:
        sid = srv.open(frames[0].shape, two_d=two_d)
        for i, c in enumerate(chunks):
            assert srv.submit(sid, c, timeout_s=30)
            if i % 3 == 2:
                sp, px = srv.take(sid)
                got_spots.append(sp.copy())
                got_pixels.append(px.copy())
        srv.finish(sid)
        held = srv.spots(sid)
        if len(held):
            with pytest.raises(sf.Overflow):
                srv.take(sid, spot_capacity=0)
        sp, px = srv.take(sid)
        got_spots.append(sp.copy())
        got_pixels.append(px.copy())
        assert len(srv.spots(sid)) == 0 and len(srv.pixels(sid)) == 0
        st, counts = srv.stats(sid), srv.signal_counts(sid)
    check_oracle(frames, two_d, np.concatenate(got_spots), np.concatenate(got_pixels), st, counts)
