"""The serving loop (include/spotfinder_b200.h, sf_server_*): live series on
one device, admitted by device-memory budget, frames submitted as detector
chunks and decoded, thresholded and grouped on the device as they arrive,
concurrent series overlapping on the device. Also a driver that replays
streams at fixed frame rates and reports latency percentiles, and the plain
per-frame GPU form (worker threads decoding on the host and calling sf_find
per frame, a labeller fed in frame order) run on the same streams for
comparison."""

from __future__ import annotations

import ctypes
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from ._lib import (COUNT_NAMES, PIXEL, SPOT, GroupOptions, ServerConfig, lib, raise_for,
                   require_device)
from .chunk import algorithm_code


class Busy(RuntimeError):
    """sf_server_open -2: the device-memory budget cannot hold the series now."""


class Server:
    def __init__(self, hbm_budget: int = 0, slots: int = 3, use_graph: bool = True):
        require_device()
        cfg = ServerConfig(hbm_budget, slots, int(use_graph))
        h = ctypes.c_void_p()
        raise_for(lib.sf_server_create(ctypes.byref(cfg), ctypes.byref(h)), "sf_server_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.sf_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def open(self, shape, dtype=np.uint16, first_frame=0, min_spot_size=3, max_spot_size=1000,
             max_separation=2.0, two_d=False) -> int:
        opt = GroupOptions(min_spot_size, max_spot_size, max_separation, int(two_d), 0)
        sid = ctypes.c_int(-1)
        status = lib.sf_server_open(self._h, shape[0], shape[1], np.dtype(dtype).itemsize,
                                    ctypes.byref(opt), first_frame, ctypes.byref(sid))
        if status == -2:
            raise Busy("the device-memory budget cannot hold this series now")
        raise_for(status, "sf_server_open")
        return sid.value

    def set_pixel_mask(self, series: int, mask: np.ndarray) -> None:
        """Before the series' first frame: nonzero = masked."""
        mask = np.ascontiguousarray(mask != 0, dtype=np.uint8)
        raise_for(lib.sf_server_set_pixel_mask(self._h, series, mask.ctypes.data),
                  "sf_server_set_pixel_mask")

    def submit(self, series: int, chunk: np.ndarray, algorithm="bslz4", timeout_s=1.0) -> bool:
        """False if no slot freed up within the timeout (the frame is dropped)."""
        status = lib.sf_server_submit(self._h, series, chunk.ctypes.data, len(chunk),
                                      algorithm_code(algorithm), int(timeout_s * 1e6))
        if status == -2:
            return False
        raise_for(status, "sf_server_submit")
        return True

    def finish(self, series: int) -> None:
        raise_for(lib.sf_server_close(self._h, series), "sf_server_close")

    def stats(self, series: int) -> dict:
        c = (ctypes.c_uint64 * 6)()
        o = (ctypes.c_uint64 * 4)()
        raise_for(lib.sf_server_stats(self._h, series, c, o), "sf_server_stats")
        d = dict(zip(COUNT_NAMES, (int(v) for v in c)))
        d.update(frames_done=int(o[0]), dropped=int(o[1]), device_bytes=int(o[2]),
                 closed=bool(o[3]))
        return d

    def _array(self, fn, series, dtype, *extra):
        n = ctypes.c_size_t(0)
        status = fn(self._h, series, *extra, None, 0, ctypes.byref(n))
        if status not in (0, -2):
            raise_for(status, fn.__name__)
        out = np.zeros(n.value, dtype)
        raise_for(fn(self._h, series, *extra, out.ctypes.data if n.value else None, n.value,
                     ctypes.byref(n)), fn.__name__)
        return out[: n.value]

    def spots(self, series: int) -> np.ndarray:
        return self._array(lib.sf_server_spots, series, SPOT)

    def pixels(self, series: int) -> np.ndarray:
        return self._array(lib.sf_server_pixels, series, PIXEL)

    def take(self, series: int, spot_capacity: int = 1 << 18, pixel_capacity: int = 1 << 24,
             out=None):
        """The spots (and their pixels) finished so far and still held, which
        the series then forgets (sf_server_take): call it as results are
        consumed so a long series does not hold every spot in host memory.
        `out` = (spot array, pixel array) to fill; returns views of the
        filled parts."""
        if out is None:
            out = (np.zeros(spot_capacity, SPOT), np.zeros(pixel_capacity, PIXEL))
        sp, px = out
        ns, npx = ctypes.c_size_t(0), ctypes.c_size_t(0)
        raise_for(lib.sf_server_take(self._h, series, sp.ctypes.data, len(sp), ctypes.byref(ns),
                                     px.ctypes.data, len(px), ctypes.byref(npx)), "sf_server_take")
        return sp[: ns.value], px[: npx.value]

    def signal_counts(self, series: int) -> np.ndarray:
        return self._array(lib.sf_server_signal_counts, series, np.uint32)

    def latencies_us(self, series: int, kind: str = "mask") -> np.ndarray:
        k = {"mask": 0, "grouped": 1, "spot": 2}[kind]
        return self._array(lib.sf_server_latencies, series, np.float64, k)


@dataclass
class Stream:
    """A live series: `chunks` (pre-encoded frames, cycled) submitted at
    `rate_hz` for `frames` frames."""
    shape: tuple
    chunks: list
    rate_hz: float
    frames: int
    algorithm: str = "bslz4"
    two_d: bool = False
    results: dict = field(default_factory=dict)


def percentiles(v):
    v = np.asarray(v, dtype=np.float64)
    if len(v) == 0:
        return {"p50": None, "p99": None, "max": None}
    return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99)),
            "max": float(v.max())}


class _NoGc:
    """Python's cyclic garbage collector off for the replay: a full
    collection in a process holding many arrays holds the interpreter lock
    for tens of milliseconds, which would stall the producer threads (the
    stand-ins for the detector) rather than anything being measured."""

    def __enter__(self):
        import gc
        self._was = gc.isenabled()
        gc.collect()
        gc.disable()
        return self

    def __exit__(self, *exc):
        import gc
        if self._was:
            gc.enable()


def drive(streams, hbm_budget=0, slots=3, use_graph=True, drain_s=0.05):
    """Replays every stream on its own thread at its frame rate through one
    Server and returns per-stream results (latencies in ms). A consumer
    thread per stream takes the finished spots every `drain_s` seconds (as
    a live writer of the reflection table would), so the series do not hold
    a whole acquisition's spots in host memory."""
    with _NoGc():
        return _drive(streams, hbm_budget, slots, use_graph, drain_s)


def _drive(streams, hbm_budget, slots, use_graph, drain_s):
    out = []
    with Server(hbm_budget=hbm_budget, slots=slots, use_graph=use_graph) as srv:
        ids = [srv.open(s.shape, two_d=s.two_d) for s in streams]
        late = [0] * len(streams)
        taken = [[0, 0] for _ in streams]
        running = threading.Event()
        running.set()
        bufs = [(np.zeros(1 << 18, SPOT), np.zeros(1 << 24, PIXEL)) for _ in streams]

        def consume(k):
            while True:
                stop = not running.is_set()
                while True:
                    sp, px = srv.take(ids[k], out=bufs[k])
                    taken[k][0] += len(sp)
                    taken[k][1] += len(px)
                    if len(sp) == 0:
                        break
                if stop:
                    return
                time.sleep(drain_s)

        consumers = [threading.Thread(target=consume, args=(k,)) for k in range(len(streams))]
        if drain_s:
            for t in consumers:
                t.start()
        t0 = time.perf_counter() + 0.05

        def produce(k):
            s = streams[k]
            period = 1.0 / s.rate_hz
            for i in range(s.frames):
                due = t0 + i * period
                while True:
                    now = time.perf_counter()
                    if now >= due:
                        break
                    time.sleep(min(due - now, 0.0005))
                if time.perf_counter() - due > period:
                    late[k] += 1
                srv.submit(ids[k], s.chunks[i % len(s.chunks)], s.algorithm, timeout_s=period)

        threads = [threading.Thread(target=produce, args=(k,)) for k in range(len(streams))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        wall = time.perf_counter() - t0
        for k in range(len(streams)):
            srv.finish(ids[k])
        running.clear()
        if drain_s:
            for t in consumers:
                t.join()
        for k, s in enumerate(streams):
            st = srv.stats(ids[k])
            out.append({
                "shape": list(s.shape), "rate_hz": s.rate_hz, "frames": s.frames,
                "frames_done": st["frames_done"], "dropped": st["dropped"],
                "late_submits": late[k], "sustained_fps": st["frames_done"] / wall,
                "frame_to_mask_ms": {k2: (v / 1e3 if v is not None else None) for k2, v in
                                     percentiles(srv.latencies_us(ids[k], "mask")).items()},
                "frame_to_grouped_ms": {k2: (v / 1e3 if v is not None else None) for k2, v in
                                        percentiles(srv.latencies_us(ids[k], "grouped")).items()},
                "frame_to_spot_ms": {k2: (v / 1e3 if v is not None else None) for k2, v in
                                     percentiles(srv.latencies_us(ids[k], "spot")).items()},
                "spots": int(st["accepted"]), "spots_taken_live": taken[k][0],
                "device_bytes": st["device_bytes"],
            })
    return out


def drive_plain(streams, workers: int | None = None, give_up_s: float = 5.0):
    """The plain per-frame GPU form on the same streams, threaded the way the
    reference CLI runs it with -gpu (src/find_spots.cc:472-591): per stream,
    `workers` threads take frames as they fall due, each decoding its chunk
    on the host and calling sf_find_u16 (the reference's gpu::find: upload,
    threshold, list back); one thread per stream adds the lists to a device
    labeller in frame order. A frame not started within `give_up_s` of its
    due time is dropped (the run stays bounded when the form cannot keep
    up). Latencies in ms from due times: frame-to-mask when the frame's list
    is on the host, frame-to-spot when the labeller has emitted the spot,
    from its last frame's due time."""
    with _NoGc():
        return _drive_plain(streams, workers, give_up_s)


def _drive_plain(streams, workers, give_up_s):
    
    import os
    import queue

    from . import chunk as C
    from . import find
    from .labeller import Labeller
    if workers is None:
        workers = min(8, max(2, (os.cpu_count() or 4) // (2 * max(1, len(streams)))))
    t0 = time.perf_counter() + 0.05
    results = [None] * len(streams)

    def run_stream(k):
        s = streams[k]
        period = 1.0 / s.rate_hz
        jobs = queue.Queue()
        done = {}
        cv = threading.Condition()
        mask = []

        def produce():
            for i in range(s.frames):
                due = t0 + i * period
                while True:
                    now = time.perf_counter()
                    if now >= due:
                        break
                    time.sleep(min(due - now, 0.0005))
                jobs.put(i)
            for _ in range(workers):
                jobs.put(None)

        def work():
            while True:
                i = jobs.get()
                if i is None:
                    return
                due = t0 + i * period
                sig = None
                if time.perf_counter() - due <= give_up_s:
                    img = C.decode(s.chunks[i % len(s.chunks)], s.shape, np.uint16, s.algorithm)
                    sig = find(img)
                t = time.perf_counter()
                with cv:
                    done[i] = (sig, t)
                    cv.notify_all()

        lab = Labeller(*s.shape, two_d=s.two_d)
        emitted = []  # (spots emitted so far, time) after each add
        dropped = 0
        threads = [threading.Thread(target=produce)]
        threads += [threading.Thread(target=work) for _ in range(workers)]
        for t in threads:
            t.start()
        for i in range(s.frames):
            with cv:
                cv.wait_for(lambda: i in done)
                sig, t_mask = done.pop(i)
            if sig is None:
                dropped += 1
                continue
            mask.append(t_mask - (t0 + i * period))
            lab.add(i, sig)
            emitted.append((int(lib.sf_labeller_nspots(lab._h)), time.perf_counter()))
        for t in threads:
            t.join()
        spots = lab.spots()
        lab.close()
        spot_lat, j = [], 0
        for n_after, t in emitted:
            while j < min(n_after, len(spots)):
                last = int(spots[j]["bbox"][5]) - 1
                spot_lat.append(t - (t0 + last * period))
                j += 1
        results[k] = (mask, spot_lat, dropped)

    threads = [threading.Thread(target=run_stream, args=(k,)) for k in range(len(streams))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t0
    out = []
    for k, s in enumerate(streams):
        mask, spot_lat, dropped = results[k]
        out.append({
            "shape": list(s.shape), "rate_hz": s.rate_hz, "frames": s.frames,
            "workers": workers, "dropped": dropped,
            "sustained_fps": (s.frames - dropped) / wall,
            "frame_to_mask_ms": {k2: (v * 1e3 if v is not None else None)
                                 for k2, v in percentiles(mask).items()},
            "frame_to_spot_ms": {k2: (v * 1e3 if v is not None else None)
                                 for k2, v in percentiles(spot_lat).items()},
        })
    return out
