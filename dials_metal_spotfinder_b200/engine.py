"""The batched engine (include/spotfinder_b200.h, sf_engine_*): many frames
of equal or uneven shapes thresholded per launch from device-resident slots,
optionally replayed from CUDA graphs. Per frame, results are exactly
``find()``'s (the reference's gpu::find, src/dext_gpu.hh:141-158)."""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import (COUNT_NAMES, PIXEL, SIGNAL_PIXEL, SPOT, EngineConfig, GroupOptions,
                   TuneResult, lib, raise_for, require_device)


class Engine:
    """seg_rows and warps_per_block 0 (the default): the tuner file's choice
    for this frame shape on this device (see tune.py), else the cost model's
    task height and 2 warps per block (1 for 32-bit pixels)."""

    def __init__(self, shapes, dtype=np.uint16, slots=1, seg_rows=0, warps_per_block=0,
                 blocks_per_sm=0):
        require_device()
        self.dtype = np.dtype(dtype)
        if self.dtype not in (np.uint16, np.uint32):
            raise ValueError("pixels are uint16 or uint32")
        self.shapes = [tuple(int(v) for v in s) for s in shapes]
        n = len(self.shapes)
        heights = (ctypes.c_int32 * n)(*[h for h, _ in self.shapes])
        widths = (ctypes.c_int32 * n)(*[w for _, w in self.shapes])
        cfg = EngineConfig(seg_rows, warps_per_block, blocks_per_sm, slots)
        handle = ctypes.c_void_p()
        status = lib.sf_engine_create(self.dtype.itemsize, n, heights, widths,
                                      ctypes.byref(cfg), ctypes.byref(handle))
        raise_for(status, "sf_engine_create")
        self._h = handle
        self.slots = slots
        self._keep = {}

    def close(self):
        if getattr(self, "_h", None):
            lib.sf_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def nframes(self):
        return len(self.shapes)

    def info(self) -> dict:
        out = (ctypes.c_int64 * 8)()
        raise_for(lib.sf_engine_info(self._h, out), "sf_engine_info")
        keys = ("seg_rows", "warps_per_block", "grid_blocks", "tasks", "slots",
                "device_bytes", "pitch", "capacity")
        return dict(zip(keys, list(out)))

    def tuning(self) -> dict:
        """frames_per_launch, warps_per_block, seg_rows, blocks_per_sm and
        from_cache (the tuning came from the tuner file)."""
        out = TuneResult()
        raise_for(lib.sf_engine_tuning(self._h, ctypes.byref(out)), "sf_engine_tuning")
        d = out.as_dict()
        d["from_cache"] = bool(d["from_cache"])
        return {k: d[k] for k in ("frames_per_launch", "warps_per_block", "seg_rows",
                                  "blocks_per_sm", "from_cache")}

    def upload(self, slot: int, frame: int, image: np.ndarray) -> None:
        """Asynchronous host-to-device copy; keep `image` alive (and unchanged)
        until the next synchronize()."""
        if image.dtype != self.dtype or image.shape != self.shapes[frame]:
            raise ValueError("frame shape or type does not match the engine")
        if not image.flags.c_contiguous:
            raise ValueError("frames must be C-contiguous")
        raise_for(lib.sf_engine_upload(self._h, slot, frame, image.ctypes.data), "upload")

    def upload_device(self, slot: int, frame: int, ptr: int, pitch_bytes: int) -> None:
        raise_for(lib.sf_engine_upload_device(self._h, slot, frame, ptr, pitch_bytes),
                  "upload_device")

    def upload_chunk(self, slot: int, frame: int, chunk: np.ndarray, algorithm="bslz4") -> None:
        """A compressed frame (see chunk.py), decoded on the device into the
        slot; keep `chunk` alive until the next synchronize()."""
        from .chunk import algorithm_code
        chunk = np.ascontiguousarray(chunk, dtype=np.uint8)
        raise_for(lib.sf_engine_upload_chunk(self._h, slot, frame, chunk.ctypes.data, len(chunk),
                                             algorithm_code(algorithm)), "upload_chunk")

    def upload_chunks(self, slot: int, chunks, frames=None, algorithm="bslz4") -> None:
        """Several compressed frames at once (chunk k to frame frames[k], or
        to frame k): their framing is checked on host threads in parallel,
        all before any is enqueued. Keep the chunks alive until the next
        synchronize()."""
        from .chunk import algorithm_code
        chunks = [np.ascontiguousarray(c, dtype=np.uint8) for c in chunks]
        n = len(chunks)
        ptrs = (ctypes.c_void_p * max(n, 1))(*[c.ctypes.data for c in chunks])
        sizes = (ctypes.c_size_t * max(n, 1))(*[len(c) for c in chunks])
        fr = None
        if frames is not None:
            if len(frames) != n:
                raise ValueError("one frame number per chunk")
            fr = (ctypes.c_int * max(n, 1))(*[int(f) for f in frames])
        # Alive until the copies are done: one list per slot, dropped by
        # synchronize(), so a slot still in flight keeps its chunks.
        self._keep[slot] = chunks
        raise_for(lib.sf_engine_upload_chunks(self._h, slot, n, fr, ptrs, sizes,
                                              algorithm_code(algorithm)), "upload_chunks")

    def set_pixel_mask(self, frame: int, mask) -> None:
        """Frame `frame`'s pixel mask (nonzero = masked), stamped as the masked
        sentinel before every threshold; None clears it."""
        if mask is None:
            raise_for(lib.sf_engine_set_pixel_mask(self._h, frame, None), "set_pixel_mask")
            return
        mask = np.ascontiguousarray(mask != 0, dtype=np.uint8)
        if mask.shape != self.shapes[frame]:
            raise ValueError("mask shape does not match the frame")
        raise_for(lib.sf_engine_set_pixel_mask(self._h, frame, mask.ctypes.data), "set_pixel_mask")

    def run(self, slot: int = 0) -> None:
        raise_for(lib.sf_engine_run(self._h, slot), "run")

    def use_graph(self, on: bool = True) -> None:
        raise_for(lib.sf_engine_use_graph(self._h, int(on)), "use_graph")

    def synchronize(self) -> None:
        raise_for(lib.sf_engine_synchronize(self._h), "synchronize")
        self._keep.clear()

    def counts(self, slot: int = 0) -> np.ndarray:
        out = np.zeros(self.nframes, np.uint32)
        raise_for(lib.sf_engine_counts(self._h, slot, out.ctypes.data), "counts")
        return out

    def signal_status(self, slot: int, frame: int, out: np.ndarray | None = None):
        """(status, list) of one frame of the slot's last run. With `out` (a
        SIGNAL_PIXEL array of at least the frame's capacity, height * width *
        itemsize / 16 records; page-locked copies fastest) the list is copied
        into it and a view of the filled part returned."""
        h, w = self.shapes[frame]
        cap = max(h * w * self.dtype.itemsize // 16, 1)
        given = out is not None
        if given:
            if out.dtype != SIGNAL_PIXEL or out.ndim != 1 or not out.flags.c_contiguous \
                    or len(out) < cap:
                raise ValueError("out must be a contiguous SIGNAL_PIXEL array of the "
                                 "frame's capacity")
        else:
            out = np.empty(cap, SIGNAL_PIXEL)
        found = ctypes.c_size_t(0)
        status = lib.sf_engine_signal(self._h, slot, frame, out.ctypes.data, len(out),
                                      ctypes.byref(found))
        if status == -3:
            raise_for(status, "signal")
        if status != 0:
            return status, np.zeros(0, SIGNAL_PIXEL)
        return 0, out[: found.value] if given else out[: found.value].copy()

    def signals(self, slot: int, out: np.ndarray | None = None):
        """Every frame's list of the slot's last run: (lists, counts), the
        lists back to back in frame order in `out` (or a new array) and
        returned as views. Overflow if a frame overflowed or they do not
        fit."""
        counts = np.zeros(self.nframes, np.uint32)
        if out is None:
            cap = sum(max(h * w * self.dtype.itemsize // 16, 1) for h, w in self.shapes)
            out = np.empty(cap, SIGNAL_PIXEL)
        elif out.dtype != SIGNAL_PIXEL or out.ndim != 1 or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous SIGNAL_PIXEL array")
        raise_for(lib.sf_engine_signals(self._h, slot, out.ctypes.data, len(out),
                                        counts.ctypes.data), "signals")
        ends = np.cumsum(counts.astype(np.int64))
        starts = ends - counts
        return [out[a:b] for a, b in zip(starts, ends)], counts

    def signal(self, slot: int, frame: int, out: np.ndarray | None = None) -> np.ndarray:
        status, sig = self.signal_status(slot, frame, out)
        raise_for(status, "signal")
        return sig

    # -- CUDA events on the engine's compute stream ------------------------
    def record(self, mark: int) -> None:
        raise_for(lib.sf_engine_record(self._h, mark), "record")

    def elapsed_ms(self, start: int, end: int) -> float:
        ms = ctypes.c_float(0)
        raise_for(lib.sf_engine_elapsed(self._h, start, end, ctypes.byref(ms)), "elapsed")
        return float(ms.value)

    def profile(self, on: bool = True) -> None:
        raise_for(lib.sf_engine_profile(self._h, int(on)), "profile")

    def stage_totals(self) -> dict:
        out = (ctypes.c_double * 4)()
        raise_for(lib.sf_engine_stage_totals(self._h, out), "stage_totals")
        return {"runs": int(out[0]), "threshold_ms": out[1], "place_ms": out[2],
                "group_ms": out[3]}

    # -- grouping inside each run ------------------------------------------
    def enable_grouping(self, first_frame: int = 0, min_spot_size=3, max_spot_size=1000,
                        max_separation=2.0, two_d=False, carry_capacity=0) -> None:
        """The batch's frames of one shape are one series; each run's frames of
        a series are its next consecutive frames, grouped on the device right
        after their threshold by that series' labeller (the reference's
        Labeller::add per frame, src/dials_spots.cc:57-145)."""
        opt = GroupOptions(min_spot_size, max_spot_size, max_separation, int(two_d), 0)
        raise_for(lib.sf_engine_enable_grouping(self._h, ctypes.byref(opt), int(first_frame),
                                                int(carry_capacity)), "enable_grouping")

    def nseries(self) -> int:
        return int(lib.sf_engine_nseries(self._h))

    def series_shape(self, series: int = 0):
        h, w = ctypes.c_int32(0), ctypes.c_int32(0)
        raise_for(lib.sf_engine_series_shape(self._h, series, ctypes.byref(h), ctypes.byref(w)),
                  "series_shape")
        return int(h.value), int(w.value)

    def group_counts(self, series: int = 0):
        out = (ctypes.c_uint64 * 6)()
        live = ctypes.c_uint64(0)
        raise_for(lib.sf_engine_series_counts(self._h, series, out, ctypes.byref(live)),
                  "group_counts")
        return dict(zip(COUNT_NAMES, (int(v) for v in out))), int(live.value)

    def _records(self, fn, series, dtype, out, what):
        n = ctypes.c_size_t(0)
        if out is not None:
            if out.dtype != dtype or out.ndim != 1 or not out.flags.c_contiguous:
                raise ValueError(f"out must be a contiguous 1-D array of {what} records")
            raise_for(fn(self._h, series, out.ctypes.data if len(out) else None, len(out),
                         ctypes.byref(n)), what)
            return out[:n.value]
        status = fn(self._h, series, None, 0, ctypes.byref(n))
        if status not in (0, -2):
            raise_for(status, what)
        out = np.zeros(n.value, dtype)
        raise_for(fn(self._h, series, out.ctypes.data if n.value else None, n.value,
                     ctypes.byref(n)), what)
        return out

    def spots(self, series: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """Spots of a series finished by the last run (or by finish()).

        With `out` (a SPOT array, best a HostBuffer's page-locked one) the
        records are copied into it and a view of the filled part returned;
        Overflow if it is too short."""
        return self._records(lib.sf_engine_series_spots, series, SPOT, out, "spots")

    def pixels(self, series: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """The finished spots' pixels, in spot order; `out` as for spots()."""
        return self._records(lib.sf_engine_series_pixels, series, PIXEL, out, "pixels")

    def finish(self) -> None:
        raise_for(lib.sf_engine_finish(self._h), "finish")
