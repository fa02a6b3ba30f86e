"""The batched engine's autotuner (include/spotfinder_b200.h, sf_tune): a
timed search on the current device for frames per launch, warps per block,
threshold task height and threshold blocks per SM, on sample frames of one
shape. The result goes
to a tuner file that engines created without explicit tuning read. The
reference chooses its own stage windows by measurement the same way
(src/dext_gpu.cc:18-37, tests/bench_dext_gpu.cc:242-337)."""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import TuneOptions, TuneResult, lib, raise_for, require_device


def tune(frames, min_frames: int = 8, max_frames: int = 32, steps: int = 4,
         grouping: bool = True, use_cache: bool = True, hbm_budget: int = 0,
         cache_path: str | None = None) -> dict:
    """Tunes the engine for the shape and type of `frames` (a sequence of
    consecutive frames, cycled into the trial batches). Returns the chosen
    frames_per_launch, warps_per_block, seg_rows (for that many frames),
    seg_ratio, blocks_per_sm (0: as many as fit), us_per_frame, candidates
    (configurations timed) and from_cache (read from the tuner file,
    nothing timed)."""
    require_device()
    frames = [np.ascontiguousarray(f) for f in frames]
    if not frames:
        raise ValueError("tune needs at least one sample frame")
    shape, dtype = frames[0].shape, frames[0].dtype
    if dtype not in (np.uint16, np.uint32) or len(shape) != 2:
        raise ValueError("frames are 2D uint16 or uint32")
    if any(f.shape != shape or f.dtype != dtype for f in frames):
        raise ValueError("sample frames must share one shape and type")
    ptrs = (ctypes.c_void_p * len(frames))(*[f.ctypes.data for f in frames])
    opt = TuneOptions(min_frames, max_frames, steps, int(grouping), int(use_cache), 0,
                      hbm_budget, cache_path.encode() if cache_path else None)
    out = TuneResult()
    raise_for(lib.sf_tune(dtype.itemsize, shape[0], shape[1], ptrs, len(frames),
                          ctypes.byref(opt), ctypes.byref(out)), "sf_tune")
    d = out.as_dict()
    d["from_cache"] = bool(d["from_cache"])
    return d
