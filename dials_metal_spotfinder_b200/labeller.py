"""dials_spots::Labeller (src/dials_spots.hh:108-126) on the device: 3D or
2D six-connected grouping of signal pixels across frames, and DIALS'
centroid, variance, summed intensity and filters, through the C ABI
(sf_labeller_*). Same methods, same order of results, same refusals."""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import (COUNT_NAMES, PIXEL, SIGNAL_PIXEL, SPOT, GroupOptions, lib, raise_for,
                   require_device)


@dataclass
class Options:
    """src/dials_spots.hh:81-95; the dials.find_spots defaults."""
    min_spot_size: int = 3
    max_spot_size: int = 1000
    max_separation: float = 2.0
    two_d: bool = False


class Labeller:
    def __init__(self, height: int, width: int, options: Options | None = None, **kw):
        require_device()
        opt = options or Options(**kw)
        c_opt = GroupOptions(opt.min_spot_size, opt.max_spot_size, opt.max_separation,
                             int(opt.two_d), 0)
        h = ctypes.c_void_p()
        raise_for(lib.sf_labeller_create(height, width, ctypes.byref(c_opt), ctypes.byref(h)),
                  "sf_labeller_create")
        self._h = h
        self.height, self.width, self.options = height, width, opt

    def close(self):
        if getattr(self, "_h", None):
            lib.sf_labeller_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def add(self, frame: int, signal: np.ndarray) -> None:
        """Labeller::add. Raises Refused (the reference's runtime_error) for a
        frame out of order, a pixel off the frame or pixels not ascending."""
        signal = np.ascontiguousarray(signal, dtype=SIGNAL_PIXEL)
        raise_for(lib.sf_labeller_add(self._h, int(frame), signal.ctypes.data if len(signal) else None,
                                      len(signal)), "add")

    def finish(self) -> None:
        raise_for(lib.sf_labeller_finish(self._h), "finish")

    def spots(self) -> np.ndarray:
        n = lib.sf_labeller_nspots(self._h)
        out = np.zeros(n, SPOT)
        raise_for(lib.sf_labeller_spots(self._h, out.ctypes.data if n else None, n), "spots")
        return out

    def pixels(self) -> np.ndarray:
        n = lib.sf_labeller_npixels(self._h)
        out = np.zeros(n, PIXEL)
        raise_for(lib.sf_labeller_pixels(self._h, out.ctypes.data if n else None, n), "pixels")
        return out

    def counts(self) -> dict:
        out = (ctypes.c_uint64 * 6)()
        raise_for(lib.sf_labeller_counts(self._h, out), "counts")
        return dict(zip(COUNT_NAMES, (int(v) for v in out)))

    def live(self) -> int:
        return int(lib.sf_labeller_live(self._h))


def group(signals, height, width, frames=None, **options):
    """Adds every frame's signal list in order, finishes, and returns
    (spots, pixels, counts)."""
    lab = Labeller(height, width, **options)
    numbers = range(len(signals)) if frames is None else frames
    for z, sig in zip(numbers, signals):
        lab.add(int(z), sig)
    lab.finish()
    result = lab.spots(), lab.pixels(), lab.counts()
    lab.close()
    return result
