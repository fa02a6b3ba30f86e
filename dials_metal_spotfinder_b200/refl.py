"""Writing a DIALS reflection table (include/spotfinder_b200.h, sf_refl_write;
the reference's refl::write, src/refl.hh:72-74): byte-identical output, with
the shoebox column built on the device."""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import PIXEL, SPOT, ReflOptions, lib, raise_for, require_device


def write(path: str, spots: np.ndarray, pixels: np.ndarray, width: int, identifier: str = "",
          experiment_id: int = 0, panel: int = 0, shoeboxes: bool = True) -> None:
    """Raises BadArgument (-1), Refused (-4: pixels past the list or outside
    their box, a column over 4 GB) or DeviceError (-3: I/O or device)."""
    require_device()
    spots = np.ascontiguousarray(spots, dtype=SPOT)
    pixels = np.ascontiguousarray(pixels, dtype=PIXEL)
    opt = ReflOptions(panel, experiment_id, int(bool(shoeboxes)), identifier.encode())
    status = lib.sf_refl_write(str(path).encode(), spots.ctypes.data if len(spots) else None,
                               len(spots), pixels.ctypes.data if len(pixels) else None,
                               len(pixels), int(width), ctypes.byref(opt))
    raise_for(status, "refl.write")
