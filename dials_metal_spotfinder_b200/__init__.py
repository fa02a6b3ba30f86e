"""B200-native spot finding: the DIALS dispersion-extended threshold, 3D
six-connected grouping and the centroid/intensity/shoebox pass, as CUDA
kernels for sm_100a behind a C ABI (include/spotfinder_b200.h).

This module is the Python mirror of the reference's host interface
(graeme-winter/dials-metal-spotfinder ``src/dext_gpu.hh`` and
``src/dials_spots.hh``): the same names, argument meaning and error
behaviour, calling the C ABI through ctypes. There is no CPU fallback: a
missing library or device raises.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import (COUNT_NAMES, PIXEL, SIGNAL_PIXEL, SPOT, BadArgument, DeviceError,
                   GroupOptions, Overflow, Refused, lib, raise_for, require_device)

__all__ = [
    "SIGNAL_PIXEL", "PIXEL", "SPOT", "COUNT_NAMES", "BadArgument", "Overflow",
    "DeviceError", "Refused", "backend", "available", "memory_free", "find",
    "find_status", "profile_stages", "last_stage_times", "HostBuffer",
]


def backend() -> str:
    """gpu::backend() (src/dext_gpu.hh:28)."""
    return lib.sf_backend().decode()


def available() -> bool:
    """gpu::available() (src/dext_gpu.hh:126)."""
    return bool(lib.sf_available())


def memory_free() -> int:
    """gpu::memory_free() (src/dext_gpu.hh:131)."""
    return int(lib.sf_memory_free())


def _capacity(image: np.ndarray) -> int:
    h, w = image.shape
    return h * w * image.dtype.itemsize // 16


def find_status(image: np.ndarray, out: np.ndarray | None = None):
    """gpu::find<T> with the reference's return codes (src/dext_gpu.hh:141-158).

    Returns ``(status, signal)``: status 0, -1 (bad argument) or -2 (more
    signal than the device list holds); ``signal`` is the SignalPixel array
    ascending by index (empty unless status is 0). A device failure raises
    DeviceError, as the reference's std::runtime_error does.

    ``out``, a SIGNAL_PIXEL array of at least height*width*itemsize/16
    records, receives the list and ``signal`` is then a view into it.
    """
    if image is None or image.ndim != 2 or image.dtype not in (np.uint16, np.uint32):
        return -1, np.zeros(0, SIGNAL_PIXEL)
    image = np.ascontiguousarray(image)
    h, w = image.shape
    if h == 0 or w == 0:
        return -1, np.zeros(0, SIGNAL_PIXEL)
    cap = max(_capacity(image), 1)
    given = out is not None and len(out) >= cap
    if given:
        if out.dtype != SIGNAL_PIXEL or out.ndim != 1 or not out.flags.c_contiguous:
            return -1, np.zeros(0, SIGNAL_PIXEL)
    else:
        out = np.empty(cap, SIGNAL_PIXEL)
    found = ctypes.c_size_t(0)
    fn = lib.sf_find_u16 if image.dtype == np.uint16 else lib.sf_find_u32
    status = fn(image.ctypes.data, h, w, out.ctypes.data, cap, ctypes.byref(found))
    if status == -3:
        raise_for(status, "find")
    if status != 0:
        return status, np.zeros(0, SIGNAL_PIXEL)
    # into the caller's array (a HostBuffer's page-locked one copies fastest)
    # a view of the filled part; otherwise a compact copy
    return 0, out[: found.value] if given else out[: found.value].copy()


def find(image: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
    """Threshold one frame; raises BadArgument / Overflow / DeviceError.
    `out` as for find_status."""
    status, signal = find_status(image, out)
    raise_for(status, "find")
    return signal


def profile_stages(on: bool | None = None) -> bool:
    """gpu::profile_stages (src/dext_gpu.hh:112-113)."""
    if on is not None:
        lib.sf_profile_stages(int(bool(on)))
    return bool(lib.sf_profile_stages_enabled())


def last_stage_times() -> dict:
    """gpu::last_stage_times (src/dext_gpu.hh:116): milliseconds per stage."""
    out = (ctypes.c_double * 6)()
    lib.sf_last_stage_times(out)
    return dict(zip(("upload", "stage0", "stage1", "stage2", "copy", "sort"), list(out)))


class HostBuffer:
    """Page-locked host memory (gpu::host_alloc / host_free, src/dext_gpu.hh:
    133-139) viewed as a numpy array."""

    def __init__(self, shape, dtype):
        dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * dtype.itemsize
        self._ptr = lib.sf_host_alloc(max(nbytes, 1))
        self._free = lib.sf_host_free  # still bound when module globals are gone at exit
        if not self._ptr:
            raise DeviceError("sf_host_alloc failed")
        buf = (ctypes.c_char * max(nbytes, 1)).from_address(self._ptr)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def close(self):
        if getattr(self, "_ptr", None):
            self.array = None
            self._free(self._ptr)
            self._ptr = None

    def __del__(self):
        self.close()
