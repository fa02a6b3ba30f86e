"""Detector chunk formats (include/spotfinder_b200.h, sf_chunk_*; the
reference's decompress::image, src/decompress.hh:14-31): frames as the HDF5
filters store them, uncompressed ("raw"), "lz4" or "bslz4" (bitshuffle +
LZ4). encode() is the detector / replay side, decode() the host decoder;
decode_device() and Engine.upload_chunk() decode on the device."""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib, raise_for

ALGORITHMS = {"raw": 0, "lz4": 1, "bslz4": 2}


def algorithm_code(algorithm) -> int:
    if isinstance(algorithm, str):
        return ALGORITHMS[algorithm]
    return int(algorithm)


def encode(image: np.ndarray, algorithm="bslz4") -> np.ndarray:
    image = np.ascontiguousarray(image)
    if image.dtype not in (np.uint16, np.uint32) or image.ndim != 2:
        raise ValueError("frames are 2D uint16 or uint32")
    h, w = image.shape
    cap = lib.sf_chunk_bound(h, w, image.dtype.itemsize)
    out = np.empty(cap, np.uint8)
    n = ctypes.c_size_t(0)
    raise_for(lib.sf_chunk_encode(algorithm_code(algorithm), image.ctypes.data, h, w,
                                  image.dtype.itemsize, out.ctypes.data, cap, ctypes.byref(n)),
              "chunk.encode")
    return out[: n.value].copy()


def decode(chunk, shape, dtype=np.uint16, algorithm="bslz4") -> np.ndarray:
    chunk = np.ascontiguousarray(np.frombuffer(chunk, np.uint8) if isinstance(chunk, bytes)
                                 else chunk, dtype=np.uint8)
    h, w = shape
    out = np.empty((h, w), dtype)
    raise_for(lib.sf_chunk_decode(algorithm_code(algorithm), chunk.ctypes.data, len(chunk), h, w,
                                  np.dtype(dtype).itemsize, out.ctypes.data), "chunk.decode")
    return out


def decode_device(chunk, shape, dtype, device_ptr: int, pitch_bytes: int | None = None,
                  algorithm="bslz4") -> None:
    """Decodes `chunk` on the device into device memory at `device_ptr`
    (rows `pitch_bytes` apart, default the row length); waits for it."""
    chunk = np.ascontiguousarray(np.frombuffer(chunk, np.uint8) if isinstance(chunk, bytes)
                                 else chunk, dtype=np.uint8)
    h, w = shape
    eb = np.dtype(dtype).itemsize
    pitch = w * eb if pitch_bytes is None else int(pitch_bytes)
    raise_for(lib.sf_chunk_decode_device(algorithm_code(algorithm), chunk.ctypes.data, len(chunk),
                                         h, w, eb, device_ptr, pitch), "chunk.decode_device")
